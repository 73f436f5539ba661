/*
 * dedisp_b200.h -- extensions of the dedisp C interface (no counterpart in
 * the reference unless noted). All entry points take the ordinary
 * dedisp_plan handle from dedisp.h and use plain C types only.
 */
#ifndef DEDISP_B200_H_INCLUDE_GUARD
#define DEDISP_B200_H_INCLUDE_GUARD

#include "dedisp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* TDD kernel selection for DEDISP_DEDISP / DEDISP_TDD plans. AUTO uses the
 * tiled shared-memory kernel when the killmask holds only 0/1 values; PLAIN
 * is the one-thread-per-sample-pair baseline (the reference's decomposition,
 * src/tdd/dedisperse/TDDKernel.cu:133-151). */
typedef enum {
    DEDISP_B200_TDD_AUTO = 0,
    DEDISP_B200_TDD_PLAIN = 1,
    DEDISP_B200_TDD_TILED = 2
} dedisp_b200_tdd_kernel;

dedisp_error dedisp_b200_set_tdd_kernel(dedisp_plan plan, int kernel);

/* Runs the plan's device work on a caller-provided cudaStream_t (NULL
 * restores the plan's own stream). */
dedisp_error dedisp_b200_set_stream(dedisp_plan plan, void* cuda_stream);

/* Device-time instrumentation of execute(): when enabled, the next calls
 * record CUDA events around the preprocessing (transpose / unpack + FFT) and
 * the dedispersion kernels on the plan's stream. */
dedisp_error dedisp_b200_set_timing(dedisp_plan plan, int enable);
dedisp_error dedisp_b200_get_timing(dedisp_plan plan, float* kernel_ms, float* prep_ms,
                                    int* launches, int* variant);

/* The C functions of dedisp.h report every failure inside the plan classes
 * as DEDISP_UNKNOWN_ERROR, like the reference (src/clib/dedisp.cpp:520-523).
 * This returns the specific code of the most recent such failure in the
 * calling thread and copies its message (may be NULL). */
dedisp_error dedisp_b200_last_error(char* msg, dedisp_size len);

/* FDD options (DEDISP_FDD plans):
 *   segmented      -1 follow USE_SEGMENTED, 0 whole series, 1 segmented
 *   timeseries     whole-series output: 0 spectrum (default), 1 time series
 *   precision      0 FP32 CUDA cores, 1 3xBF16 tensor-core GEMM
 *   round_delays   0 truncate (reference FDD), 1 round half to even (TDD)
 *   segment_nfft   0 reference doubling rule, else a power of two */
dedisp_error dedisp_b200_set_fdd_options(dedisp_plan plan, int segmented, int timeseries,
                                         int precision, int round_delays,
                                         dedisp_size segment_nfft);

/* Measures the device's 32-bit integer add throughput (lane-adds per
 * second) with a kernel of independent add chains on every SM. Used to
 * state the roofline of the integer-bound TDD kernel. */
dedisp_error dedisp_b200_alu_probe(int device, double* lane_adds_per_s);

/* Floats per DM row that execute() writes for nsamps input samples. */
dedisp_size dedisp_b200_output_row_length(dedisp_plan plan, dedisp_size nsamps);

#ifdef __cplusplus
}
#endif

#endif /* DEDISP_B200_H_INCLUDE_GUARD */
