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

/* Tile shape of the tiled TDD kernel (8-bit input: DMs per block, samples
 * per thread); variant in [0, dedisp_b200_tdd_variant_count(in_nbits)).
 * Every variant computes the same bit-exact sums; they differ in speed.
 * Other input widths have a single shape and ignore the setting. */
dedisp_error dedisp_b200_set_tdd_variant(dedisp_plan plan, int variant);
int dedisp_b200_tdd_variant_count(dedisp_size in_nbits);

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

/* Allocation-free time-domain dedispersion. No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc -- real-time pipelines that forbid
 * allocation once started (an allocation can block on the driver for an
 * unbounded time), or processes whose device memory belongs to another
 * allocator.
 * Computes what a DEDISP_TDD plan with DEDISP_DEVICE_POINTERS computes (same
 * bit-exact output) for a plan described by (nchans, dt, f0, df), the host
 * DM list and killmask (NULL: all channels; values must be 0 or 1), reading
 * d_in (device, time-major, in_stride bytes per sample) and writing d_out
 * (device, dm_count rows of out_stride bytes), then waits for `stream`.
 *
 * It allocates no device memory: its scratch is a fixed 64 MiB array in the
 * library (plus small tables for up to 16384 DMs and 8192 channels), held by
 * every GPU that loads the library until the process exits. Requests whose
 * channel-major copy, (nchans + 1) x (nsamps rounded up + padding) samples,
 * does not fit are rejected with DEDISP_MEM_ALLOC_FAILED. The first call on
 * a device looks up the arrays' device addresses (cudaGetSymbolAddress) and
 * should therefore come before any stream capture on that device. All calls
 * share the scratch: calls that overlap on the GPU race. On failure,
 * dedisp_b200_noalloc_last_message() describes the reason. */
dedisp_error dedisp_b200_tdd_execute_noalloc(
    dedisp_size nchans, dedisp_float dt, dedisp_float f0, dedisp_float df,
    const dedisp_float* dm_list, dedisp_size dm_count, const dedisp_bool* killmask,
    dedisp_size nsamps, const dedisp_byte* d_in, dedisp_size in_nbits, dedisp_size in_stride,
    dedisp_byte* d_out, dedisp_size out_nbits, dedisp_size out_stride, void* stream);
const char* dedisp_b200_noalloc_last_message(void);

/* Floats per DM row that execute() writes for nsamps input samples. */
dedisp_size dedisp_b200_output_row_length(dedisp_plan plan, dedisp_size nsamps);

#ifdef __cplusplus
}
#endif

#endif /* DEDISP_B200_H_INCLUDE_GUARD */
