/*
 * oracle.h -- CPU restatement of the dedisp reference arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the shipped library links or calls
 * this code. It exists so that tests/, the smoke check and the CPU-baseline
 * leg of bench.py can check (and time) the CUDA path against an independent,
 * plainly written CPU version of the same algorithm.
 *
 * Every function cites the reference file:line it restates (paths are relative
 * to the root of the reference project, piyushplcr7/dedisp_tests).
 *
 * Parity pins: the delay table, DM list, max delay and the TDD epilogue are
 * checked bit-for-bit against the reference's own sources compiled on the host
 * (oracle/ref/, outputs in oracle/_ref/), and the full TDD loop against golden
 * outputs of the reference's GPU TDDPlan/DedispPlan stored in tests/golden/.
 *
 * Floating point: build with -ffp-contract=off, no -ffast-math, SSE (x86-64)
 * arithmetic, so every float/double operation rounds exactly once, in the
 * same order as the reference expression.
 */
#ifndef DEDISP_ORACLE_H
#define DEDISP_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Plan setup ---------------------------------------------------------------*/

/* src/Plan.cpp:29-36,109-119: FP32 delay table (samples per unit DM) with the
 * channel width forced negative. */
void orc_delay_table(size_t nchans, float dt, float f0, float df, float* out);

/* src/Plan.cpp:45-70: Levin DM-list recurrence in double, stored as float.
 * Writes at most `cap` values; returns the number of DMs the reference would
 * produce (which may exceed cap), or (size_t)-1 if the recurrence stalls
 * (the reference loops forever in that case). */
size_t orc_generate_dm_list(float dm_start, float dm_end, double dt, double ti,
                            double f0, double df, size_t nchans, double tol,
                            float* out, size_t cap);

/* src/Plan.cpp:85-86,152-153 and src/clib/dedisp.cpp:333:
 * size_t(float(dm * delay) + 0.5); negative products clamp to 0. */
size_t orc_max_delay(float dm_last, float delay_last);

/* src/tdd/dedisperse/dedisperse_kernel.cuh:163-165: __float2uint_rn(dm*delay)
 * (round half to even, saturating to [0, 2^32-1], NaN -> 0). */
uint32_t orc_delay_rn(float dm, float delay);

/* src/fdd/dedisperse/fdd_kernel.cuh:226-229: (int)(dm*delay), truncation. */
int32_t orc_delay_trunc(float dm, float delay);

/* src/tdd/dedisperse/dedisperse_kernel.cuh:45-87: the TDD output epilogue.
 * Writes one output value of out_nbits (8, 16 or 32=float) at out. */
void orc_scale_output(uint64_t sum, int in_nbits, int out_nbits, size_t nchans,
                      void* out);

/* TDD brute force -----------------------------------------------------------
 * src/tdd/dedisperse/dedisperse_kernel.cuh:98-198 (same sums as the legacy
 * src/dedisp/dedisperse/dedisperse_kernel.cuh:100-248):
 *   out[dm][t] = scale( sum_c killmask[c] * sub(in, t + rn(dm*delay[c]), c) )
 * `in` is time-major, rows of in_stride bytes, channels packed LSB-first in
 * little-endian 32-bit words (src/clib/dedisp.h:336-345). Output rows are
 * out_stride bytes apart, nsamps_out samples each. Samples t+delay beyond
 * nsamps read as zero. nthreads<=0 uses all OpenMP threads. */
int orc_tdd(const uint8_t* in, size_t nsamps, size_t in_stride, int in_nbits,
            size_t nchans, const float* delay_table, const int32_t* killmask,
            const float* dm_list, size_t dm_count, uint8_t* out, int out_nbits,
            size_t out_stride, size_t nsamps_out, int nthreads);

/* Same sums, without the epilogue: raw integer sums as uint64 [dm][t]. */
int orc_tdd_sums(const uint8_t* in, size_t nsamps, size_t in_stride,
                 int in_nbits, size_t nchans, const float* delay_table,
                 const int32_t* killmask, const float* dm_list,
                 size_t dm_count, uint64_t* sums, size_t nsamps_out,
                 int nthreads);

/* FDD (FP64) ----------------------------------------------------------------
 * Sample map: 8-bit -> ((float)v - 127.5f) * (float)(1.0/nchans)
 * (src/fdd/unpack/unpack_kernel.cuh:60, src/fdd/FDDGPUPlan.cpp:472);
 * in_nbits 32 -> IEEE float32 sample * (float)(1.0/nchans).
 * Delays: trunc (FDD GPU, fdd_kernel.cuh:226-229) if round_delays==0,
 * else round-half-even as in TDD. */

/* Unpack FDD input to float32 channel-major x[c][t] (c < nchans, t < nsamps). */
int orc_fdd_unpack(const uint8_t* in, size_t nsamps, size_t in_stride,
                   int in_nbits, size_t nchans, float* x);

/* Time-series output (upstream EXPORT_DEDISP_TIME_SERIES whole-series mode,
 * src/fdd/FDDGPUPlan.cpp:618-636, and the segmented mode after stitching,
 * chunk.cpp:80-110): y[dm][t] = sum_c km[c] * x[c][t + d(dm,c)], FP64,
 * t < nsamps_out; samples past nsamps read as zero. */
int orc_fdd_timeseries(const float* x, size_t nsamps, size_t nchans,
                       const float* delay_table, const int32_t* killmask,
                       const float* dm_list, size_t dm_count, int round_delays,
                       double* y, size_t nsamps_out, int nthreads);

/* Spectrum output (this fork's default, src/fdd/FDDGPUPlan.cpp:85-93,
 * 394-400): Y[dm] = FFT_N( z ), z[n] = sum_c km[c] * x[c][(n + d) mod N],
 * x zero-padded to N = nfft. Writes the first N/2 bins, interleaved re/im,
 * as doubles: spec[dm][2k], spec[dm][2k+1]. */
int orc_fdd_spectrum(const float* x, size_t nsamps, size_t nchans,
                     const float* delay_table, const int32_t* killmask,
                     const float* dm_list, size_t dm_count, int round_delays,
                     size_t nfft, double* spec, int nthreads);

/* In-place FP64 complex FFT of any length (radix-2, Bluestein otherwise);
 * sign -1 forward (e^{-2 pi i k n / N}), +1 inverse (unnormalised). */
int orc_fft(double* re, double* im, size_t n, int sign);

/* Geometry helpers restating the reference sizing rules. */
/* FDDGPUPlan.cpp:89: round_up(nsamp + max_delay, 16384). */
size_t orc_fdd_nfft_spectrum(size_t nsamp, size_t max_delay);
/* FDDGPUPlan.cpp:742-768: nfft doubling rule, nsamp_good, nchunk. */
void orc_fdd_segment_geometry(size_t nsamp, size_t max_delay, size_t* nfft,
                              size_t* nsamp_good, size_t* nchunk);

#ifdef __cplusplus
}
#endif

#endif /* DEDISP_ORACLE_H */
