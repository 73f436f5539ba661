/*
 * oracle.c -- CPU restatement of the dedisp reference arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h). Not linked into the product.
 * Build: -O2 -ffp-contract=off -fno-fast-math -fopenmp (oracle/Makefile).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Plan setup                                                                */
/* ------------------------------------------------------------------------ */

void orc_delay_table(size_t nchans, float dt, float f0, float df, float* out)
{
    /* src/Plan.cpp:31: the table always uses a negative channel width. */
    df = -fabsf(df);
    for (size_t c = 0; c < nchans; ++c) {
        /* src/Plan.cpp:114-117, every operation in the reference's type:
         * a, b and (a*a - b*b) in float; 4.15e3/dt and the product in double,
         * rounded once to float on store. */
        float a = 1.f / (f0 + (float)c * df);
        float b = 1.f / f0;
        float aa = a * a;
        float bb = b * b;
        float diff = aa - bb;
        double k = 4.15e3 / (double)dt;
        out[c] = (float)(k * (double)diff);
    }
}

size_t orc_generate_dm_list(float dm_start, float dm_end, double dt, double ti,
                            double f0, double df, size_t nchans, double tol,
                            float* out, size_t cap)
{
    /* src/Plan.cpp:54-60 (Levin's recurrence, all in double). */
    dt *= 1e6;
    double f = (f0 + ((double)(nchans / 2) - 0.5) * df) * 1e-3;
    double tol2 = tol * tol;
    double a = 8.3 * df / (f * f * f);
    double a2 = a * a;
    double b2 = a2 * ((double)(nchans * nchans) / 16.0);
    double c = (dt * dt + ti * ti) * (tol2 - 1.0);

    size_t n = 0;
    float back = dm_start;
    if (n < cap) out[n] = back;
    ++n;
    /* src/Plan.cpp:63-69: the list is stored as float and the previous
     * element is read back from the float list. */
    while (back < dm_end) {
        double prev = (double)back;
        double prev2 = prev * prev;
        double k = c + tol2 * a2 * prev2;
        double dm = ((b2 * prev + sqrt(-a2 * b2 * prev2 + (a2 + b2) * k)) /
                     (a2 + b2));
        float next = (float)dm;
        if (!(next > back)) return (size_t)-1; /* reference would spin forever */
        if (n < cap) out[n] = next;
        ++n;
        back = next;
        if (n > ((size_t)1 << 26)) return (size_t)-1;
    }
    return n;
}

size_t orc_max_delay(float dm_last, float delay_last)
{
    /* float product, then + 0.5 in double, then truncation to size_t. */
    float p = dm_last * delay_last;
    double v = (double)p + 0.5;
    if (!(v > 0.0)) return 0;
    return (size_t)v;
}

uint32_t orc_delay_rn(float dm, float delay)
{
    float x = dm * delay;
    if (!(x > 0.0f)) return 0u;               /* negatives and NaN saturate to 0 */
    if (x >= 4294967295.5f) return 0xFFFFFFFFu;
    return (uint32_t)rintf(x);                /* default rounding: half to even */
}

int32_t orc_delay_trunc(float dm, float delay)
{
    float x = dm * delay;
    if (x != x) return 0;
    if (x >= 2147483647.0f) return 2147483647;
    if (x <= -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)x;                        /* C conversion truncates */
}

/* ------------------------------------------------------------------------ */
/* TDD epilogue: src/tdd/dedisperse/dedisperse_kernel.cuh:29-87               */
/* ------------------------------------------------------------------------ */

static uint32_t max_value_u32(int nbits)
{
    /* max_value<NBITS>::value = ((1u<<(NBITS-1))-1)*2+1, in unsigned int */
    return ((((uint32_t)1) << (nbits - 1)) - 1u) * 2u + 1u;
}

void orc_scale_output(uint64_t sum, int in_nbits, int out_nbits, size_t nchans,
                      void* out)
{
    float in_range = (float)max_value_u32(in_nbits);
    float out_range = (out_nbits == 32) ? 1.f : (float)max_value_u32(out_nbits);
    /* (3.f * 1024.f) / 255.f / 16.f, evaluated in float */
    float f1 = 3.f * 1024.f;
    float f2 = f1 / 255.f;
    float factor = f2 / 16.f;
    float fsum = (in_nbits == 32) ? (float)sum : (float)(uint32_t)sum;
    float num = fsum * out_range;
    float den = in_range * (float)nchans;
    float q = num / den;
    float scaled = q * factor;
    if (out_nbits == 32) {
        *(float*)out = scaled;
    } else {
        /* min(max(scaled, 0.), out_range) evaluated in double, stored back
         * to float, then truncated by the integer cast. */
        double s = (double)scaled;          /* sums are >= 0, never NaN */
        double m = s > 0.0 ? s : 0.0;
        double r = m < (double)out_range ? m : (double)out_range;
        float rf = (float)r;
        if (out_nbits == 8) *(uint8_t*)out = (uint8_t)rf;
        else *(uint16_t*)out = (uint16_t)rf;
    }
}

/* ------------------------------------------------------------------------ */
/* Input access                                                              */
/* ------------------------------------------------------------------------ */

/* One sample of channel c at row t: the c%cpw-th subword (LSB first) of the
 * c/cpw-th little-endian 32-bit word of the row
 * (dedisperse_kernel.cuh:38-43,151-179). */
static inline uint32_t get_sample(const uint8_t* in, size_t in_stride,
                                  int nbits, size_t t, size_t c)
{
    const uint8_t* row = in + t * in_stride;
    size_t bit = c * (size_t)nbits;
    size_t byte = bit >> 3;
    switch (nbits) {
    case 32:
        return (uint32_t)row[byte] | ((uint32_t)row[byte + 1] << 8) |
               ((uint32_t)row[byte + 2] << 16) | ((uint32_t)row[byte + 3] << 24);
    case 16:
        return (uint32_t)row[byte] | ((uint32_t)row[byte + 1] << 8);
    case 8:
        return row[byte];
    default:
        return ((uint32_t)row[byte] >> (bit & 7)) & ((1u << nbits) - 1u);
    }
}

static int valid_nbits(int nbits)
{
    return nbits == 1 || nbits == 2 || nbits == 4 || nbits == 8 ||
           nbits == 16 || nbits == 32;
}

/* ------------------------------------------------------------------------ */
/* TDD brute force                                                           */
/* ------------------------------------------------------------------------ */

#define ORC_TBLOCK 4096

int orc_tdd_sums(const uint8_t* in, size_t nsamps, size_t in_stride,
                 int in_nbits, size_t nchans, const float* delay_table,
                 const int32_t* killmask, const float* dm_list,
                 size_t dm_count, uint64_t* sums, size_t nsamps_out,
                 int nthreads)
{
    if (!valid_nbits(in_nbits)) return -1;
    if ((nchans * (size_t)in_nbits) % 32 != 0) return -2;
    if (nsamps_out > nsamps) return -3;
    if (dm_count == 0 || nsamps_out == 0) return 0;

    /* Channel-major copy of the input, one uint32 per sample. */
    uint32_t* x = (uint32_t*)malloc(nchans * nsamps * sizeof(uint32_t));
    if (!x) return -4;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (long long cc = 0; cc < (long long)nchans; ++cc) {
        size_t c = (size_t)cc;
        uint32_t* xr = x + c * nsamps;
        for (size_t t = 0; t < nsamps; ++t)
            xr[t] = get_sample(in, in_stride, in_nbits, t, c);
    }

    size_t ntb = (nsamps_out + ORC_TBLOCK - 1) / ORC_TBLOCK;
    long long njobs = (long long)(dm_count * ntb);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (long long job = 0; job < njobs; ++job) {
        size_t dm_idx = (size_t)job / ntb;
        size_t t0 = ((size_t)job % ntb) * ORC_TBLOCK;
        size_t nt = nsamps_out - t0 < ORC_TBLOCK ? nsamps_out - t0 : ORC_TBLOCK;
        float dm = dm_list[dm_idx];
        uint64_t* srow = sums + dm_idx * nsamps_out + t0;
        if (in_nbits == 32) {
            uint64_t acc[ORC_TBLOCK];
            memset(acc, 0, sizeof(acc));
            for (size_t c = 0; c < nchans; ++c) {
                uint32_t km = (uint32_t)killmask[c];
                if (km == 0) continue;
                size_t d = orc_delay_rn(dm, delay_table[c]);
                const uint32_t* xr = x + c * nsamps;
                for (size_t i = 0; i < nt; ++i) {
                    size_t t = t0 + i + d;
                    uint32_t v = t < nsamps ? xr[t] : 0u;
                    acc[i] += (uint64_t)(uint32_t)(km * v);
                }
            }
            for (size_t i = 0; i < nt; ++i) srow[i] = acc[i];
        } else {
            /* dedisp_word accumulation: wraps modulo 2^32 like the kernel */
            uint32_t acc[ORC_TBLOCK];
            memset(acc, 0, sizeof(acc));
            for (size_t c = 0; c < nchans; ++c) {
                uint32_t km = (uint32_t)killmask[c];
                if (km == 0) continue;
                size_t d = orc_delay_rn(dm, delay_table[c]);
                const uint32_t* xr = x + c * nsamps;
                if (t0 + nt + d <= nsamps) {
                    const uint32_t* src = xr + t0 + d;
                    if (km == 1) {
                        for (size_t i = 0; i < nt; ++i) acc[i] += src[i];
                    } else {
                        for (size_t i = 0; i < nt; ++i) acc[i] += km * src[i];
                    }
                } else {
                    for (size_t i = 0; i < nt; ++i) {
                        size_t t = t0 + i + d;
                        uint32_t v = t < nsamps ? xr[t] : 0u;
                        acc[i] += km * v;
                    }
                }
            }
            for (size_t i = 0; i < nt; ++i) srow[i] = acc[i];
        }
    }
    free(x);
    return 0;
}

int orc_tdd(const uint8_t* in, size_t nsamps, size_t in_stride, int in_nbits,
            size_t nchans, const float* delay_table, const int32_t* killmask,
            const float* dm_list, size_t dm_count, uint8_t* out, int out_nbits,
            size_t out_stride, size_t nsamps_out, int nthreads)
{
    if (out_nbits != 8 && out_nbits != 16 && out_nbits != 32) return -5;
    if (dm_count == 0 || nsamps_out == 0) return 0;
    uint64_t* sums = (uint64_t*)malloc(dm_count * nsamps_out * sizeof(uint64_t));
    if (!sums) return -4;
    int rc = orc_tdd_sums(in, nsamps, in_stride, in_nbits, nchans, delay_table,
                          killmask, dm_list, dm_count, sums, nsamps_out,
                          nthreads);
    if (rc == 0) {
        size_t ob = (size_t)out_nbits / 8;
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
        for (long long dd = 0; dd < (long long)dm_count; ++dd) {
            size_t d = (size_t)dd;
            for (size_t t = 0; t < nsamps_out; ++t)
                orc_scale_output(sums[d * nsamps_out + t], in_nbits, out_nbits,
                                 nchans, out + d * out_stride + t * ob);
        }
    }
    free(sums);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* FDD (FP64)                                                                */
/* ------------------------------------------------------------------------ */

int orc_fdd_unpack(const uint8_t* in, size_t nsamps, size_t in_stride,
                   int in_nbits, size_t nchans, float* x)
{
    if (in_nbits != 1 && in_nbits != 2 && in_nbits != 4 && in_nbits != 8 && in_nbits != 16 &&
        in_nbits != 32)
        return -1;
    /* FDDGPUPlan.cpp:472 passes 1.0/nchan to a float parameter. */
    float scale = (float)(1.0 / (double)nchans);
    /* 8-bit: (v - 127.5) * scale (unpack_kernel.cuh:60); other packed widths
       (an extension of this library) are centred at (2^nbits - 1) / 2. */
    float mid = in_nbits == 32 ? 0.f : (float)((1u << in_nbits) - 1u) * 0.5f;
    for (size_t c = 0; c < nchans; ++c) {
        for (size_t t = 0; t < nsamps; ++t) {
            float v;
            if (in_nbits == 8) {
                uint32_t u = in[t * in_stride + c];
                v = ((float)u - 127.5f) * scale;
            } else if (in_nbits == 32) {
                float f;
                memcpy(&f, in + t * in_stride + 4 * c, 4);
                v = f * scale;
            } else if (in_nbits == 16) {
                const uint8_t* p = in + t * in_stride + 2 * c;
                uint32_t u = (uint32_t)p[0] | ((uint32_t)p[1] << 8);
                v = ((float)u - mid) * scale;
            } else {
                size_t bit = c * (size_t)in_nbits;
                uint32_t u = (in[t * in_stride + bit / 8] >> (bit % 8)) & ((1u << in_nbits) - 1u);
                v = ((float)u - mid) * scale;
            }
            x[c * nsamps + t] = v;
        }
    }
    return 0;
}

static long long fdd_delay(float dm, float delay, int round_delays)
{
    if (round_delays) return (long long)orc_delay_rn(dm, delay);
    return (long long)orc_delay_trunc(dm, delay);
}

int orc_fdd_timeseries(const float* x, size_t nsamps, size_t nchans,
                       const float* delay_table, const int32_t* killmask,
                       const float* dm_list, size_t dm_count, int round_delays,
                       double* y, size_t nsamps_out, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (long long dd = 0; dd < (long long)dm_count; ++dd) {
        size_t d = (size_t)dd;
        double* yr = y + d * nsamps_out;
        for (size_t t = 0; t < nsamps_out; ++t) yr[t] = 0.0;
        for (size_t c = 0; c < nchans; ++c) {
            if (killmask[c] == 0) continue;
            double km = (double)killmask[c];
            long long dl = fdd_delay(dm_list[d], delay_table[c], round_delays);
            const float* xr = x + c * nsamps;
            for (size_t t = 0; t < nsamps_out; ++t) {
                long long s = (long long)t + dl;
                if (s >= 0 && (size_t)s < nsamps) yr[t] += km * (double)xr[s];
            }
        }
    }
    return 0;
}

/* Iterative radix-2 FFT, n a power of two. */
static void fft_pow2(double* re, double* im, size_t n, int sign)
{
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        size_t half = len >> 1;
        for (size_t k = 0; k < half; ++k) {
            /* exact-argument twiddle: 2*pi*k/len computed in double */
            double ang = (double)sign * 2.0 * M_PI * (double)k / (double)len;
            double wr = cos(ang), wi = sin(ang);
            for (size_t i = k; i < n; i += len) {
                size_t j = i + half;
                double xr = re[j] * wr - im[j] * wi;
                double xi = re[j] * wi + im[j] * wr;
                re[j] = re[i] - xr; im[j] = im[i] - xi;
                re[i] += xr; im[i] += xi;
            }
        }
    }
}

int orc_fft(double* re, double* im, size_t n, int sign)
{
    if (n <= 1) return 0;
    if ((n & (n - 1)) == 0) { fft_pow2(re, im, n, sign); return 0; }
    /* Bluestein: chirp z-transform through a power-of-two convolution. */
    size_t m = 1;
    while (m < 2 * n - 1) m <<= 1;
    double* ar = (double*)calloc(m, sizeof(double));
    double* ai = (double*)calloc(m, sizeof(double));
    double* br = (double*)calloc(m, sizeof(double));
    double* bi = (double*)calloc(m, sizeof(double));
    double* wr = (double*)malloc(n * sizeof(double));
    double* wi = (double*)malloc(n * sizeof(double));
    if (!ar || !ai || !br || !bi || !wr || !wi) {
        free(ar); free(ai); free(br); free(bi); free(wr); free(wi);
        return -4;
    }
    for (size_t k = 0; k < n; ++k) {
        /* k^2 mod 2n keeps the chirp argument exact */
        unsigned long long k2 = ((unsigned long long)k * k) % (2ull * n);
        double ang = (double)sign * M_PI * (double)k2 / (double)n;
        wr[k] = cos(ang); wi[k] = sin(ang);
    }
    for (size_t k = 0; k < n; ++k) {
        ar[k] = re[k] * wr[k] - im[k] * wi[k];
        ai[k] = re[k] * wi[k] + im[k] * wr[k];
    }
    br[0] = wr[0]; bi[0] = -wi[0];
    for (size_t k = 1; k < n; ++k) {
        br[k] = wr[k]; bi[k] = -wi[k];
        br[m - k] = wr[k]; bi[m - k] = -wi[k];
    }
    fft_pow2(ar, ai, m, -1);
    fft_pow2(br, bi, m, -1);
    for (size_t k = 0; k < m; ++k) {
        double r = ar[k] * br[k] - ai[k] * bi[k];
        double i = ar[k] * bi[k] + ai[k] * br[k];
        ar[k] = r; ai[k] = i;
    }
    fft_pow2(ar, ai, m, +1);
    for (size_t k = 0; k < n; ++k) {
        double r = ar[k] / (double)m, i = ai[k] / (double)m;
        re[k] = r * wr[k] - i * wi[k];
        im[k] = r * wi[k] + i * wr[k];
    }
    free(ar); free(ai); free(br); free(bi); free(wr); free(wi);
    return 0;
}

int orc_fdd_spectrum(const float* x, size_t nsamps, size_t nchans,
                     const float* delay_table, const int32_t* killmask,
                     const float* dm_list, size_t dm_count, int round_delays,
                     size_t nfft, double* spec, int nthreads)
{
    if (nfft < nsamps || nfft % 2) return -1;
    int rc = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (long long dd = 0; dd < (long long)dm_count; ++dd) {
        size_t d = (size_t)dd;
        double* zr = (double*)calloc(nfft, sizeof(double));
        double* zi = (double*)calloc(nfft, sizeof(double));
        if (!zr || !zi) { rc = -4; free(zr); free(zi); continue; }
        for (size_t c = 0; c < nchans; ++c) {
            if (killmask[c] == 0) continue;
            double km = (double)killmask[c];
            long long dl = fdd_delay(dm_list[d], delay_table[c], round_delays);
            long long N = (long long)nfft;
            long long sh = ((dl % N) + N) % N;
            const float* xr = x + c * nsamps;
            /* z[n] += x[(n + dl) mod N] for the nsamps nonzero samples */
            for (size_t s = 0; s < nsamps; ++s) {
                long long n = ((long long)s - sh + N) % N;
                zr[n] += km * (double)xr[s];
            }
        }
        orc_fft(zr, zi, nfft, -1);
        double* out = spec + d * nfft;
        for (size_t k = 0; k < nfft / 2; ++k) {
            out[2 * k] = zr[k];
            out[2 * k + 1] = zi[k];
        }
        free(zr); free(zi);
    }
    return rc;
}

size_t orc_fdd_nfft_spectrum(size_t nsamp, size_t max_delay)
{
    size_t n = nsamp + max_delay;
    return ((n + 16383) / 16384) * 16384;
}

void orc_fdd_segment_geometry(size_t nsamp, size_t max_delay, size_t* nfft,
                              size_t* nsamp_good, size_t* nchunk)
{
    /* FDDGPUPlan.cpp:742,762-768: nsamp_dm = ceil(max_delay); double nfft
     * from 16384 while nfft*(1-0.8) < nsamp_dm (0.8 is a float constant). */
    size_t n = 16384;
    unsigned int nsamp_dm = (unsigned int)ceil((double)(float)max_delay);
    float min_eff = 0.8f;
    while (((double)n * (1.0 - (double)min_eff)) < (double)nsamp_dm) n *= 2;
    *nfft = n;
    *nsamp_good = n - nsamp_dm;
    *nchunk = (size_t)ceilf((float)nsamp / (float)(n - nsamp_dm));
}
