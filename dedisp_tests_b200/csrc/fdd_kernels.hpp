// Launch interface of the Fourier-domain (FDD) kernels.
//
// Layouts (complex values are float2 {re, im}):
//   x   [nchans][x_pitch] float      unpacked input, channel-major, zero past
//                                    the last sample
//   X   [nchans*nseg][bin_pitch]     spectrum of segment s of channel c in row
//                                    c*nseg + s, bins 0..nfft/2
//   Xt  [nbins][nseg][nact]          bin-major, active channels only, killmask
//                                    multiplier applied
//   Yt  [nbins][nseg][ndm]           dedispersed spectra, bin-major
//   Y   [ndm*nseg][bin_pitch]        dedispersed spectra, DM-major
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

namespace dedisp {
namespace kern {

// Two-level table of W_N^t = exp(-2*pi*i*t/N), t = hi*LO + lo (LO = 256):
// W = hi_tab[t >> 8] * lo_tab[t & 255]. N must be a multiple of 256.
struct TwiddleTable {
    const float2* lo;  // 256 entries
    const float2* hi;  // N / 256 entries
    unsigned n;
};

// Host tables of W_N^t (two-level, FP64-computed): lo[t] t < 256,
// hi[h] = W_N^{256 h}, h < N / 256.
void make_twiddle_tables(size_t n, std::vector<float2>& lo, std::vector<float2>& hi);

// Bin order of a spectrum row. Q <= 1: natural (bin k at position k).
// Q > 1 (transforms of N = 16384 Q points, M = N / 2 = P Q, P = 8192): bin
// k < M at position (k mod Q) P + k / Q, bin M at position M.
struct BinMap {
    unsigned P = 8192;
    unsigned Q = 1;
    size_t M = 0;
};

// Radices of the Q-point passes (product Q), from fftq_radices.
struct QRadices {
    int n = 0;
    int r[24] = {};
};
QRadices fftq_radices(unsigned Q);
constexpr size_t kFqMaxSmem = 200 * 1024;

// 8-bit or float32 time-major input -> x rows, scaled (FDDGPUPlan.cpp:472,
// unpack_kernel.cuh:60): 8-bit ((float)v - 127.5f) * scale, float v * scale.
void launch_fdd_unpack(const uint8_t* in, size_t in_stride, int in_nbits, size_t nsamps,
                       size_t nchans, float scale, float* x, size_t x_pitch, size_t x_len,
                       cudaStream_t s);

// Largest real transform length handled in one CTA (shared memory).
constexpr int kMaxSmemFft = 32768;   // one CTA per transform up to this length
constexpr int kMaxFft = 1 << 20;      // four-step transforms up to this length

// Forward real FFT of nfft samples (power of two, 32..kMaxSmemFft) for every
// (channel, segment): input x[c][seg*seg_stride + n], output X row
// c*nseg + seg, bins 0..nfft/2.
// nfft up to 32768: one CTA per transform; 65536 .. 2^20: four-step
// (column and row passes through `scratch`, fft_scratch_elems complex values).
void launch_fft_r2c(const float* x, size_t x_pitch, size_t nchans, size_t nseg,
                    size_t seg_stride, int nfft, float2* X, size_t bin_pitch,
                    const TwiddleTable& tw, float2* scratch, cudaStream_t s);
size_t fft_scratch_elems(int nfft, size_t rows);

// Inverse real FFT (normalised by 1/nfft) of every row r = dm*nseg + seg of
// Y (bins 0..nfft/2); samples n < keep of segment seg go to
// out[dm][seg*keep + n] when that index is < out_len.
// Y is overwritten (the four-step path prepares it in place).
void launch_fft_c2r(float2* Y, size_t bin_pitch, size_t ndm, size_t nseg, int nfft,
                    float* out, size_t out_stride, size_t keep, size_t out_len,
                    const TwiddleTable& tw, float2* scratch, cudaStream_t s);

// Transforms of N = 16384 Q real points for any Q (not a power-of-two
// length, or above 2^20): X rows (bins 0..N/2) in the BinMap order of
// fdd_binmap(N). tw: table for N; twp: table for 16384; wq: W_Q^x, x < Q
// (fftq_wq_table); scratch: fft_scratch_elems complex values.
bool fftq_length(size_t nfft);  // handled by this path (N = 16384 Q, Q >= 1)
BinMap fdd_binmap(size_t nfft); // the order launch_fft_r2c / _q leaves X in
std::vector<float2> fftq_wq_table(unsigned Q);
void launch_fft_r2c_q(const float* x, size_t x_pitch, size_t nchans, size_t nseg, size_t seg_stride,
                      size_t nfft, float2* X, size_t bin_pitch, const TwiddleTable& tw,
                      const TwiddleTable& twp, const float2* wq, float2* scratch, cudaStream_t s);
// Y rows in the BinMap order (overwritten).
void launch_fft_c2r_q(float2* Y, size_t bin_pitch, size_t ndm, size_t nseg, size_t nfft, float* out,
                      size_t out_stride, size_t keep, size_t out_len, const TwiddleTable& tw,
                      const TwiddleTable& twp, const float2* wq, float2* scratch, cudaStream_t s);

// X -> Xt over active channels (chan[j], multiplier km[j]); X rows in the
// order `map`.
void launch_fdd_to_binmajor(const float2* X, size_t bin_pitch, size_t nseg, size_t nbins,
                            const int32_t* chan, const float* km, int nact, float2* Xt,
                            const BinMap& map, cudaStream_t s);

// Yt -> Y (DM-major spectra); with spectrum_out, writes the first nspec bins
// straight into output rows instead: out[dm][2k], out[dm][2k+1].
void launch_fdd_to_dmmajor(const float2* Yt, size_t nseg, size_t ndm, size_t nbins,
                           float2* Y, size_t bin_pitch, const BinMap& map, cudaStream_t s);
void launch_fdd_spectrum_out(const float2* Yt, size_t ndm, size_t nspec, float* out,
                             size_t out_stride, cudaStream_t s);

// Plain FP32 phasor multiply-accumulate (CUDA cores):
//   Yt[k][seg][dm] = sum_j exp(+2*pi*i*(k*d(dm,j) mod N)/N) * Xt[k][seg][j]
// with d = (int)(dm * delay[j]) (round_delays: __float2uint_rn).
struct MacArgs {
    const float2* Xt;
    float2* Yt;
    const float* dms;
    const float* delay_act;   // delay of each active channel
    int nact;
    int ndm;
    int nseg;
    size_t nbins;
    unsigned nfft;
    int round_delays;
    TwiddleTable tw;
};
void launch_fdd_mac_plain(const MacArgs& a, cudaStream_t s);
// One segment (whole series): per-bin phasor table over delays 0..dmax (the
// largest delay index of the plan's DMs and channels), same sums as the
// tiled kernel. fdd_mac_series_fits: dmax known and the tables fit.
bool fdd_mac_series_fits(int dmax, unsigned nfft, int nact);
void launch_fdd_mac_series(const MacArgs& a, int dmax, cudaStream_t s);

}  // namespace kern
}  // namespace dedisp
