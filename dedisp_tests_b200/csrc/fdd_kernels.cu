// Fourier-domain dedispersion kernels for sm_100a (FP32 forms).
//
//   fdd_unpack          time-major input -> channel-major float rows
//   fft_r2c / fft_c2r   batched real FFTs, one CTA per transform, the whole
//                       transform resident in shared memory; radix-16 DIF
//                       passes in registers; real<->complex via the
//                       half-length complex transform
//   to_binmajor         X[c][seg][k] -> Xt[k][seg][j] (active channels,
//                       killmask multiplier folded in)
//   mac_plain           per-bin complex GEMM on CUDA cores: phasors
//                       W(k*d mod N) generated on chip from exact integer
//                       phase indices and a two-level twiddle table
//   to_dmmajor / spectrum_out
//
// Conventions follow the reference: forward transform e^{-2 pi i k n/N}
// (cuFFT R2C, FDDGPUPlan.cpp:160-175), phasor e^{+2 pi i k d/N} with
// d = (int)(dm * delay[c]) (fdd_kernel.cuh:226-235), inverse scaled by 1/N
// (fdd_kernel.cuh:262-273).
#include "fdd_kernels.hpp"

#include <cmath>

#include "runtime.hpp"

namespace dedisp {
namespace kern {
namespace {

__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

// Bin at row position p of the BinMap order.
__device__ __forceinline__ size_t qbin(size_t p, const BinMap& m)
{
    return (m.Q <= 1 || p >= m.M) ? p : (size_t)m.Q * (p & (m.P - 1)) + p / m.P;
}

// exp(-2 pi i t / 32), t = 0..15 (forward); conjugated for the inverse.
__device__ __forceinline__ float2 w32(int t, bool inv)
{
    const float c[16] = {1.0f, 0.98078528040323044f, 0.92387953251128674f, 0.83146961230254524f,
                         0.70710678118654752f, 0.55557023301960218f, 0.38268343236508977f,
                         0.19509032201612826f, 0.0f, -0.19509032201612826f, -0.38268343236508977f,
                         -0.55557023301960218f, -0.70710678118654752f, -0.83146961230254524f,
                         -0.92387953251128674f, -0.98078528040323044f};
    const float s[16] = {0.0f, 0.19509032201612826f, 0.38268343236508977f, 0.55557023301960218f,
                         0.70710678118654752f, 0.83146961230254524f, 0.92387953251128674f,
                         0.98078528040323044f, 1.0f, 0.98078528040323044f, 0.92387953251128674f,
                         0.83146961230254524f, 0.70710678118654752f, 0.55557023301960218f,
                         0.38268343236508977f, 0.19509032201612826f};
    return make_float2(c[t], inv ? s[t] : -s[t]);
}

// In-register DFT of R = 2,4,8,16,32 points (radix-2 DIF network), output
// in natural order.
template <int R, bool INV>
__device__ __forceinline__ void dft_reg(float2 (&v)[R])
{
#pragma unroll
    for (int span = R / 2; span >= 1; span >>= 1) {
#pragma unroll
        for (int i = 0; i < R; ++i) {
            if ((i & span) == 0) {
                const int j = i + span;
                const float2 a = v[i], b = v[j];
                v[i] = a + b;
                const float2 d = a - b;
                const int t = (i & (span - 1)) * (16 / span);  // W_{2 span}^t' in units of W_32
                // W_32^8 = -i (forward) or +i (inverse): a swap and a sign
                // (a product with the constants would keep the multiplications
                // by 0 and 1 under IEEE rules)
                v[j] = (t == 0) ? d
                     : (t == 8) ? (INV ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x))
                                : cmul(d, w32(t, INV));
            }
        }
    }
    float2 o[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
        int r = 0;
#pragma unroll
        for (int b = 1, rb = R / 2; b < R; b <<= 1, rb >>= 1)
            if (q & b) r |= rb;
        o[q] = v[r];
    }
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = o[q];
}

// Radix of pass p for M = 2^LOGM: radix 2^FFT_RB while possible, the
// remainder last (16384 points: 16 x 16 x 16 x 4).
constexpr int FFT_RB = 4;
template <int LOGM>
struct FftPlan {
    static constexpr int NP = (LOGM + FFT_RB - 1) / FFT_RB;
    __host__ __device__ static constexpr int last_bits() { return LOGM - FFT_RB * (NP - 1); }
    __host__ __device__ static constexpr int bits(int p) { return p < NP - 1 ? FFT_RB : last_bits(); }
    // threads per transform: one radix-32 group each
    __host__ __device__ static constexpr unsigned threads() { return (1u << LOGM) / 32 > 32 ? (1u << LOGM) / 32 : 32; }
};

// Shared-memory slot of element a: the low 4 index bits are XORed with bits
// 4-7, 8-11 and 12-15 (a bijection on [0, M), no padding), so 16 lanes that
// access a power-of-two stride up to 2^12 elements hit 16 different 8-byte
// bank pairs (the passes' strides and the digit-reversed final gather).
// pa is linear over XOR: pa(x ^ y) = pa(x) ^ pa(y), so the slot of an index
// made of disjoint bit fields is the XOR of the fields' slots.
__host__ __device__ constexpr unsigned pa(unsigned a) { return a ^ (((a >> 4) ^ (a >> 8) ^ (a >> 12)) & 15u); }
__host__ __device__ constexpr unsigned padded_len(unsigned m) { return m; }

// Smem position of frequency k after all DIF passes (mixed-radix digit
// reversal; each pass's output digit is the next frequency digit).
template <int LOGM>
__host__ __device__ constexpr unsigned fft_pos(unsigned k)
{
    using P = FftPlan<LOGM>;
    unsigned pos = 0, rem = LOGM;
    for (int p = 0; p < P::NP; ++p) {
        const int b = P::bits(p);
        const unsigned q = k & ((1u << b) - 1u);
        k >>= b;
        rem -= b;
        pos |= q << rem;
    }
    return pos;
}

__device__ __forceinline__ float2 twiddle(const float2* lo, const float2* hi, unsigned t, bool inv)
{
    const float2 w = cmul(hi[t >> 8], lo[t & 255]);
    return inv ? conjf2(w) : w;
}

// One DIF pass of radix R = 2^LOG_R on sub-transforms of length
// L = R * 2^LOG_SUB (in place) over M points. Element r of group
// (blk, j) is index blk*L + r*SUB + j: three disjoint bit fields, so its
// slot is pa(blk*L + j) ^ pa(r*SUB), the second term a constant.
template <int LOG_R, int LOG_SUB, bool INV>
__device__ __forceinline__ void fft_pass(float2* s, unsigned M, int log_nl, const float2* lo, const float2* hi)
{
    constexpr int R = 1 << LOG_R;
    constexpr unsigned SUB = 1u << LOG_SUB;
    const unsigned groups = M >> LOG_R;
    for (unsigned g = threadIdx.x; g < groups; g += blockDim.x) {
        const unsigned j = g & (SUB - 1u);
        const unsigned pb = pa(((g >> LOG_SUB) << (LOG_SUB + LOG_R)) | j);
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = s[pb ^ pa((unsigned)r << LOG_SUB)];
        dft_reg<R, INV>(v);
        if constexpr (SUB > 1) {
            if (j) {
                // W_L^{j q} = W_N^{j q N / L} (N = 2M) as powers of one looked-up
                // W_L^j: squarings for even q, one more factor for odd q (at
                // most 4 roundings per factor for R <= 16).
                float2 p[R];
                p[1] = twiddle(lo, hi, j << log_nl, INV);
#pragma unroll
                for (int q = 2; q < R; ++q) p[q] = (q & 1) ? cmul(p[q - 1], p[1]) : cmul(p[q / 2], p[q / 2]);
#pragma unroll
                for (int q = 1; q < R; ++q) v[q] = cmul(v[q], p[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < R; ++q) s[pb ^ pa((unsigned)q << LOG_SUB)] = v[q];
    }
}

// The DIF passes of FftPlan<LOG> over M points (one transform of 2^LOG, or
// several concatenated), pass P on, with log_nl = log2(N / L) of pass P.
template <int LOG, int P, bool INV>
__device__ __forceinline__ void fft_passes(float2* s, unsigned M, int log_nl, const float2* lo, const float2* hi)
{
    using PL = FftPlan<LOG>;
    if constexpr (P < PL::NP) {
        constexpr int B = PL::bits(P);
        constexpr int LOGL = LOG - FFT_RB * P;  // every earlier pass has FFT_RB bits
        __syncthreads();
        fft_pass<B, LOGL - B, INV>(s, M, log_nl, lo, hi);
        fft_passes<LOG, P + 1, INV>(s, M, log_nl + B, lo, hi);
    }
}

template <int LOGM, bool INV>
__device__ __forceinline__ void fft_smem(float2* s, const float2* lo, const float2* hi)
{
    fft_passes<LOGM, 0, INV>(s, 1u << LOGM, 1, lo, hi);
    __syncthreads();
}

// L2 prefetch of the bytes [p, p + n) (the 16-byte aligned part; a hint,
// no shared memory, completes on its own).
__device__ __forceinline__ void prefetch_l2(const void* p, size_t n)
{
    const uintptr_t a = ((uintptr_t)p + 15u) & ~(uintptr_t)15u;
    const uintptr_t e = ((uintptr_t)p + n) & ~(uintptr_t)15u;
    if (e > a) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((uint32_t)(e - a)) : "memory");
}

// Slots of the transform's element n = t + i*T (t < T = threads, both powers
// of two, so the fields are disjoint): pa(n) = pa(t) ^ pa(i*T); the final
// order fft_pos is a permutation of bit fields, so likewise
// pa(fft_pos(n)) = pa(fft_pos(t)) ^ pa(fft_pos(i*T)).
//
// Both single-CTA transforms are persistent: CTA b takes rows b, b + G,
// b + 2G, ... (G = gridDim.x, at most one wave). A 2^14-point transform fills
// the shared memory of an SM, so its load, transform and store phases cannot
// overlap with another CTA's; instead each CTA loads its next row into
// registers while it stores the current one, and asks L2 for the row after
// that, so that the loads of the next row find it there.
template <int LOGM>
__global__ void __launch_bounds__(FftPlan<LOGM>::threads()) fft_r2c_kernel(
    const float* x, size_t x_pitch, size_t nseg, size_t seg_stride, float2* X, size_t bin_pitch,
    TwiddleTable tw, size_t rows)
{
    constexpr unsigned M = 1u << LOGM;
    constexpr unsigned T = FftPlan<LOGM>::threads();
    constexpr unsigned PER = M >= T ? M / T : 1;  // sample pairs per thread
    extern __shared__ __align__(16) float2 s_fft[];
    float2* s = s_fft;
    float2* lo = s + padded_len(M);
    float2* hi = lo + 256;
    const unsigned nhi = (2 * M) / 256;
    for (unsigned i = threadIdx.x; i < 256; i += blockDim.x) lo[i] = tw.lo[i];
    for (unsigned i = threadIdx.x; i < nhi; i += blockDim.x) hi[i] = tw.hi[i];

    const unsigned t = threadIdx.x;
    auto row_src = [&](size_t row) {
        const size_t c = row / nseg;
        return x + c * x_pitch + (row - c * nseg) * seg_stride;
    };
    // pairs n = t + i*T of the row (segments that start on an 8-byte boundary
    // load them as float2): pairs i < PF are loaded during the previous row's
    // output phase, the rest when the row starts (register budget)
    constexpr unsigned PF = PER > 16 ? PER / 2 : PER;
    float2 v[PER];
    auto fetch = [&](size_t row, bool ahead) {
        const float* src = row_src(row);
        if ((reinterpret_cast<uintptr_t>(src) & 7u) == 0) {
            const float2* src2 = reinterpret_cast<const float2*>(src);
#pragma unroll
            for (unsigned i = 0; i < PER; ++i)
                if ((i < PF) == ahead && (M >= T || t < M)) v[i] = src2[t + i * T];
        } else {
#pragma unroll
            for (unsigned i = 0; i < PER; ++i) {
                const unsigned n = t + i * T;
                if ((i < PF) == ahead && (M >= T || t < M)) v[i] = make_float2(src[2 * n], src[2 * n + 1]);
            }
        }
    };
    const size_t G = gridDim.x;
    size_t row = blockIdx.x;
    if (row < rows) fetch(row, true);
    if (t == 0 && row + G < rows) prefetch_l2(row_src(row + G), (size_t)2 * M * sizeof(float));
    for (; row < rows; row += G) {
        if (t == 0 && row + 2 * G < rows) prefetch_l2(row_src(row + 2 * G), (size_t)2 * M * sizeof(float));
        if constexpr (PF < PER) fetch(row, false);
        __syncthreads();  // the previous row's output phase has read s
        if constexpr (M >= T) {
            const unsigned pt = pa(t);
#pragma unroll
            for (unsigned i = 0; i < PER; ++i) s[pt ^ pa(i * T)] = v[i];
        } else {
            if (t < M) s[pa(t)] = v[0];
        }
        fft_smem<LOGM, false>(s, lo, hi);
        if (row + G < rows) fetch(row + G, true);

        // Bins k and M - k from the pair z_k, z_{M-k} (k = 0..M/2): with
        // e = (z_k + conj z_{M-k}) / 2, o = (z_k - conj z_{M-k}) / (2i), w = W_2M^k,
        // X[k] = e + w o and X[M-k] = conj(e - w o).
        float2* dst = X + row * bin_pitch;
        auto pair = [&](unsigned k, float2 zk, float2 zm) {
            const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
            const float2 d = make_float2(zk.x - zm.x, zk.y + zm.y);  // zk - conj(zm)
            const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);   // d / (2i)
            const float2 wo = cmul(twiddle(lo, hi, k, false), o);
            dst[k] = e + wo;
            if (2 * k != M) dst[M - k] = make_float2(e.x - wo.x, wo.y - e.y);
        };
        if constexpr (M >= 2 * T) {
            // k = t + i*T < M/2; M - k = (M-1) ^ (k-1) for k >= 1
            const unsigned pk = pa(fft_pos<LOGM>(t));
            const unsigned pm = t ? pa(M - 1u) ^ pa(fft_pos<LOGM>(t - 1)) : 0u;
#pragma unroll 4
            for (unsigned i = 0; i < M / (2 * T); ++i) {
                const unsigned k = t + i * T;
                const float2 zk = s[pk ^ pa(fft_pos<LOGM>(i * T))];
                float2 zm;
                if (t) zm = s[pm ^ pa(fft_pos<LOGM>(i * T))];
                else zm = s[pa(fft_pos<LOGM>((M - k) & (M - 1u)))];
                pair(k, zk, zm);
            }
            if (t == 0) {
                const float2 z = s[pa(fft_pos<LOGM>(M / 2))];
                pair(M / 2, z, z);
            }
        } else {
            for (unsigned k = t; k <= M / 2; k += T) {
                const float2 zk = s[pa(fft_pos<LOGM>(k & (M - 1u)))];
                const float2 zm = s[pa(fft_pos<LOGM>((M - k) & (M - 1u)))];
                pair(k, zk, zm);
            }
        }
    }
}

template <int LOGM>
__global__ void __launch_bounds__(FftPlan<LOGM>::threads()) fft_c2r_kernel(
    const float2* Y, size_t bin_pitch, size_t nseg, float* out, size_t out_stride, size_t keep,
    size_t out_len, TwiddleTable tw, size_t rows)
{
    constexpr unsigned M = 1u << LOGM;
    constexpr unsigned T = FftPlan<LOGM>::threads();
    constexpr bool WIDE = M >= 2 * T;
    constexpr unsigned PER = WIDE ? M / (2 * T) : 1;  // bin pairs (k, M - k) per thread
    extern __shared__ __align__(16) float2 s_fft[];
    float2* s = s_fft;
    float2* lo = s + padded_len(M);
    float2* hi = lo + 256;
    const unsigned nhi = (2 * M) / 256;
    for (unsigned i = threadIdx.x; i < 256; i += blockDim.x) lo[i] = tw.lo[i];
    for (unsigned i = threadIdx.x; i < nhi; i += blockDim.x) hi[i] = tw.hi[i];

    const unsigned t = threadIdx.x;
    // bins a = Y[k], b = Y[M-k] for k = t + i*T (k <= M/2), and Y[M/2] on
    // thread 0 of the wide form
    // (pairs i < PF loaded during the previous row's output phase, the rest
    // when the row starts)
    constexpr unsigned PF = PER > 8 ? PER / 2 : PER;
    float2 xa[PER], xb[PER], ym = make_float2(0.f, 0.f);
    auto fetch = [&](size_t row, bool ahead) {
        const float2* src = Y + row * bin_pitch;
#pragma unroll
        for (unsigned i = 0; i < PER; ++i) {
            const unsigned k = t + i * T;
            if ((i < PF) == ahead && (WIDE || k <= M / 2)) {
                xa[i] = src[k];
                xb[i] = src[M - k];
            }
        }
        if (WIDE && ahead && t == 0) ym = src[M / 2];
    };
    const size_t G = gridDim.x;
    size_t row = blockIdx.x;
    if (row < rows) fetch(row, true);
    if (t == 0 && row + G < rows) prefetch_l2(Y + (row + G) * bin_pitch, (size_t)(M + 1) * sizeof(float2));
    for (; row < rows; row += G) {
        if (t == 0 && row + 2 * G < rows)
            prefetch_l2(Y + (row + 2 * G) * bin_pitch, (size_t)(M + 1) * sizeof(float2));
        if constexpr (PF < PER) fetch(row, false);
        __syncthreads();  // the previous row's output phase has read s (and lo/hi are in place)
        // z_k = E_k + i O_k and z_{M-k} from the bins a = Y[k], b = Y[M-k]
        // (k = 0..M/2): e = (a + conj b) / 2, d = (a - conj b) / 2, o = d conj(w),
        // w = W_2M^k; z_k = e + i o, z_{M-k} = conj(e) + i conj(o). The DC and
        // Nyquist imaginary parts are ignored (C2R).
        auto pair = [&](unsigned k, float2 a, float2 b, unsigned slot_k, unsigned slot_m) {
            if (k == 0) {
                a.y = 0.f;
                b.y = 0.f;
            }
            const float2 e = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y));
            const float2 d = make_float2(0.5f * (a.x - b.x), 0.5f * (a.y + b.y));
            const float2 o = cmul(d, conjf2(twiddle(lo, hi, k, false)));
            s[slot_k] = make_float2(e.x - o.y, e.y + o.x);
            if (k != 0 && 2 * k != M) s[slot_m] = make_float2(e.x + o.y, o.x - e.y);
        };
        if constexpr (WIDE) {
            const unsigned pt = pa(t);
            // slot of M - k = (M-1) ^ (k-1), k >= 1
            const unsigned pm = t ? pa(M - 1u) ^ pa(t - 1) : 0u;
#pragma unroll
            for (unsigned i = 0; i < PER; ++i) {
                const unsigned k = t + i * T;
                const unsigned sk = pt ^ pa(i * T);
                const unsigned sm = t ? pm ^ pa(i * T) : pa((M - k) & (M - 1u));
                pair(k, xa[i], xb[i], sk, sm);
            }
            if (t == 0) pair(M / 2, ym, ym, pa(M / 2), pa(M / 2));
        } else {
            if (t <= M / 2) pair(t, xa[0], xb[0], pa(t & (M - 1u)), pa((M - t) & (M - 1u)));
        }
        fft_smem<LOGM, true>(s, lo, hi);
        if (row + G < rows) fetch(row + G, true);

        const size_t dm = row / nseg, seg = row - dm * nseg;
        const float scale = 1.0f / (float)M;
        const size_t o0 = seg * keep;
        float* dst = out + dm * out_stride + o0;
        // samples of this segment that are kept and inside the row (<= 2M)
        const size_t room = o0 >= out_len ? 0 : out_len - o0;
        const unsigned lim = (unsigned)(keep < room ? keep : room);
        auto put = [&](unsigned n, float2 z) {
            const unsigned i0 = 2 * n;
            if (i0 < lim) dst[i0] = z.x * scale;
            if (i0 + 1 < lim) dst[i0 + 1] = z.y * scale;
        };
        if constexpr (M >= T) {
            const unsigned pn = pa(fft_pos<LOGM>(t));
#pragma unroll 4
            for (unsigned i = 0; i < M / T; ++i) put(t + i * T, s[pn ^ pa(fft_pos<LOGM>(i * T))]);
        } else {
            if (t < M) put(t, s[pa(fft_pos<LOGM>(t))]);
        }
    }
}

// ---------------------------------------------------------------------------
// Four-step FFT for M = M1 * M2 complex points (M > 16384): the columns
// n2 of z[n1 M2 + n2] are transformed (length M1) in tiles of FT_TILE columns
// per CTA, multiplied by W_M^{n2 k1} and stored as Z1[n2][k1]; then the rows
// k1 (length M2) in tiles of FT_TILE, giving X[k1 + M1 k2]. Each tile is a
// batch of independent transforms in shared memory; every global access is a
// run of FT_TILE consecutive complex values (128 bytes). Real input/output
// use the same half-length packing as the single-CTA kernels, with the
// real<->complex step as separate in-place passes over (k, M - k) pairs.
// ---------------------------------------------------------------------------
constexpr int FT_TILE = 16;
constexpr int FT_THREADS = 512;

// DIF passes over nb concatenated transforms of 2^LOG points each.
template <int LOG, bool INV>
__device__ __forceinline__ void fft_smem_multi(float2* s, unsigned nb, int log_nl0, const float2* lo,
                                               const float2* hi)
{
    fft_passes<LOG, 0, INV>(s, nb << LOG, log_nl0, lo, hi);
    __syncthreads();
}

__device__ __forceinline__ void load_twiddles(float2* lo, float2* hi, const TwiddleTable& tw)
{
    const unsigned nhi = tw.n / 256;
    for (unsigned i = threadIdx.x; i < 256; i += blockDim.x) lo[i] = tw.lo[i];
    for (unsigned i = threadIdx.x; i < nhi; i += blockDim.x) hi[i] = tw.hi[i];
}

// Step A. REAL_IN: row r = (c, seg) of real samples x (pairs packed as
// complex); else complex rows `zin` (pitch zin_pitch). Output Z1 rows of M.
template <int L1, int L2, bool REAL_IN, bool INV>
__global__ void __launch_bounds__(FT_THREADS) fft4_cols_kernel(
    const float* x, size_t x_pitch, size_t nseg, size_t seg_stride, const float2* zin, size_t zin_pitch,
    float2* Z1, TwiddleTable tw)
{
    constexpr unsigned M1 = 1u << L1, M2 = 1u << L2, M = M1 * M2;
    extern __shared__ __align__(16) float2 s_ft[];
    float2* s = s_ft;
    float2* lo = s + FT_TILE * M1;
    float2* hi = lo + 256;
    load_twiddles(lo, hi, tw);
    const size_t row = blockIdx.y;
    const unsigned c0 = blockIdx.x * FT_TILE;
    const float* xr = nullptr;
    const float2* zr = nullptr;
    if (REAL_IN) {
        const size_t c = row / nseg, seg = row - c * nseg;
        xr = x + c * x_pitch + seg * seg_stride;
    } else {
        zr = zin + row * zin_pitch;
    }
    for (unsigned idx = threadIdx.x; idx < FT_TILE * M1; idx += FT_THREADS) {
        const unsigned col = idx % FT_TILE, n1 = idx / FT_TILE;
        const size_t n = (size_t)n1 * M2 + c0 + col;
        s[pa(col * M1 + n1)] = REAL_IN ? make_float2(xr[2 * n], xr[2 * n + 1]) : zr[n];
    }
    fft_smem_multi<L1, INV>(s, FT_TILE, L1 + L2 + 1 - L1, lo, hi);
    float2* zo = Z1 + row * (size_t)M;
    const unsigned nmask = 2 * M - 1;
    for (unsigned idx = threadIdx.x; idx < FT_TILE * M1; idx += FT_THREADS) {
        const unsigned col = idx / M1, k1 = idx - col * M1;
        const unsigned n2 = c0 + col;
        const float2 v = s[pa(col * M1 + fft_pos<L1>(k1))];
        // W_M^{n2 k1} = W_N^{2 n2 k1}, N = 2M
        const float2 w = twiddle(lo, hi, (2u * n2 * k1) & nmask, INV);
        zo[(size_t)n2 * M1 + k1] = cmul(v, w);
    }
}

// Step B. REAL_OUT: time samples x[2n], x[2n+1] = Re, Im of z[n] / M into
// out rows (segment `seg` at column seg * keep, the first `keep` samples,
// at most out_len), else complex rows X (pitch x_pitch).
template <int L1, int L2, bool REAL_OUT, bool INV>
__global__ void __launch_bounds__(FT_THREADS) fft4_rows_kernel(
    const float2* Z1, float2* X, size_t x_pitch, float* out, size_t out_stride, size_t nseg, size_t keep,
    size_t out_len, TwiddleTable tw)
{
    constexpr unsigned M1 = 1u << L1, M2 = 1u << L2, M = M1 * M2;
    extern __shared__ __align__(16) float2 s_ft[];
    float2* s = s_ft;
    float2* lo = s + FT_TILE * M2;
    float2* hi = lo + 256;
    load_twiddles(lo, hi, tw);
    const size_t row = blockIdx.y;
    const unsigned t0 = blockIdx.x * FT_TILE;
    const float2* zr = Z1 + row * (size_t)M;
    for (unsigned idx = threadIdx.x; idx < FT_TILE * M2; idx += FT_THREADS) {
        const unsigned col = idx % FT_TILE, n2 = idx / FT_TILE;
        s[pa(col * M2 + n2)] = zr[(size_t)n2 * M1 + t0 + col];
    }
    fft_smem_multi<L2, INV>(s, FT_TILE, L1 + L2 + 1 - L2, lo, hi);
    if (REAL_OUT) {
        const float scale = 1.0f / (float)M;
        const size_t dm = row / nseg, seg = row - dm * nseg;
        float* dst = out + dm * out_stride;
        const size_t o0 = seg * keep;
        for (unsigned idx = threadIdx.x; idx < FT_TILE * M2; idx += FT_THREADS) {
            const unsigned col = idx % FT_TILE, k2 = idx / FT_TILE;
            const float2 z = s[pa(col * M2 + fft_pos<L2>(k2))];
            const size_t n = (size_t)t0 + col + (size_t)M1 * k2;
            const size_t i0 = 2 * n, i1 = i0 + 1;
            if (i0 < keep && o0 + i0 < out_len) dst[o0 + i0] = z.x * scale;
            if (i1 < keep && o0 + i1 < out_len) dst[o0 + i1] = z.y * scale;
        }
    } else {
        float2* xo = X + row * x_pitch;
        for (unsigned idx = threadIdx.x; idx < FT_TILE * M2; idx += FT_THREADS) {
            const unsigned col = idx % FT_TILE, k2 = idx / FT_TILE;
            xo[(size_t)t0 + col + (size_t)M1 * k2] = s[pa(col * M2 + fft_pos<L2>(k2))];
        }
    }
}

// Real-FFT post step in place: rows of M complex z -> M + 1 bins (same
// formula as fft_r2c_kernel), one thread per pair (k, M - k).
__global__ void __launch_bounds__(256) r2c_post_kernel(float2* X, size_t x_pitch, unsigned M, TwiddleTable tw)
{
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > M / 2) return;
    float2* r = X + (size_t)blockIdx.y * x_pitch;
    const float2 a = r[k & (M - 1)], b = r[(M - k) & (M - 1)];
    auto bin = [&](float2 zk, float2 zm, unsigned kk) {
        const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 d = make_float2(zk.x - zm.x, zk.y + zm.y);
        const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
        const float2 w = (kk == M) ? make_float2(-1.f, 0.f) : cmul(tw.hi[kk >> 8], tw.lo[kk & 255]);
        return e + cmul(w, o);
    };
    const float2 xk = bin(a, b, k);
    const float2 xm = bin(b, a, M - k);
    r[k] = xk;
    if (M - k != k) r[M - k] = xm;
}

// Inverse real-FFT pre step in place: M + 1 bins -> M complex z (same
// formula as fft_c2r_kernel), one thread per pair (k, M - k).
__global__ void __launch_bounds__(256) c2r_pre_kernel(float2* Y, size_t y_pitch, unsigned M, TwiddleTable tw)
{
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > M / 2) return;
    float2* r = Y + (size_t)blockIdx.y * y_pitch;
    float2 a = r[k], b = r[M - k];
    if (k == 0) {  // the DC and Nyquist imaginary parts are ignored (C2R)
        a.y = 0.f;
        b.y = 0.f;
    }
    auto pre = [&](float2 xk, float2 xm, unsigned kk) {
        const float2 e = make_float2(0.5f * (xk.x + xm.x), 0.5f * (xk.y - xm.y));
        const float2 d = make_float2(0.5f * (xk.x - xm.x), 0.5f * (xk.y + xm.y));
        const float2 w = cmul(tw.hi[kk >> 8], tw.lo[kk & 255]);
        const float2 o = cmul(d, conjf2(w));
        return make_float2(e.x - o.y, e.y + o.x);
    };
    const float2 zk = pre(a, b, k);
    if (k != 0 && M - k != k) r[M - k] = pre(b, a, M - k);
    r[k] = zk;
}

template <int L1, int L2>
void launch_r2c_4step(const float* x, size_t x_pitch, size_t rows, size_t nseg, size_t seg_stride,
                      float2* X, size_t bin_pitch, float2* Z1, const TwiddleTable& tw, cudaStream_t s)
{
    constexpr unsigned M1 = 1u << L1, M2 = 1u << L2, M = M1 * M2;
    const size_t tws = (256 + (size_t)tw.n / 256) * sizeof(float2);
    const size_t sa = FT_TILE * M1 * sizeof(float2) + tws, sb = FT_TILE * M2 * sizeof(float2) + tws;
    auto ka = fft4_cols_kernel<L1, L2, true, false>;
    auto kb = fft4_rows_kernel<L1, L2, false, false>;
    rt::raise_smem_limit(ka, sa);
    rt::raise_smem_limit(kb, sb);
    ka<<<dim3(M2 / FT_TILE, (unsigned)rows), FT_THREADS, sa, s>>>(x, x_pitch, nseg, seg_stride, nullptr, 0,
                                                                Z1, tw);
    RT_CHECK(cudaGetLastError());
    kb<<<dim3(M1 / FT_TILE, (unsigned)rows), FT_THREADS, sb, s>>>(Z1, X, bin_pitch, nullptr, 0, 1, 0, 0, tw);
    RT_CHECK(cudaGetLastError());
    r2c_post_kernel<<<dim3((M / 2 + 256) / 256, (unsigned)rows), 256, 0, s>>>(X, bin_pitch, M, tw);
    RT_CHECK(cudaGetLastError());
}

template <int L1, int L2>
void launch_c2r_4step(float2* Y, size_t bin_pitch, size_t rows, size_t nseg, float* out, size_t out_stride,
                      size_t keep, size_t out_len, float2* Z1, const TwiddleTable& tw, cudaStream_t s)
{
    constexpr unsigned M1 = 1u << L1, M2 = 1u << L2, M = M1 * M2;
    const size_t tws = (256 + (size_t)tw.n / 256) * sizeof(float2);
    const size_t sa = FT_TILE * M1 * sizeof(float2) + tws, sb = FT_TILE * M2 * sizeof(float2) + tws;
    c2r_pre_kernel<<<dim3((M / 2 + 256) / 256, (unsigned)rows), 256, 0, s>>>(Y, bin_pitch, M, tw);
    RT_CHECK(cudaGetLastError());
    auto ka = fft4_cols_kernel<L1, L2, false, true>;
    auto kb = fft4_rows_kernel<L1, L2, true, true>;
    rt::raise_smem_limit(ka, sa);
    rt::raise_smem_limit(kb, sb);
    ka<<<dim3(M2 / FT_TILE, (unsigned)rows), FT_THREADS, sa, s>>>(nullptr, 0, 1, 0, Y, bin_pitch, Z1, tw);
    RT_CHECK(cudaGetLastError());
    kb<<<dim3(M1 / FT_TILE, (unsigned)rows), FT_THREADS, sb, s>>>(Z1, nullptr, 0, out, out_stride, nseg, keep,
                                                                out_len, tw);
    RT_CHECK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Transforms of N = 16384 Q real points for any Q >= 1 (the whole-series
// length rule round_up(nsamp + max_delay, 16384), FDDGPUPlan.cpp:85-93, is
// rarely a power of two): M = N / 2 = P Q complex points, P = 8192. With
// n = n1 + P n2 and k = Q k1 + k2,
//   Z[Q k1 + k2] = sum_n1 W_P^{n1 k1} W_M^{n1 k2} sum_n2 z[n1 + P n2] W_Q^{n2 k2}:
// (1) Q-point DFTs over n2 for tiles of T consecutive n1 (mixed-radix
//     Stockham passes in shared memory; radices 4, 2, 3, 5, 7 in registers,
//     larger prime radices as direct sums), times W_M^{n1 k2}, stored as rows
//     k2 of P points in scratch;
// (2) P-point transforms of those rows (the shared-memory radix-16 kernel).
// The spectrum stays in this transposed order: bin k < M of a row at position
// (k mod Q) P + k / Q, bin M at position M (BinMap); the layout kernels read
// and write it in that order, the MAC sees true bins. The inverse runs the
// steps backwards. The Stockham formulation (autosort, decimation in time)
// follows Govindaraju et al., "High performance discrete Fourier transforms
// on graphics processors", SC 2008.
// ---------------------------------------------------------------------------
constexpr int FQ_LOGP = 13;
constexpr unsigned FQ_P = 1u << FQ_LOGP;
constexpr int FQ_THREADS = 256;

// One radix-r pass over T columns of Q points ([T][Q] in shared memory,
// from `in` to `out`); Ns = product of the earlier passes' radices;
// wq[x] = W_Q^x (conjugated for the inverse).
template <bool INV>
__device__ __forceinline__ void stockham_pass(const float2* __restrict__ in, float2* __restrict__ out, int Q,
                                              int T, int r, int Ns, const float2* __restrict__ wq)
{
    const int R = Q / r;
    const int ws = Q / (Ns * r);  // W_{Ns r}^x = W_Q^{x ws}
    const int wr = R;             // W_r^x = W_Q^{x Q / r}
    auto W = [&](int x) {
        const float2 w = wq[x];
        return INV ? conjf2(w) : w;
    };
    if (r <= 8) {
        for (int g = threadIdx.x; g < T * R; g += blockDim.x) {
            const int col = g / R, j = g - col * R;
            const int k = j % Ns;
            const float2* src = in + col * Q + j;
            float2 v[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                if (t < r) {
                    float2 a = src[t * R];
                    if (t > 0 && k > 0) a = cmul(a, W(t * k * ws));
                    v[t] = a;
                }
            }
            float2* dst = out + col * Q + (j / Ns) * Ns * r + k;
            if (r == 2) {
                dst[0] = v[0] + v[1];
                dst[Ns] = v[0] - v[1];
            } else if (r == 4) {
                const float2 s02 = v[0] + v[2], d02 = v[0] - v[2], s13 = v[1] + v[3], d13 = v[1] - v[3];
                // W_4 = -i (forward) or +i (inverse) times d13
                const float2 rot = INV ? make_float2(-d13.y, d13.x) : make_float2(d13.y, -d13.x);
                dst[0] = s02 + s13;
                dst[Ns] = d02 + rot;
                dst[2 * Ns] = s02 - s13;
                dst[3 * Ns] = d02 - rot;
            } else {
                // W_r^{t u} = W_Q^{t u wr}: index stepped by u wr (mod Q)
                for (int u = 0; u < r; ++u) {
                    float2 acc = v[0];
                    const int su = u * wr;
                    int x = 0;
#pragma unroll
                    for (int t = 1; t < 8; ++t) {
                        if (t < r) {
                            x += su;
                            if (x >= Q) x -= Q;
                            acc = acc + cmul(v[t], W(x));
                        }
                    }
                    dst[u * Ns] = acc;
                }
            }
        }
    } else {
        // one output (butterfly j, output u) per work item
        for (int g = threadIdx.x; g < T * Q; g += blockDim.x) {
            const int col = g / Q, rem = g - col * Q;
            const int j = rem % R, u = rem / R;
            const int k = j % Ns;
            const float2* src = in + col * Q + j;
            float2 acc = src[0];
            // input twiddle W_{Ns r}^{t k} times W_r^{t u}: W_Q^{t s}, s = k ws + u wr
            // (wr r = Q), the index stepped by s (mod Q)
            const int s = (k * ws + u * wr) % Q;
            int x = 0;
            for (int t = 1; t < r; ++t) {
                x += s;
                if (x >= Q) x -= Q;
                acc = acc + cmul(src[t * R], W(x));
            }
            out[col * Q + (j / Ns) * Ns * r + k + u * Ns] = acc;
        }
    }
}

// All passes; returns the buffer holding the natural-order result.
template <bool INV>
__device__ __forceinline__ float2* stockham_all(float2* b0, float2* b1, int Q, int T, const QRadices& rad,
                                                const float2* wq)
{
    float2* cur = b0;
    float2* nxt = b1;
    int Ns = 1;
    for (int p = 0; p < rad.n; ++p) {
        stockham_pass<INV>(cur, nxt, Q, T, rad.r[p], Ns, wq);
        __syncthreads();
        float2* t = cur;
        cur = nxt;
        nxt = t;
        Ns *= rad.r[p];
    }
    return cur;
}

// W_N^t from the two-level table in global memory (L1/L2 resident).
__device__ __forceinline__ float2 twiddle_g(const TwiddleTable& tw, size_t t, bool inv)
{
    const float2 w = cmul(__ldg(tw.hi + (t >> 8)), __ldg(tw.lo + (t & 255)));
    return inv ? conjf2(w) : w;
}

// Step (1), forward: row `row` = (c, seg) of real samples, columns
// n1 in [blockIdx.x T, +T): Z1[row][k2 P + n1] = W_M^{n1 k2} DFT_Q(z[n1 + P n2]).
__global__ void __launch_bounds__(FQ_THREADS) fftq_cols_fwd_kernel(
    const float* x, size_t x_pitch, size_t nseg, size_t seg_stride, float2* Z1, int Q, int T, QRadices rad,
    const float2* wq_g, TwiddleTable tw)
{
    extern __shared__ __align__(16) float2 s_q[];
    float2* b0 = s_q;
    float2* b1 = b0 + T * Q;
    float2* wq = b1 + T * Q;
    for (int i = threadIdx.x; i < Q; i += blockDim.x) wq[i] = wq_g[i];
    const size_t row = blockIdx.y;
    const unsigned n1_0 = blockIdx.x * (unsigned)T;
    const size_t c = row / nseg, seg = row - c * nseg;
    const float* xr = x + c * x_pitch + seg * seg_stride;
    for (int idx = threadIdx.x; idx < T * Q; idx += blockDim.x) {
        const int col = idx % T, n2 = idx / T;
        const size_t n = (size_t)n1_0 + col + (size_t)FQ_P * n2;
        b0[col * Q + n2] = make_float2(xr[2 * n], xr[2 * n + 1]);
    }
    __syncthreads();
    const float2* res = stockham_all<false>(b0, b1, Q, T, rad, wq);
    const size_t M = (size_t)FQ_P * Q;
    float2* zo = Z1 + row * M;
    for (int idx = threadIdx.x; idx < T * Q; idx += blockDim.x) {
        const int col = idx % T, k2 = idx / T;
        const size_t n1 = (size_t)n1_0 + col;
        // W_M^{n1 k2} = W_N^{2 n1 k2}, 2 n1 k2 < 2M = N
        zo[(size_t)k2 * FQ_P + n1] = cmul(res[col * Q + k2], twiddle_g(tw, 2 * n1 * (size_t)k2, false));
    }
}

// Step (1) backwards: u rows k2 (Z1[row][k2 P + n1]) times W_M^{-n1 k2},
// inverse Q-point DFTs over k2, then z[n1 + P n2] / M as real samples
// 2n, 2n + 1 of segment `seg` (the first `keep`, at most out_len).
__global__ void __launch_bounds__(FQ_THREADS) fftq_cols_inv_kernel(
    const float2* Z1, float* out, size_t out_stride, size_t nseg, size_t keep, size_t out_len, int Q, int T,
    QRadices rad, const float2* wq_g, TwiddleTable tw)
{
    extern __shared__ __align__(16) float2 s_q[];
    float2* b0 = s_q;
    float2* b1 = b0 + T * Q;
    float2* wq = b1 + T * Q;
    for (int i = threadIdx.x; i < Q; i += blockDim.x) wq[i] = wq_g[i];
    const size_t row = blockIdx.y;
    const unsigned n1_0 = blockIdx.x * (unsigned)T;
    const size_t M = (size_t)FQ_P * Q;
    const float2* zr = Z1 + row * M;
    for (int idx = threadIdx.x; idx < T * Q; idx += blockDim.x) {
        const int col = idx % T, k2 = idx / T;
        const size_t n1 = (size_t)n1_0 + col;
        b0[col * Q + k2] = cmul(zr[(size_t)k2 * FQ_P + n1], twiddle_g(tw, 2 * n1 * (size_t)k2, true));
    }
    __syncthreads();
    const float2* res = stockham_all<true>(b0, b1, Q, T, rad, wq);
    const float scale = 1.0f / (float)M;
    const size_t dm = row / nseg, seg = row - dm * nseg;
    float* dst = out + dm * out_stride;
    const size_t o0 = seg * keep;
    for (int idx = threadIdx.x; idx < T * Q; idx += blockDim.x) {
        const int col = idx % T, n2 = idx / T;
        const float2 z = res[col * Q + n2];
        const size_t n = (size_t)n1_0 + col + (size_t)FQ_P * n2;
        const size_t i0 = 2 * n, i1 = i0 + 1;
        if (i0 < keep && o0 + i0 < out_len) dst[o0 + i0] = z.x * scale;
        if (i1 < keep && o0 + i1 < out_len) dst[o0 + i1] = z.y * scale;
    }
}

// Step (2): P-point complex transforms of contiguous rows; row g = o Q + k2
// at src + o src_pitch + k2 P, natural-order result to the same place in dst.
// twp: twiddle table for 2P.
template <int LOGP, bool INV>
__global__ void __launch_bounds__(FftPlan<LOGP>::threads()) fft_c2c_rows_kernel(
    const float2* src, size_t src_pitch, float2* dst, size_t dst_pitch, unsigned Q, TwiddleTable twp, size_t rows)
{
    constexpr unsigned P = 1u << LOGP;
    constexpr unsigned T = FftPlan<LOGP>::threads();
    constexpr unsigned PER = P / T;
    extern __shared__ __align__(16) float2 s_fft[];
    float2* s = s_fft;
    float2* lo = s + P;
    float2* hi = lo + 256;
    for (unsigned i = threadIdx.x; i < 256; i += blockDim.x) lo[i] = twp.lo[i];
    for (unsigned i = threadIdx.x; i < 2 * P / 256; i += blockDim.x) hi[i] = twp.hi[i];
    const unsigned t = threadIdx.x;
    const unsigned pt = pa(t);
    for (size_t g = blockIdx.x; g < rows; g += gridDim.x) {
        const size_t o = g / Q, k2 = g - o * Q;
        const float2* in = src + o * src_pitch + k2 * P;
        float2 v[PER];
#pragma unroll
        for (unsigned i = 0; i < PER; ++i) v[i] = in[t + i * T];
        __syncthreads();  // the previous row's output phase has read s
#pragma unroll
        for (unsigned i = 0; i < PER; ++i) s[pt ^ pa(i * T)] = v[i];
        fft_smem<LOGP, INV>(s, lo, hi);
        float2* outp = dst + o * dst_pitch + k2 * P;
        const unsigned pk = pa(fft_pos<LOGP>(t));
#pragma unroll 4
        for (unsigned i = 0; i < PER; ++i) outp[t + i * T] = s[pk ^ pa(fft_pos<LOGP>(i * T))];
    }
}

__device__ __forceinline__ size_t qpos(size_t k, const BinMap& m)
{
    return (m.Q <= 1 || k >= m.M) ? k : (k % m.Q) * m.P + k / m.Q;
}

// Real-FFT post step in place over rows in the transposed order: bins k and
// M - k (k = 0..M/2) from z at the positions of k and M - k (formula of
// fft_r2c_kernel; bin M at position M). Threads run over consecutive
// positions p (bin k = qbin(p)); the thread whose bin is the smaller of the
// pair does the work, so both the bin and its partner are contiguous runs.
__global__ void __launch_bounds__(256) r2c_post_q_kernel(float2* X, size_t x_pitch, BinMap map, TwiddleTable tw)
{
    const size_t M = map.M;
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= M) return;
    const size_t k = qbin(p, map);
    if (k > M / 2) return;
    float2* r = X + (size_t)blockIdx.y * x_pitch;
    const size_t pk = qpos(k, map), pm = qpos(k ? M - k : 0, map);
    const float2 a = r[pk], b = r[pm];
    auto bin = [&](float2 zk, float2 zm, size_t kk) {
        const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 d = make_float2(zk.x - zm.x, zk.y + zm.y);
        const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
        const float2 w = (kk == M) ? make_float2(-1.f, 0.f) : twiddle_g(tw, kk, false);
        return e + cmul(w, o);
    };
    const float2 xk = bin(a, b, k);
    const float2 xm = bin(b, a, M - k);
    r[pk] = xk;
    if (M - k != k) r[qpos(M - k, map)] = xm;
}

// Inverse real-FFT pre step in place over transposed rows (formula of
// fft_c2r_kernel): bins k and M - k -> z at the positions of k and M - k.
// Threads run over consecutive positions, as in r2c_post_q_kernel.
__global__ void __launch_bounds__(256) c2r_pre_q_kernel(float2* Y, size_t y_pitch, BinMap map, TwiddleTable tw)
{
    const size_t M = map.M;
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= M) return;
    const size_t k = qbin(p, map);
    if (k > M / 2) return;
    float2* r = Y + (size_t)blockIdx.y * y_pitch;
    const size_t pk = qpos(k, map), pm = qpos(M - k, map);
    float2 a = r[pk], b = r[pm];
    if (k == 0) {  // the DC and Nyquist imaginary parts are ignored (C2R)
        a.y = 0.f;
        b.y = 0.f;
    }
    auto pre = [&](float2 xk, float2 xm, size_t kk) {
        const float2 e = make_float2(0.5f * (xk.x + xm.x), 0.5f * (xk.y - xm.y));
        const float2 d = make_float2(0.5f * (xk.x - xm.x), 0.5f * (xk.y + xm.y));
        const float2 o = cmul(d, conjf2(twiddle_g(tw, kk, false)));
        return make_float2(e.x - o.y, e.y + o.x);
    };
    const float2 zk = pre(a, b, k);
    if (k != 0 && M - k != k) r[pm] = pre(b, a, M - k);
    r[pk] = zk;
}

// Columns per CTA of step (1): the largest of 16, 8, 4 whose two [T][Q]
// buffers and the W_Q table fit in shared memory (0: none fits).
int fftq_tile(unsigned Q)
{
    for (int T : {16, 8, 4})
        if ((2 * (size_t)T * Q + Q) * sizeof(float2) <= kFqMaxSmem) return T;
    return 0;
}

// ---------------------------------------------------------------------------
// unpack / transposes
// ---------------------------------------------------------------------------
// Tiles of 64 samples x 64 channels per 256 threads: each thread issues its
// 16 loads before it uses any of them (64 KB in flight per SM at 8 blocks),
// then writes 16 time-contiguous values per channel run.
constexpr int UNPACK_TILE = 64;

template <int NB, bool ALIGNED>
__device__ __forceinline__ float unpack_sample(const uint8_t* in, size_t in_stride, size_t t, size_t c,
                                               float scale, float mid)
{
    if constexpr (NB == 8) {
        return ((float)__ldg(in + t * in_stride + c) - 127.5f) * scale;
    } else if constexpr (NB == 32) {
        const uint8_t* p = in + t * in_stride + 4 * c;
        uint32_t u;
        if constexpr (ALIGNED) u = __ldg(reinterpret_cast<const uint32_t*>(p));
        else u = (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
        return __uint_as_float(u) * scale;
    } else if constexpr (NB == 16) {
        const uint8_t* p = in + t * in_stride + 2 * c;
        const uint32_t u = ALIGNED ? (uint32_t)__ldg(reinterpret_cast<const uint16_t*>(p))
                                   : (uint32_t)p[0] | ((uint32_t)p[1] << 8);
        return ((float)u - mid) * scale;
    } else {
        // 1/2/4-bit samples packed LSB-first within each byte
        const size_t bit = c * (size_t)NB;
        const uint32_t u = (__ldg(in + t * in_stride + (bit >> 3)) >> (bit & 7)) & ((1u << NB) - 1u);
        return ((float)u - mid) * scale;
    }
}

// ALIGNED: every 16/32-bit sample starts on its own size (whole-sample loads)
template <int NB, bool ALIGNED>
__global__ void __launch_bounds__(256) fdd_unpack_kernel(const uint8_t* in, size_t in_stride, size_t nsamps,
                                                         size_t nchans, float scale, float mid, float* x,
                                                         size_t x_pitch, size_t x_len)
{
    constexpr int TL = UNPACK_TILE, PER = TL * TL / 256;
    __shared__ float tile[TL][TL + 1];
    const size_t t0 = (size_t)blockIdx.x * TL, c0 = (size_t)blockIdx.y * TL;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    float v[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        // element (sample t0 + ty + 8 (j % 8), channel c0 + tx + 32 (j / 8))
        const size_t t = t0 + ty + 8 * (j & 7), c = c0 + tx + 32 * (j >> 3);
        v[j] = (t < nsamps && c < nchans) ? unpack_sample<NB, ALIGNED>(in, in_stride, t, c, scale, mid) : 0.f;
    }
#pragma unroll
    for (int j = 0; j < PER; ++j) tile[ty + 8 * (j & 7)][tx + 32 * (j >> 3)] = v[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        // channel c0 + ty + 8 (j % 8), sample t0 + tx + 32 (j / 8)
        const int r = ty + 8 * (j & 7), tt = tx + 32 * (j >> 3);
        const size_t c = c0 + r, t = t0 + tt;
        if (c < nchans && t < x_len) x[c * x_pitch + t] = tile[tt][r];
    }
}

// X[c*nseg + seg][k] -> Xt[k][seg][j] for active channel j (km[j] applied).
// Tiles of 64 bins x 32 channels per 256 threads; every thread issues its 8
// loads before their first use.
constexpr int BMT_BINS = 64;
__global__ void __launch_bounds__(256) to_binmajor_kernel(const float2* X, size_t bin_pitch,
                                                          size_t nseg, size_t nbins,
                                                          const int32_t* chan, const float* km,
                                                          int nact, float2* Xt, BinMap map)
{
    // tiles run over row positions (contiguous reads); each position's bin
    // is qbin(position)
    constexpr int PER = BMT_BINS / 8;
    __shared__ float2 tile[32][BMT_BINS + 1];
    const size_t k0 = (size_t)blockIdx.x * BMT_BINS;
    const int j0 = blockIdx.y * 32;
    const size_t seg = blockIdx.z;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    float2 v[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        // channel j0 + ty + 8 (i % 4), bin k0 + tx + 32 (i / 4)
        const int j = j0 + ty + 8 * (i & 3);
        const size_t k = k0 + tx + 32 * (i >> 2);
        v[i] = (j < nact && k < nbins) ? X[((size_t)chan[j] * nseg + seg) * bin_pitch + k] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int r = ty + 8 * (i & 3), j = j0 + r;
        const float m = j < nact ? km[j] : 0.f;
        tile[r][tx + 32 * (i >> 2)] = make_float2(v[i].x * m, v[i].y * m);
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        // position k0 + ty + 8 i, channel j0 + tx
        const int kk = ty + 8 * i;
        const size_t p = k0 + kk;
        const int j = j0 + tx;
        if (p < nbins && j < nact) Xt[(qbin(p, map) * nseg + seg) * nact + j] = tile[tx][kk];
    }
}

// Yt[k][seg][dm] -> Y[dm*nseg + seg][k]
// Tiles of 64 bins x 32 DMs per 256 threads; every thread issues its 8
// loads before their first use.
constexpr int DMT_BINS = 64;
__global__ void __launch_bounds__(256) to_dmmajor_kernel(const float2* Yt, size_t nseg, size_t ndm,
                                                         size_t nbins, float2* Y, size_t bin_pitch,
                                                         BinMap map)
{
    // tiles run over row positions of Y (contiguous writes)
    constexpr int PER = DMT_BINS / 8;
    __shared__ float2 tile[DMT_BINS][33];
    const size_t k0 = (size_t)blockIdx.x * DMT_BINS, d0 = (size_t)blockIdx.y * 32;
    const size_t seg = blockIdx.z;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    float2 v[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const size_t p = k0 + ty + 8 * i, d = d0 + tx;
        v[i] = (p < nbins && d < ndm) ? Yt[(qbin(p, map) * nseg + seg) * ndm + d] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int i = 0; i < PER; ++i) tile[ty + 8 * i][tx] = v[i];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        // DM d0 + ty + 8 (i % 4), bin k0 + tx + 32 (i / 4)
        const int r = ty + 8 * (i & 3), kk = tx + 32 * (i >> 2);
        const size_t d = d0 + r, k = k0 + kk;
        if (d < ndm && k < nbins) Y[(d * nseg + seg) * bin_pitch + k] = tile[kk][r];
    }
}

// Yt[k][0][dm] -> out[dm][2k], out[dm][2k+1] for k < nspec
__global__ void __launch_bounds__(256) spectrum_out_kernel(const float2* Yt, size_t ndm, size_t nspec,
                                                           float* out, size_t out_stride)
{
    __shared__ float2 tile[32][33];
    const size_t k0 = (size_t)blockIdx.x * 32, d0 = (size_t)blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int r = ty; r < 32; r += 8) {
        const size_t k = k0 + r, d = d0 + tx;
        tile[r][tx] = (k < nspec && d < ndm) ? Yt[k * ndm + d] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const size_t d = d0 + r, k = k0 + tx;
        if (d < ndm && k < nspec) {
            const float2 v = tile[tx][r];
            out[d * out_stride + 2 * k] = v.x;
            out[d * out_stride + 2 * k + 1] = v.y;
        }
    }
}

// ---------------------------------------------------------------------------
// Plain FP32 phasor MAC: a complex GEMM per bin on CUDA cores.
// Block tile: 64 DMs x 40 segments (thread tile 4 x 5), channel chunk 32.
// ---------------------------------------------------------------------------
// Segment tiles: 40 (thread tile 4 x 5) for many segments, 8 (4 x 1) for
// few (whole-series and short segmented inputs, where a 40-wide tile would
// multiply padding); 16 x 8 threads either way.
constexpr int MAC_BM = 64, MAC_BK = 32, MAC_TM = 4;
constexpr int MAC_THREADS = 128;

__device__ __forceinline__ int fdd_delay(float dm, float delay, int round_delays)
{
    const float x = __fmul_rn(dm, delay);
    return round_delays ? (int)__float2uint_rn(x) : __float2int_rz(x);
}

// exp(+2 pi i m / N) for 0 <= m < N
__device__ __forceinline__ float2 phasor(const float2* lo, const float2* hi, unsigned m)
{
    return conjf2(cmul(hi[m >> 8], lo[m & 255]));
}

__device__ __forceinline__ unsigned phase_index(size_t k, int d, unsigned nfft, bool pow2)
{
    if (pow2) return (unsigned)((unsigned)k * (unsigned)d) & (nfft - 1u);
    long long p = (long long)k * (long long)d % (long long)nfft;
    if (p < 0) p += nfft;
    return (unsigned)p;
}

template <int MAC_BN, int MAC_TN>
__global__ void __launch_bounds__(MAC_THREADS) mac_plain_kernel(MacArgs a, int bins_per_block)
{
    static_assert((MAC_BM / MAC_TM) * (MAC_BN / MAC_TN) == MAC_THREADS, "thread tile");
    extern __shared__ __align__(16) float2 s_mac[];
    float2* As = s_mac;                        // [BK][BM]
    float2* Bs = As + MAC_BK * MAC_BM;         // [BK][BN]
    float2* lo = Bs + MAC_BK * MAC_BN;         // 256
    float2* hi = lo + 256;                     // nfft / 256
    const unsigned nhi = a.nfft / 256;
    for (unsigned i = threadIdx.x; i < 256; i += blockDim.x) lo[i] = a.tw.lo[i];
    for (unsigned i = threadIdx.x; i < nhi; i += blockDim.x) hi[i] = a.tw.hi[i];

    const int tid = threadIdx.x;
    const int tm = tid % (MAC_BM / MAC_TM), tn = tid / (MAC_BM / MAC_TM);
    const int dm0 = blockIdx.x * MAC_BM;
    const bool pow2 = (a.nfft & (a.nfft - 1u)) == 0;
    // phasor generation: this thread owns DM (dm0 + tid % 64), channels
    // tid/64 + 2i of each chunk
    const int gdm = tid % MAC_BM, gk0 = tid / MAC_BM;
    const float my_dm = a.dms[min(dm0 + gdm, a.ndm - 1)];

    const size_t kb0 = (size_t)blockIdx.y * bins_per_block;
    const size_t kb1 = min(a.nbins, kb0 + bins_per_block);
    for (size_t k = kb0; k < kb1; ++k) {
        for (int s0 = 0; s0 < a.nseg; s0 += MAC_BN) {
            float2 acc[MAC_TM][MAC_TN];
#pragma unroll
            for (int i = 0; i < MAC_TM; ++i)
#pragma unroll
                for (int j = 0; j < MAC_TN; ++j) acc[i][j] = make_float2(0.f, 0.f);

            for (int c0 = 0; c0 < a.nact; c0 += MAC_BK) {
                __syncthreads();
                for (int kc = gk0; kc < MAC_BK; kc += MAC_THREADS / MAC_BM) {
                    const int j = c0 + kc;
                    float2 w = make_float2(0.f, 0.f);
                    if (j < a.nact) {
                        const int d = fdd_delay(my_dm, a.delay_act[j], a.round_delays);
                        w = phasor(lo, hi, phase_index(k, d, a.nfft, pow2));
                    }
                    As[kc * MAC_BM + gdm] = w;
                }
                for (int i = tid; i < MAC_BK * MAC_BN; i += MAC_THREADS) {
                    const int kc = i / MAC_BN, sn = i - kc * MAC_BN;
                    const int j = c0 + kc, seg = s0 + sn;
                    Bs[kc * MAC_BN + sn] = (j < a.nact && seg < a.nseg)
                                               ? a.Xt[(k * a.nseg + seg) * a.nact + j]
                                               : make_float2(0.f, 0.f);
                }
                __syncthreads();
#pragma unroll 4
                for (int kc = 0; kc < MAC_BK; ++kc) {
                    float2 av[MAC_TM], bv[MAC_TN];
#pragma unroll
                    for (int i = 0; i < MAC_TM; ++i) av[i] = As[kc * MAC_BM + tm + i * (MAC_BM / MAC_TM)];
#pragma unroll
                    for (int j = 0; j < MAC_TN; ++j) bv[j] = Bs[kc * MAC_BN + tn + j * (MAC_BN / MAC_TN)];
#pragma unroll
                    for (int i = 0; i < MAC_TM; ++i)
#pragma unroll
                        for (int j = 0; j < MAC_TN; ++j) {
                            acc[i][j].x = fmaf(av[i].x, bv[j].x, acc[i][j].x);
                            acc[i][j].x = fmaf(-av[i].y, bv[j].y, acc[i][j].x);
                            acc[i][j].y = fmaf(av[i].x, bv[j].y, acc[i][j].y);
                            acc[i][j].y = fmaf(av[i].y, bv[j].x, acc[i][j].y);
                        }
                }
            }
#pragma unroll
            for (int i = 0; i < MAC_TM; ++i) {
                const int dm = dm0 + tm + i * (MAC_BM / MAC_TM);
                if (dm >= a.ndm) continue;
#pragma unroll
                for (int j = 0; j < MAC_TN; ++j) {
                    const int seg = s0 + tn + j * (MAC_BN / MAC_TN);
                    if (seg < a.nseg) a.Yt[(k * a.nseg + seg) * a.ndm + dm] = acc[i][j];
                }
            }
        }
    }
}

// FP32 MAC for one segment (the whole-series forms): each phasor feeds a
// single product, so generating it is the work. Per bin the CTA builds the
// phasors of every delay 0..dmax in shared memory (index k d mod N stepped
// exactly by (k S) mod N, the same phasor() product as the tiled kernel), loads
// the bin's spectra, and each thread accumulates SERIES_DPT DMs over all
// channels, in the tiled kernel's channel order and FMA sequence (so the sums
// are the same). Delays: dm * delay rounded by adding 2^23 (toward zero, or to
// nearest even), exact for 0 <= dm * delay < 2^22 (dmax bounds it).
constexpr int SERIES_THREADS = 256;
constexpr int SERIES_DPT = 8;  // DMs per thread and pass

__global__ void __launch_bounds__(SERIES_THREADS) mac_series_kernel(MacArgs a, int dmax, int bins_per_block)
{
    extern __shared__ __align__(16) float2 s_ser[];
    const unsigned tab_n = ((unsigned)dmax + 2u) & ~1u;  // even counts keep the float2 arrays aligned
    const unsigned nhi = a.nfft / 256;
    float2* table = s_ser;
    float2* lo = table + tab_n;
    float2* hi = lo + 256;
    float2* xs = hi + ((nhi + 1u) & ~1u);
    float* dl = reinterpret_cast<float*>(xs + ((a.nact + 1) & ~1));
    const int tid = threadIdx.x;
    for (unsigned i = tid; i < 256; i += SERIES_THREADS) lo[i] = a.tw.lo[i];
    for (unsigned i = tid; i < nhi; i += SERIES_THREADS) hi[i] = a.tw.hi[i];
    for (int i = tid; i < a.nact; i += SERIES_THREADS) dl[i] = a.delay_act[i];
    const bool rn = a.round_delays != 0;
    const uint32_t dcap = (uint32_t)dmax;

    const size_t kb0 = (size_t)blockIdx.x * bins_per_block;
    const size_t kb1 = min(a.nbins, kb0 + bins_per_block);
    for (size_t k = kb0; k < kb1; ++k) {
        __syncthreads();  // the previous bin's table and spectra are no longer read
        {
            constexpr uint32_t S = SERIES_THREADS;
            uint32_t idx = (uint32_t)(((uint64_t)k * (uint64_t)tid) % a.nfft);
            const uint32_t step = (uint32_t)(((uint64_t)k * S) % a.nfft);
            for (int d = tid; d <= dmax; d += S) {
                table[d] = phasor(lo, hi, idx);
                idx = (idx + step >= a.nfft) ? idx + step - a.nfft : idx + step;
            }
        }
        for (int i = tid; i < a.nact; i += SERIES_THREADS) xs[i] = a.Xt[k * (size_t)a.nact + i];
        __syncthreads();
        for (int m0 = 0; m0 < a.ndm; m0 += SERIES_THREADS * SERIES_DPT) {
            float dmv[SERIES_DPT];
            float2 acc[SERIES_DPT];
#pragma unroll
            for (int q = 0; q < SERIES_DPT; ++q) {
                dmv[q] = a.dms[min(m0 + tid + q * SERIES_THREADS, a.ndm - 1)];
                acc[q] = make_float2(0.f, 0.f);
            }
#pragma unroll 2
            for (int c = 0; c < a.nact; ++c) {
                const float delay = dl[c];
                const float2 bv = xs[c];
#pragma unroll
                for (int q = 0; q < SERIES_DPT; ++q) {
                    const float x = __fmul_rn(dmv[q], delay);
                    const float y = rn ? __fadd_rn(x, 8388608.0f) : __fadd_rz(x, 8388608.0f);
                    const float2 av = table[min(__float_as_uint(y) - 0x4B000000u, dcap)];
                    acc[q].x = fmaf(av.x, bv.x, acc[q].x);
                    acc[q].x = fmaf(-av.y, bv.y, acc[q].x);
                    acc[q].y = fmaf(av.x, bv.y, acc[q].y);
                    acc[q].y = fmaf(av.y, bv.x, acc[q].y);
                }
            }
#pragma unroll
            for (int q = 0; q < SERIES_DPT; ++q) {
                const int m = m0 + tid + q * SERIES_THREADS;
                if (m < a.ndm) a.Yt[k * (size_t)a.ndm + m] = acc[q];
            }
        }
    }
}

size_t series_smem_bytes(int dmax, unsigned nfft, int nact)
{
    return ((size_t)(((unsigned)dmax + 2u) & ~1u) + 256 + ((nfft / 256 + 1) & ~1u) + (size_t)((nact + 1) & ~1)) *
               sizeof(float2) +
           (size_t)nact * sizeof(float);
}

// CTAs of one wave of a persistent kernel: resident CTAs per SM x SMs,
// at most `rows` (at least one).
template <typename K>
unsigned persistent_grid(K kernel, unsigned threads, size_t smem, size_t rows)
{
    int dev = 0, sms = 0, per_sm = 0;
    RT_CHECK(cudaGetDevice(&dev));
    RT_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    RT_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, (int)threads, smem));
    const size_t wave = (size_t)std::max(per_sm, 1) * (size_t)std::max(sms, 1);
    return (unsigned)std::max<size_t>(1, std::min(wave, rows));
}

template <int LOGM>
void launch_r2c_n(const float* x, size_t x_pitch, size_t nchans, size_t nseg, size_t seg_stride,
                  float2* X, size_t bin_pitch, const TwiddleTable& tw, cudaStream_t s)
{
    constexpr unsigned M = 1u << LOGM;
    const size_t smem = (padded_len(M) + 256 + 2 * M / 256) * sizeof(float2);
    auto k = fft_r2c_kernel<LOGM>;
    rt::raise_smem_limit(k, smem);
    const unsigned threads = FftPlan<LOGM>::threads();
    const size_t rows = nchans * nseg;
    if (rows == 0) return;
    k<<<persistent_grid(k, threads, smem, rows), threads, smem, s>>>(x, x_pitch, nseg, seg_stride, X, bin_pitch,
                                                                     tw, rows);
    RT_CHECK(cudaGetLastError());
}

template <int LOGM>
void launch_c2r_n(const float2* Y, size_t bin_pitch, size_t ndm, size_t nseg, float* out,
                  size_t out_stride, size_t keep, size_t out_len, const TwiddleTable& tw,
                  cudaStream_t s)
{
    constexpr unsigned M = 1u << LOGM;
    const size_t smem = (padded_len(M) + 256 + 2 * M / 256) * sizeof(float2);
    auto k = fft_c2r_kernel<LOGM>;
    rt::raise_smem_limit(k, smem);
    const unsigned threads = FftPlan<LOGM>::threads();
    const size_t rows = ndm * nseg;
    if (rows == 0) return;
    k<<<persistent_grid(k, threads, smem, rows), threads, smem, s>>>(Y, bin_pitch, nseg, out, out_stride, keep,
                                                                     out_len, tw, rows);
    RT_CHECK(cudaGetLastError());
}

int log2_exact(int n)
{
    int l = 0;
    while ((1 << l) < n) ++l;
    return (1 << l) == n ? l : -1;
}

}  // namespace

void launch_fdd_unpack(const uint8_t* in, size_t in_stride, int in_nbits, size_t nsamps,
                       size_t nchans, float scale, float* x, size_t x_pitch, size_t x_len,
                       cudaStream_t s)
{
    // packed unsigned samples are centred at mid-scale, (2^nbits - 1) / 2
    // (127.5 for 8-bit, as the reference's unpack_kernel.cuh:60)
    const float mid = in_nbits == 32 ? 0.f : (float)((1u << in_nbits) - 1u) * 0.5f;
    if (x_len == 0 || nchans == 0) return;
    dim3 grid((unsigned)((x_len + UNPACK_TILE - 1) / UNPACK_TILE),
              (unsigned)((nchans + UNPACK_TILE - 1) / UNPACK_TILE));
    // whole-sample loads when every sample starts on its own size
    const size_t sb = in_nbits >= 16 ? (size_t)in_nbits / 8 : 1;
    const bool aligned = ((uintptr_t)in % sb == 0) && (in_stride % sb == 0);
    switch (in_nbits) {
#define UNPACK(NB, AL) fdd_unpack_kernel<NB, AL><<<grid, 256, 0, s>>>(in, in_stride, nsamps, nchans, scale, mid, x, x_pitch, x_len)
    case 1: UNPACK(1, true); break;
    case 2: UNPACK(2, true); break;
    case 4: UNPACK(4, true); break;
    case 8: UNPACK(8, true); break;
    case 16: if (aligned) UNPACK(16, true); else UNPACK(16, false); break;
    case 32: if (aligned) UNPACK(32, true); else UNPACK(32, false); break;
#undef UNPACK
    default: DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "unsupported FDD input width");
    }
    RT_CHECK(cudaGetLastError());
}

// The four-step and Q-point kernels carry the row (channel x segment or DM x
// segment) in grid.y: launches of whole channels or DMs, at most 65535 rows
// each, one after another (they share the scratch buffer).
static size_t rows_per_launch(size_t nseg)
{
    if (nseg == 0 || nseg > 65535) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "too many segments");
    return 65535 / nseg;
}

void launch_fft_r2c(const float* x, size_t x_pitch, size_t nchans, size_t nseg, size_t seg_stride,
                    int nfft, float2* X, size_t bin_pitch, const TwiddleTable& tw, float2* scratch,
                    cudaStream_t s)
{
    const int lg = log2_exact(nfft);
    if (lg >= 5 && lg <= 15) {
        switch (lg) {
#define R2C(L) case L + 1: launch_r2c_n<L>(x, x_pitch, nchans, nseg, seg_stride, X, bin_pitch, tw, s); break;
            R2C(4) R2C(5) R2C(6) R2C(7) R2C(8) R2C(9) R2C(10) R2C(11) R2C(12) R2C(13) R2C(14)
#undef R2C
        }
        return;
    }
    const size_t per = rows_per_launch(nseg);
    for (size_t c0 = 0; c0 < nchans; c0 += per) {
        const size_t rows = std::min(per, nchans - c0) * nseg;
        const float* xc = x + c0 * x_pitch;
        float2* Xc = X + c0 * nseg * bin_pitch;
        switch (lg) {
#define R4(L1, L2) case L1 + L2 + 1: launch_r2c_4step<L1, L2>(xc, x_pitch, rows, nseg, seg_stride, Xc, bin_pitch, scratch, tw, s); break;
            R4(8, 7) R4(8, 8) R4(9, 8) R4(9, 9) R4(10, 9)
#undef R4
        default: DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "unsupported FFT length");
        }
    }
}

void launch_fft_c2r(float2* Y, size_t bin_pitch, size_t ndm, size_t nseg, int nfft,
                    float* out, size_t out_stride, size_t keep, size_t out_len,
                    const TwiddleTable& tw, float2* scratch, cudaStream_t s)
{
    const int lg = log2_exact(nfft);
    if (lg >= 5 && lg <= 15) {
        switch (lg) {
#define C2R(L) case L + 1: launch_c2r_n<L>(Y, bin_pitch, ndm, nseg, out, out_stride, keep, out_len, tw, s); break;
            C2R(4) C2R(5) C2R(6) C2R(7) C2R(8) C2R(9) C2R(10) C2R(11) C2R(12) C2R(13) C2R(14)
#undef C2R
        }
        return;
    }
    const size_t per = rows_per_launch(nseg);
    for (size_t d0 = 0; d0 < ndm; d0 += per) {
        const size_t rows = std::min(per, ndm - d0) * nseg;
        float2* Yd = Y + d0 * nseg * bin_pitch;
        float* od = out + d0 * out_stride;
        switch (lg) {
#define C4(L1, L2) case L1 + L2 + 1: launch_c2r_4step<L1, L2>(Yd, bin_pitch, rows, nseg, od, out_stride, keep, out_len, scratch, tw, s); break;
            C4(8, 7) C4(8, 8) C4(9, 8) C4(9, 9) C4(10, 9)
#undef C4
        default: DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "unsupported FFT length");
        }
    }
}

size_t fft_scratch_elems(int nfft, size_t rows) { return nfft > 32768 ? rows * (size_t)(nfft / 2) : 0; }

void make_twiddle_tables(size_t n, std::vector<float2>& lo, std::vector<float2>& hi)
{
    lo.resize(256);
    hi.resize(n / 256);
    for (unsigned l = 0; l < 256; ++l) {
        const double a = -2.0 * 3.14159265358979323846 * (double)l / (double)n;
        lo[l] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    for (size_t h = 0; h < hi.size(); ++h) {
        const double a = -2.0 * 3.14159265358979323846 * (double)h * 256.0 / (double)n;
        hi[h] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
}

bool fftq_length(size_t nfft)
{
    return nfft >= 16384 && nfft % 16384 == 0 && fftq_tile((unsigned)(nfft / 16384)) > 0 &&
           nfft / 2 <= ((size_t)1 << 31);
}

BinMap fdd_binmap(size_t nfft)
{
    BinMap m;
    m.M = nfft / 2;
    const bool pow2 = (nfft & (nfft - 1)) == 0;
    m.Q = (!pow2 || nfft > (size_t)kMaxFft) ? (unsigned)(nfft / 16384) : 1u;
    m.P = FQ_P;
    return m;
}

QRadices fftq_radices(unsigned Q)
{
    QRadices r;
    unsigned q = Q;
    auto push = [&](unsigned f) {
        if (r.n >= 24) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "too many FFT radices");
        r.r[r.n++] = (int)f;
        q /= f;
    };
    for (unsigned f : {4u, 2u, 3u, 5u, 7u})
        while (q % f == 0) push(f);
    for (unsigned f = 11; q > 1; f += 2)
        while (q % f == 0) push(f);
    return r;
}

std::vector<float2> fftq_wq_table(unsigned Q)
{
    std::vector<float2> w(Q);
    for (unsigned x = 0; x < Q; ++x) {
        const double a = -2.0 * 3.14159265358979323846 * (double)x / (double)Q;
        w[x] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    return w;
}

void launch_fft_r2c_q(const float* x, size_t x_pitch, size_t nchans, size_t nseg, size_t seg_stride,
                      size_t nfft, float2* X, size_t bin_pitch, const TwiddleTable& tw,
                      const TwiddleTable& twp, const float2* wq, float2* scratch, cudaStream_t s)
{
    if (!fftq_length(nfft)) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "unsupported FFT length");
    const unsigned Q = (unsigned)(nfft / 16384);
    if (nchans * nseg == 0) return;
    const int T = fftq_tile(Q);
    const QRadices rad = fftq_radices(Q);
    const BinMap map = fdd_binmap(nfft);
    const size_t sq = (2 * (size_t)T * Q + Q) * sizeof(float2);
    rt::raise_smem_limit(fftq_cols_fwd_kernel, sq);
    auto kr = fft_c2c_rows_kernel<FQ_LOGP, false>;
    const size_t sr = (FQ_P + 256 + 2 * FQ_P / 256) * sizeof(float2);
    rt::raise_smem_limit(kr, sr);
    const size_t per = rows_per_launch(nseg);
    for (size_t c0 = 0; c0 < nchans; c0 += per) {
        const size_t rows = std::min(per, nchans - c0) * nseg;
        const float* xc = x + c0 * x_pitch;
        float2* Xc = X + c0 * nseg * bin_pitch;
        fftq_cols_fwd_kernel<<<dim3(FQ_P / T, (unsigned)rows), FQ_THREADS, sq, s>>>(xc, x_pitch, nseg, seg_stride,
                                                                                  scratch, (int)Q, T, rad, wq, tw);
        RT_CHECK(cudaGetLastError());
        const size_t nrows = rows * Q;
        kr<<<persistent_grid(kr, FftPlan<FQ_LOGP>::threads(), sr, nrows), FftPlan<FQ_LOGP>::threads(), sr, s>>>(
            scratch, map.M, Xc, bin_pitch, Q, twp, nrows);
        RT_CHECK(cudaGetLastError());
        r2c_post_q_kernel<<<dim3((unsigned)((map.M + 255) / 256), (unsigned)rows), 256, 0, s>>>(Xc, bin_pitch, map,
                                                                                                tw);
        RT_CHECK(cudaGetLastError());
    }
}

void launch_fft_c2r_q(float2* Y, size_t bin_pitch, size_t ndm, size_t nseg, size_t nfft, float* out,
                      size_t out_stride, size_t keep, size_t out_len, const TwiddleTable& tw,
                      const TwiddleTable& twp, const float2* wq, float2* scratch, cudaStream_t s)
{
    if (!fftq_length(nfft)) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "unsupported FFT length");
    const unsigned Q = (unsigned)(nfft / 16384);
    if (ndm * nseg == 0) return;
    const int T = fftq_tile(Q);
    const QRadices rad = fftq_radices(Q);
    const BinMap map = fdd_binmap(nfft);
    auto kr = fft_c2c_rows_kernel<FQ_LOGP, true>;
    const size_t sr = (FQ_P + 256 + 2 * FQ_P / 256) * sizeof(float2);
    rt::raise_smem_limit(kr, sr);
    const size_t sq = (2 * (size_t)T * Q + Q) * sizeof(float2);
    rt::raise_smem_limit(fftq_cols_inv_kernel, sq);
    const size_t per = rows_per_launch(nseg);
    for (size_t d0 = 0; d0 < ndm; d0 += per) {
        const size_t rows = std::min(per, ndm - d0) * nseg;
        float2* Yd = Y + d0 * nseg * bin_pitch;
        float* od = out + d0 * out_stride;
        c2r_pre_q_kernel<<<dim3((unsigned)((map.M + 255) / 256), (unsigned)rows), 256, 0, s>>>(Yd, bin_pitch, map,
                                                                                               tw);
        RT_CHECK(cudaGetLastError());
        const size_t nrows = rows * Q;
        kr<<<persistent_grid(kr, FftPlan<FQ_LOGP>::threads(), sr, nrows), FftPlan<FQ_LOGP>::threads(), sr, s>>>(
            Yd, bin_pitch, scratch, map.M, Q, twp, nrows);
        RT_CHECK(cudaGetLastError());
        fftq_cols_inv_kernel<<<dim3(FQ_P / T, (unsigned)rows), FQ_THREADS, sq, s>>>(
            scratch, od, out_stride, nseg, keep, out_len, (int)Q, T, rad, wq, tw);
        RT_CHECK(cudaGetLastError());
    }
}

void launch_fdd_to_binmajor(const float2* X, size_t bin_pitch, size_t nseg, size_t nbins,
                            const int32_t* chan, const float* km, int nact, float2* Xt,
                            const BinMap& map, cudaStream_t s)
{
    dim3 grid((unsigned)((nbins + BMT_BINS - 1) / BMT_BINS), (unsigned)((nact + 31) / 32), (unsigned)nseg);
    to_binmajor_kernel<<<grid, 256, 0, s>>>(X, bin_pitch, nseg, nbins, chan, km, nact, Xt, map);
    RT_CHECK(cudaGetLastError());
}

void launch_fdd_to_dmmajor(const float2* Yt, size_t nseg, size_t ndm, size_t nbins, float2* Y,
                           size_t bin_pitch, const BinMap& map, cudaStream_t s)
{
    dim3 grid((unsigned)((nbins + DMT_BINS - 1) / DMT_BINS), (unsigned)((ndm + 31) / 32), (unsigned)nseg);
    to_dmmajor_kernel<<<grid, 256, 0, s>>>(Yt, nseg, ndm, nbins, Y, bin_pitch, map);
    RT_CHECK(cudaGetLastError());
}

void launch_fdd_spectrum_out(const float2* Yt, size_t ndm, size_t nspec, float* out,
                             size_t out_stride, cudaStream_t s)
{
    dim3 grid((unsigned)((nspec + 31) / 32), (unsigned)((ndm + 31) / 32));
    spectrum_out_kernel<<<grid, 256, 0, s>>>(Yt, ndm, nspec, out, out_stride);
    RT_CHECK(cudaGetLastError());
}

bool fdd_mac_series_fits(int dmax, unsigned nfft, int nact)
{
    return dmax >= 0 && dmax < (1 << 22) && series_smem_bytes(dmax, nfft, nact) <= 200 * 1024;
}

void launch_fdd_mac_series(const MacArgs& a, int dmax, cudaStream_t s)
{
    if (a.nseg != 1 || !fdd_mac_series_fits(dmax, a.nfft, a.nact) || a.nfft % 256 != 0)
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "one-segment MAC: shape out of range");
    const size_t smem = series_smem_bytes(dmax, a.nfft, a.nact);
    rt::raise_smem_limit(mac_series_kernel, smem);
    const unsigned grid = persistent_grid(mac_series_kernel, SERIES_THREADS, smem, a.nbins);
    const int per = (int)((a.nbins + grid - 1) / grid);
    mac_series_kernel<<<(unsigned)((a.nbins + per - 1) / per), SERIES_THREADS, smem, s>>>(a, dmax, per);
    RT_CHECK(cudaGetLastError());
}

void launch_fdd_mac_plain(const MacArgs& a, cudaStream_t s)
{
    const bool narrow = a.nseg <= 8;
    const int bn = narrow ? 8 : 40;
    const size_t smem = (MAC_BK * MAC_BM + MAC_BK * (size_t)bn + 256 + a.nfft / 256) * sizeof(float2);
    if (smem > 200 * 1024) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "FFT length too large for the MAC table");
    auto kern = narrow ? mac_plain_kernel<8, 1> : mac_plain_kernel<40, 5>;
    rt::raise_smem_limit(kern, smem);
    const unsigned dm_tiles = (unsigned)((a.ndm + MAC_BM - 1) / MAC_BM);
    // enough blocks to fill the GPU several times over
    const size_t want_blocks = 148 * 8;
    size_t bin_blocks = std::max<size_t>(1, want_blocks / dm_tiles);
    bin_blocks = std::min(bin_blocks, a.nbins);
    const int per = (int)((a.nbins + bin_blocks - 1) / bin_blocks);
    bin_blocks = (a.nbins + per - 1) / per;
    dim3 grid(dm_tiles, (unsigned)bin_blocks);
    kern<<<grid, MAC_THREADS, smem, s>>>(a, per);
    RT_CHECK(cudaGetLastError());
}

}  // namespace kern
}  // namespace dedisp
