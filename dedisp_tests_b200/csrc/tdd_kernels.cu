// Time-domain dedispersion kernels for sm_100a.
//
//   K1  transpose_kernel       time-major packed -> channel-major packed
//   K2p dedisperse_plain       one thread per (DM, sample pair), global loads
//                              (the reference algorithm, kept as baseline)
//   K2  dedisperse_tiled       shared-memory staged channel windows, packed
//                              SIMD-within-a-register accumulation
//   K1d quad_direct_kernel     time-major packed -> quad-strided rows (samples
//                              of up to 8 bits widened to bytes)
//   K2q dedisperse_quad8       the byte accumulation on quad-strided rows
//
// Exactness: the sums are the reference's integer sums
// (src/tdd/dedisperse/dedisperse_kernel.cuh:145-181): every integer delay is
// __float2uint_rn(__fmul_rn(dm, delay[c])) and every partial sum is exact
// (narrow lanes are flushed into 32-bit sums before they can overflow). The
// FP32 epilogue repeats the reference operation order with IEEE rounding
// intrinsics (dedisperse_kernel.cuh:45-64).
#include "tdd_kernels.hpp"

#include <algorithm>
#include <utility>

#include "runtime.hpp"

namespace dedisp {
namespace kern {
namespace {

// ---------------------------------------------------------------------------
// Epilogue: src/tdd/dedisperse/dedisperse_kernel.cuh:45-87
// ---------------------------------------------------------------------------
__device__ __forceinline__ float sum_to_float(uint32_t s) { return __uint2float_rn(s); }
__device__ __forceinline__ float sum_to_float(unsigned long long s) { return __ull2float_rn(s); }

template <typename S>
__device__ __forceinline__ void store_out(void* out, size_t idx, int out_nbits, S sum,
                                          float den, float factor)
{
    const float fs = sum_to_float(sum);
    if (out_nbits == 32) {
        // out_range == 1.f: (fs * 1.f) == fs exactly
        static_cast<float*>(out)[idx] = __fmul_rn(__fdiv_rn(fs, den), factor);
    } else {
        const float out_range = (out_nbits == 8) ? 255.f : 65535.f;
        float v = __fmul_rn(__fdiv_rn(__fmul_rn(fs, out_range), den), factor);
        // min(max(v, 0.), out_range) in double equals the float clip here:
        // both bounds are exact floats and v is never NaN.
        v = fminf(fmaxf(v, 0.f), out_range);
        if (out_nbits == 8) static_cast<uint8_t*>(out)[idx] = (uint8_t)__float2uint_rz(v);
        else static_cast<uint16_t*>(out)[idx] = (uint16_t)__float2uint_rz(v);
    }
}

__device__ __forceinline__ uint32_t delay_rn(float dm, float delay)
{
    // src/tdd/dedisperse/dedisperse_kernel.cuh:163-165
    return __float2uint_rn(__fmul_rn(dm, delay));
}

template <int NBITS>
__device__ __forceinline__ constexpr uint32_t sample_mask()
{
    return NBITS == 32 ? 0xFFFFFFFFu : ((1u << NBITS) - 1u);
}

// ---------------------------------------------------------------------------
// K1: transpose
// ---------------------------------------------------------------------------
template <int NBITS>
struct TrGeom {
    static constexpr int SPW = 32 / NBITS;                      // samples per word
    static constexpr int TC = (NBITS <= 8) ? 512 / NBITS : 64;  // channels per tile
    static constexpr int SEGW = TC * NBITS / 32;                // input words per row
    static constexpr int TR = 128;                              // samples per tile
    static constexpr int OW = TR / SPW;                         // output words per row
};

template <int NBITS>
__global__ void __launch_bounds__(256) transpose_kernel(TransposeArgs a, int aligned)
{
    using G = TrGeom<NBITS>;
    __shared__ uint32_t tile[G::TR][G::SEGW + 1];
    const size_t r0 = (size_t)blockIdx.x * G::TR;
    const size_t c0 = (size_t)blockIdx.y * G::TC;
    const size_t row_words = a.nchans * NBITS / 32;
    const size_t w0 = c0 * NBITS / 32;

    for (int i = threadIdx.x; i < G::TR * G::SEGW; i += 256) {
        const int r = i / G::SEGW, k = i % G::SEGW;
        const size_t row = r0 + r, wi = w0 + k;
        uint32_t v = 0;
        if (row < a.rows_valid && wi < row_words) {
            const uint8_t* p = a.in + row * a.in_pitch + wi * 4;
            if (aligned) {
                v = __ldg(reinterpret_cast<const uint32_t*>(p));
            } else {
                v = (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) |
                    ((uint32_t)p[3] << 24);
            }
        }
        tile[r][k] = v;
    }
    __syncthreads();

    constexpr uint32_t MASK = sample_mask<NBITS>();
    for (int i = threadIdx.x; i < G::TC * G::OW; i += 256) {
        const int cl = i / G::OW, w = i % G::OW;
        const size_t c = c0 + cl;
        const size_t gw = r0 / G::SPW + w;
        if (c >= a.nchans || gw >= a.tr_words) continue;
        const size_t ow = a.tr_word_offset + gw;
        const int bit = cl * NBITS, kw = bit >> 5, sh = bit & 31;
        uint32_t out = 0;
#pragma unroll
        for (int s = 0; s < G::SPW; ++s) {
            const uint32_t v = (tile[w * G::SPW + s][kw] >> sh) & MASK;
            out |= v << ((s * NBITS) & 31);
        }
        a.tr[c * a.tr_pitch_words + ow] = out;
    }
}

// ---------------------------------------------------------------------------
// K2p: plain form -- the reference thread decomposition on our layout
// (block 8 sample pairs x 32 DMs, src/tdd/dedisperse/TDDKernel.cu:133-151)
// ---------------------------------------------------------------------------
template <int NBITS>
__global__ void __launch_bounds__(256) dedisperse_plain_kernel(DedisperseArgs a)
{
    using Sum = typename std::conditional<NBITS == 32, unsigned long long, uint32_t>::type;
    constexpr int SPW = 32 / NBITS;
    constexpr uint32_t MASK = sample_mask<NBITS>();
    const size_t tp = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int slot = blockIdx.y * blockDim.y + threadIdx.y;
    if (slot >= a.ndm) return;
    const size_t t = tp * 2;
    if (t >= a.nsamp_out) return;
    const float dm = a.dms[slot];
    Sum s0 = 0, s1 = 0;
    for (int j = 0; j < a.nact; ++j) {
        const int c = a.chan_list[j];
        const uint32_t km = a.km_vals[j];
        const uint32_t d = delay_rn(dm, a.delay_table[c]);
        const uint32_t* row = a.tr + (size_t)c * a.tr_pitch_words;
        const size_t p0 = t + d, p1 = p0 + 1;
        const uint32_t v0 = (__ldg(row + p0 / SPW) >> ((p0 % SPW) * NBITS % 32)) & MASK;
        const uint32_t v1 = (__ldg(row + p1 / SPW) >> ((p1 % SPW) * NBITS % 32)) & MASK;
        s0 += (Sum)(uint32_t)(km * v0);
        s1 += (Sum)(uint32_t)(km * v1);
    }
    const int row = a.perm ? a.perm[slot] : slot;
    const size_t base = (size_t)row * a.out_stride;
    store_out(a.out, base + t, a.out_nbits, s0, a.den, a.factor);
    if (t + 1 < a.nsamp_out) store_out(a.out, base + t + 1, a.out_nbits, s1, a.den, a.factor);
}

// ---------------------------------------------------------------------------
// K2: tiled form
//
// Block = BD DMs (NW warps x DPW DMs each) x BT output samples (32 lanes x R
// consecutive samples each, R = J words). Channels are staged CS at a time:
// for every staged channel, the window of input words that any DM of the
// block can touch is copied into shared memory (cp.async, double buffered).
// A lane reads J+1 consecutive words of a channel window at word offset
// (q + lane*J); with J odd the 32 lanes hit 32 different banks. A funnel
// shift aligns each word to the lane's sample boundary, then masks split it
// into narrow lanes (8 or 16 bit) that are summed as plain 32-bit adds
// (SIMD within a register). Narrow lanes are flushed into exact 32-bit sums
// before they can overflow.
// ---------------------------------------------------------------------------
template <int NBITS>
struct Tiled;
// J: words per lane (odd); DPW: DMs per warp; FLP: channel pairs per narrow
// flush (narrow lane capacity / (2 * max sample)).
// NW: warps per block. The 8-bit kernel runs 32 warps of one DM each (more
// warps per scheduler to hide shared-memory latency); the generic kernel 16
// warps of two DMs.
template <> struct Tiled<8>  { static constexpr int J = 5, DPW = 1, NW = 32, NN = 2, FLP = 128; };
template <> struct Tiled<4>  { static constexpr int J = 3, DPW = 2, NW = 16, NN = 2, FLP = 8; };
template <> struct Tiled<2>  { static constexpr int J = 1, DPW = 2, NW = 16, NN = 4, FLP = 42; };
template <> struct Tiled<1>  { static constexpr int J = 1, DPW = 1, NW = 16, NN = 8, FLP = 127; };
template <> struct Tiled<16> { static constexpr int J = 7, DPW = 2, NW = 16, NN = 1, FLP = 0; };
template <> struct Tiled<32> { static constexpr int J = 7, DPW = 2, NW = 16, NN = 1, FLP = 0; };

template <int NBITS>
struct TiledGeom {
    static constexpr int SPW = 32 / NBITS;
    static constexpr int J = Tiled<NBITS>::J;
    static constexpr int R = J * SPW;       // samples per lane
    static constexpr int BT = 32 * R;       // samples per block
    static constexpr int DPW = Tiled<NBITS>::DPW;
    static constexpr int NW = Tiled<NBITS>::NW;
    static constexpr int BD = NW * DPW;
    static constexpr int NT = NW * 32;
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }

// Set by a kernel whose bounded wait expired (device-wide; read and cleared
// by tdd_take_error).

// mbarrier + bulk asynchronous copy (global -> shared of this CTA only).
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t* b)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes)
{
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}
// `bytes` (a multiple of 16) from global `src` to shared `dst` (both 16-byte
// aligned); completion counted on mbarrier b.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* b)
{
    asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(b))
                 : "memory");
}
// Limit of the bounded mbarrier waits (nanoseconds of global time) and the
// expiry test switch (rt::wait_limit_ns, rt::wait_expiry_test), passed to
// the kernels by value.
struct WaitCfg {
    unsigned long long ns;
    int expiry_test;
};
WaitCfg wait_cfg() { return WaitCfg{rt::wait_limit_ns(), rt::wait_expiry_test() ? 1 : 0}; }

// Wait for phase `parity` of b; false after limit_ns of global time (checked
// every 16 polls) or 2^28 polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* b, uint32_t parity, unsigned long long limit_ns)
{
    const uint32_t addr = smem_addr(b);
    uint64_t t0 = 0;
    for (uint32_t i = 0; i < (1u << 28); ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 15u) == 15u) {
            uint64_t t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            if (t0 == 0) t0 = t;
            else if (t - t0 > limit_ns) return false;
        }
    }
    return false;
}
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::); }

// Narrow-lane accumulation of two channels' aligned words v1, v2 for word k.
template <int NBITS, int J, int NN>
__device__ __forceinline__ void narrow_add(uint32_t (&n)[J][NN], int k, uint32_t v1, uint32_t v2)
{
    if constexpr (NBITS == 8) {
        // even bytes in place; odd bytes moved down into 16-bit lanes with
        // one byte permute each (selector 0x4341: b1, 0, b3, 0)
        constexpr uint32_t M = 0x00FF00FFu;
        n[k][0] += (v1 & M) + (v2 & M);
        n[k][1] += __byte_perm(v1, 0u, 0x4341) + __byte_perm(v2, 0u, 0x4341);
    } else if constexpr (NBITS == 4) {
        constexpr uint32_t M = 0x0F0F0F0Fu;
        n[k][0] += (v1 & M) + (v2 & M);
        n[k][1] += ((v1 >> 4) & M) + ((v2 >> 4) & M);
    } else if constexpr (NBITS == 2) {
        constexpr uint32_t M = 0x03030303u;
#pragma unroll
        for (int m = 0; m < 4; ++m) n[k][m] += ((v1 >> (2 * m)) & M) + ((v2 >> (2 * m)) & M);
    } else if constexpr (NBITS == 1) {
        constexpr uint32_t M = 0x01010101u;
#pragma unroll
        for (int m = 0; m < 8; ++m) n[k][m] += ((v1 >> m) & M) + ((v2 >> m) & M);
    }
}

// Narrow lanes -> exact 32-bit sums; acc index = sample offset in the lane run.
template <int NBITS, int J, int NN, int R>
__device__ __forceinline__ void narrow_flush(uint32_t (&n)[J][NN], uint32_t (&acc)[R])
{
#pragma unroll
    for (int k = 0; k < J; ++k) {
        if constexpr (NBITS == 8) {
            acc[4 * k + 0] += n[k][0] & 0xFFFFu;
            acc[4 * k + 2] += n[k][0] >> 16;
            acc[4 * k + 1] += n[k][1] & 0xFFFFu;
            acc[4 * k + 3] += n[k][1] >> 16;
        } else if constexpr (NBITS == 4) {
#pragma unroll
            for (int L = 0; L < 4; ++L) {
                acc[8 * k + 2 * L] += (n[k][0] >> (8 * L)) & 0xFFu;
                acc[8 * k + 2 * L + 1] += (n[k][1] >> (8 * L)) & 0xFFu;
            }
        } else if constexpr (NBITS == 2) {
#pragma unroll
            for (int m = 0; m < 4; ++m)
#pragma unroll
                for (int L = 0; L < 4; ++L) acc[16 * k + 4 * L + m] += (n[k][m] >> (8 * L)) & 0xFFu;
        } else if constexpr (NBITS == 1) {
#pragma unroll
            for (int m = 0; m < 8; ++m)
#pragma unroll
                for (int L = 0; L < 4; ++L) acc[32 * k + 8 * L + m] += (n[k][m] >> (8 * L)) & 0xFFu;
        }
#pragma unroll
        for (int m = 0; m < NN; ++m) n[k][m] = 0;
    }
}

template <int NBITS>
__global__ void __launch_bounds__(TiledGeom<NBITS>::NT, 1) dedisperse_tiled_kernel(DedisperseArgs a)
{
    using G = TiledGeom<NBITS>;
    constexpr int SPW = G::SPW, J = G::J, R = G::R, BT = G::BT, DPW = G::DPW, BD = G::BD,
                  NT = G::NT, NN = Tiled<NBITS>::NN, FLP = Tiled<NBITS>::FLP;
    using Acc = typename std::conditional<NBITS == 32, unsigned long long, uint32_t>::type;

    extern __shared__ __align__(16) uint32_t smem[];
    const int W = a.win_words, CS = a.chan_per_stage;
    uint32_t* s_win = smem;                       // [2][CS][W]
    uint32_t* s_info = s_win + 2 * CS * W;        // [2][BD][CS]
    float* s_dm = reinterpret_cast<float*>(s_info + 2 * BD * CS);  // [BD]

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int i0 = blockIdx.x * BD;
    const size_t t0 = (size_t)blockIdx.y * BT;
    const int nvalid = min(BD, a.ndm - i0);
    const float dm_first = a.dms[i0];
    const float dm_last = a.dms[i0 + nvalid - 1];
    if (tid < BD) s_dm[tid] = a.dms[i0 + min(tid, nvalid - 1)];
    __syncthreads();

    // Stage `stage` of the channel list into buffer `buf`.
    auto prep = [&](int stage, int buf) {
        const int32_t* cl = a.chan_list + (size_t)stage * CS;
        for (int j = warp; j < CS; j += G::NW) {
            const int c = cl[j];
            const float dl = a.delay_table[c];
            const uint32_t lo = min(delay_rn(dm_first, dl), delay_rn(dm_last, dl));
            const size_t A = ((t0 + lo) / (4 * SPW)) * (4 * SPW);
            const uint32_t* src = a.tr + (size_t)c * a.tr_pitch_words + A / SPW;
            uint32_t* dst = s_win + (size_t)(buf * CS + j) * W;
            for (int k = lane * 4; k < W; k += 128) cp_async16(dst + k, src + k);
        }
        for (int idx = tid; idx < BD * CS; idx += NT) {
            const int slot = idx / CS, j = idx - slot * CS;
            const int c = cl[j];
            const float dl = a.delay_table[c];
            const uint32_t lo = min(delay_rn(dm_first, dl), delay_rn(dm_last, dl));
            const size_t A = ((t0 + lo) / (4 * SPW)) * (4 * SPW);
            const uint32_t d = delay_rn(s_dm[slot], dl);
            const uint32_t rel = (uint32_t)(t0 + d - A);
            s_info[(buf * BD + slot) * CS + j] = ((rel / SPW) << 5) | ((rel % SPW) * NBITS);
        }
    };

    Acc acc[DPW][R];
    uint32_t nar[DPW][J][NN];
#pragma unroll
    for (int di = 0; di < DPW; ++di) {
#pragma unroll
        for (int k = 0; k < R; ++k) acc[di][k] = 0;
#pragma unroll
        for (int k = 0; k < J; ++k)
#pragma unroll
            for (int m = 0; m < NN; ++m) nar[di][k][m] = 0;
    }

    prep(0, 0);
    cp_async_commit();
    int pairs = 0;
    for (int s = 0; s < a.nstages; ++s) {
        const int buf = s & 1;
        if (s + 1 < a.nstages) prep(s + 1, buf ^ 1);
        cp_async_commit();
        cp_async_wait_1();
        __syncthreads();

        const uint32_t* win = s_win + (size_t)buf * CS * W;
        const uint32_t* info = s_info + buf * BD * CS;
        for (int j = 0; j < CS; j += 2) {
#pragma unroll
            for (int di = 0; di < DPW; ++di) {
                const int slot = warp * DPW + di;
                const uint32_t f1 = info[slot * CS + j];
                const uint32_t f2 = info[slot * CS + j + 1];
                const uint32_t* p1 = win + j * W + (f1 >> 5) + lane * J;
                const uint32_t* p2 = win + (j + 1) * W + (f2 >> 5) + lane * J;
                if constexpr (NBITS == 32) {
#pragma unroll
                    for (int k = 0; k < J; ++k)
                        acc[di][k] += (unsigned long long)p1[k] + (unsigned long long)p2[k];
                } else {
                    const uint32_t b1 = f1 & 31, b2 = f2 & 31;
                    uint32_t w1[J + 1], w2[J + 1];
#pragma unroll
                    for (int k = 0; k <= J; ++k) {
                        w1[k] = p1[k];
                        w2[k] = p2[k];
                    }
#pragma unroll
                    for (int k = 0; k < J; ++k) {
                        const uint32_t v1 = __funnelshift_r(w1[k], w1[k + 1], b1);
                        const uint32_t v2 = __funnelshift_r(w2[k], w2[k + 1], b2);
                        if constexpr (NBITS == 16) {
                            acc[di][2 * k] += (v1 & 0xFFFFu) + (v2 & 0xFFFFu);
                            acc[di][2 * k + 1] += (v1 >> 16) + (v2 >> 16);
                        } else {
                            narrow_add<NBITS, J, NN>(nar[di], k, v1, v2);
                        }
                    }
                }
            }
            if constexpr (FLP > 0) {
                if (++pairs == FLP) {
#pragma unroll
                    for (int di = 0; di < DPW; ++di) narrow_flush<NBITS, J, NN, R>(nar[di], acc[di]);
                    pairs = 0;
                }
            }
        }
        __syncthreads();
    }
    if constexpr (FLP > 0) {
#pragma unroll
        for (int di = 0; di < DPW; ++di) narrow_flush<NBITS, J, NN, R>(nar[di], acc[di]);
    }

#pragma unroll
    for (int di = 0; di < DPW; ++di) {
        const int slot = warp * DPW + di;
        if (slot >= nvalid) continue;
        const int row = a.perm ? a.perm[i0 + slot] : i0 + slot;
        const size_t base = (size_t)row * a.out_stride;
        const size_t tl = t0 + (size_t)lane * R;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const size_t t = tl + k;
            if (t < a.nsamp_out) store_out(a.out, base + t, a.out_nbits, acc[di][k], a.den, a.factor);
        }
    }
}

// ---------------------------------------------------------------------------
// K2 for 8-bit input.
//
// Byte alignment: each staged channel window is also stored shifted by 1, 2
// and 3 bytes (built once per stage with 16-byte shared loads/stores, reused
// by all BD DMs), so a lane reads already-aligned words.
//
// Accumulation (two accumulators per word of 4 samples b0..b3, exact):
//   S += w1 + w2                          raw words, carries run across bytes
//   O += prmt(w1) + prmt(w2)              odd bytes (b1, b3) in 16-bit lanes
// After at most 256 channels, E = S - 256*O holds the even bytes (b0, b2) in
// 16-bit lanes: S = sum(b0 + b1 2^8 + b2 2^16 + b3 2^24) and
// 256*O = sum(b1 2^8 + b3 2^24) modulo 2^32, and each lane sum of E and O is
// at most 256*255 < 2^16, so E < 2^32 and every lane is exact. Per word and
// channel pair: one 3-input add and two byte permutes on the ALU pipe, two
// IMAD (multiplier `one` = 1, a kernel argument) on the FMA pipe, two
// shared loads.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t imad(uint32_t a, uint32_t b, uint32_t c)
{
    uint32_t d;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

constexpr int T8_FLUSH_CHANNELS = 256;

// Tile shapes of the 8-bit kernel (one DM per warp): J words (4J samples)
// per lane, NW warps = NW DMs per block. Index = the plan's `variant`.
struct T8Shape { int J, NW; };
constexpr T8Shape T8_SHAPES[] = {{5, 28}, {5, 32}, {5, 24}, {3, 32}, {7, 16}};
constexpr int T8_NSHAPES = sizeof(T8_SHAPES) / sizeof(T8_SHAPES[0]);

// One block tile: DMs [bx*NW, bx*NW + NW) x samples [by*BT, by*BT + BT) of
// the series described by `a`. Called by the one-tile-per-block kernel and
// by the persistent multi-beam kernel.
template <int J, int NW>
__device__ __forceinline__ void tiled8_tile(const DedisperseArgs& a, int bx, size_t by, uint32_t one)
{
    constexpr int R = 4 * J, BT = 32 * R, BD = NW, NT = NW * 32;

    extern __shared__ __align__(16) uint32_t smem[];
    const int W = a.win_words, CS = a.chan_per_stage;
    const int CSW = CS * W;
    uint32_t* s_win = smem;                        // [2][CS][W]   raw windows
    uint32_t* s_shift = s_win + 2 * CSW;           // [3][CS][W]   shifted by 1..3 bytes
    uint32_t* s_info = s_shift + 3 * CSW;          // [2][BD][CS]  word offset into smem
    int* s_need = reinterpret_cast<int*>(s_info + 2 * BD * CS);    // [2][CS] words used per row
    float* s_dm = reinterpret_cast<float*>(s_need + 2 * CS);       // [BD]

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int i0 = bx * BD;
    const size_t t0 = by * BT;
    const int nvalid = min(BD, a.ndm - i0);
    const float dm_first = a.dms[i0];
    const float dm_last = a.dms[i0 + nvalid - 1];
    if (tid < BD) s_dm[tid] = a.dms[i0 + min(tid, nvalid - 1)];
    __syncthreads();

    // Window of channel row j: words [A/4, A/4 + need) of the channel, where
    // A is the block's earliest read rounded down to 16 samples and need
    // covers the latest DM's read of the last lane (plus the one word the
    // shifted copies look ahead). need <= W (W is the maximum over blocks).
    auto prep = [&](int stage, int buf) {
        const int32_t* cl = a.chan_list + (size_t)stage * CS;
        for (int j = warp; j < CS; j += NW) {
            const int c = cl[j];
            const float dl = a.delay_table[c];
            const uint32_t d0 = delay_rn(dm_first, dl), d1 = delay_rn(dm_last, dl);
            const uint32_t lo = min(d0, d1), hi = max(d0, d1);
            const size_t A = ((t0 + lo) / 16) * 16;
            const int need = min(W, (int)((t0 + hi - A) / 4) + 32 * J + 1);
            const uint32_t* src = a.tr + (size_t)c * a.tr_pitch_words + A / 4;
            uint32_t* dst = s_win + buf * CSW + j * W;
            for (int k = lane * 4; k < need; k += 128) cp_async16(dst + k, src + k);
            if (lane == 0) s_need[buf * CS + j] = need;
        }
        for (int idx = tid; idx < BD * CS; idx += NT) {
            const int slot = idx / CS, j = idx - slot * CS;
            const int c = cl[j];
            const float dl = a.delay_table[c];
            const uint32_t lo = min(delay_rn(dm_first, dl), delay_rn(dm_last, dl));
            const size_t A = ((t0 + lo) / 16) * 16;
            const uint32_t rel = (uint32_t)(t0 + delay_rn(s_dm[slot], dl) - A);
            const uint32_t r = rel & 3u, q = rel >> 2;
            const uint32_t base = r == 0 ? (uint32_t)(buf * CSW) : (uint32_t)(2 * CSW + (r - 1) * CSW);
            s_info[(buf * BD + slot) * CS + j] = base + (uint32_t)(j * W) + q;
        }
    };

    uint32_t acc[R];
    uint32_t sw[J], so[J];
#pragma unroll
    for (int k = 0; k < R; ++k) acc[k] = 0;
#pragma unroll
    for (int k = 0; k < J; ++k) sw[k] = so[k] = 0;
    auto flush = [&]() {
#pragma unroll
        for (int k = 0; k < J; ++k) {
            const uint32_t e = imad(so[k], 0xFFFFFF00u, sw[k]);  // S - 256*O
            acc[4 * k + 0] += e & 0xFFFFu;
            acc[4 * k + 2] += e >> 16;
            acc[4 * k + 1] += so[k] & 0xFFFFu;
            acc[4 * k + 3] += so[k] >> 16;
            sw[k] = so[k] = 0;
        }
    };

    prep(0, 0);
    cp_async_commit();
    int since_flush = 0;  // channels accumulated since the last flush
    const int slot = warp;
    for (int s = 0; s < a.nstages; ++s) {
        const int buf = s & 1;
        asm volatile("cp.async.wait_group 0;\n" ::);
        __syncthreads();
        // Shifted copies of this stage's windows, 4 words per lane step; the
        // word after a lane's four comes from the next lane (or, for lane 31,
        // from shared memory). The last word of each shifted row is never read.
        {
            const uint32_t* src = s_win + buf * CSW;
            for (int j = warp; j < CS; j += NW) {
                const uint32_t* row = src + j * W;
                const int need = s_need[buf * CS + j];
                for (int k0 = 0; k0 < need; k0 += 128) {
                    const int k = k0 + lane * 4;
                    uint4 v = make_uint4(0u, 0u, 0u, 0u);
                    if (k < need) v = *reinterpret_cast<const uint4*>(row + k);
                    uint32_t nx = __shfl_down_sync(0xFFFFFFFFu, v.x, 1);
                    if (lane == 31) nx = (k + 4 < W) ? row[k + 4] : 0u;
                    if (k < need) {
                        const int o = j * W + k;
                        *reinterpret_cast<uint4*>(s_shift + o) =
                            make_uint4(__funnelshift_r(v.x, v.y, 8), __funnelshift_r(v.y, v.z, 8),
                                       __funnelshift_r(v.z, v.w, 8), __funnelshift_r(v.w, nx, 8));
                        *reinterpret_cast<uint4*>(s_shift + CSW + o) =
                            make_uint4(__funnelshift_r(v.x, v.y, 16), __funnelshift_r(v.y, v.z, 16),
                                       __funnelshift_r(v.z, v.w, 16), __funnelshift_r(v.w, nx, 16));
                        *reinterpret_cast<uint4*>(s_shift + 2 * CSW + o) =
                            make_uint4(__funnelshift_r(v.x, v.y, 24), __funnelshift_r(v.y, v.z, 24),
                                       __funnelshift_r(v.z, v.w, 24), __funnelshift_r(v.w, nx, 24));
                    }
                }
            }
        }
        __syncthreads();
        if (s + 1 < a.nstages) prep(s + 1, buf ^ 1);
        cp_async_commit();

        // 16-bit lanes hold at most 256 channels of 8-bit samples
        if (since_flush + CS > T8_FLUSH_CHANNELS) {
            flush();
            since_flush = 0;
        }
        const uint32_t* info = s_info + (buf * BD + slot) * CS;
#pragma unroll 1
        for (int j = 0; j < CS; j += 2) {
            const uint2 f = *reinterpret_cast<const uint2*>(info + j);
            const uint32_t* p1 = smem + f.x + lane * J;
            const uint32_t* p2 = smem + f.y + lane * J;
            uint32_t w1[J], w2[J];
#pragma unroll
            for (int k = 0; k < J; ++k) {
                w1[k] = p1[k];
                w2[k] = p2[k];
            }
#pragma unroll
            for (int k = 0; k < J; ++k) {
                sw[k] = sw[k] + w1[k] + w2[k];
                so[k] = imad(__byte_perm(w1[k], 0u, 0x4341), one, so[k]);
                so[k] = imad(__byte_perm(w2[k], 0u, 0x4341), one, so[k]);
            }
        }
        since_flush += CS;
    }
    flush();

    if (slot < nvalid) {
        const int row = a.perm ? a.perm[i0 + slot] : i0 + slot;
        const size_t base = (size_t)row * a.out_stride;
        const size_t tl = t0 + (size_t)lane * R;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const size_t t = tl + k;
            if (t < a.nsamp_out) store_out(a.out, base + t, a.out_nbits, acc[k], a.den, a.factor);
        }
    }
}

template <int J, int NW>
__global__ void __launch_bounds__(NW * 32, 1) dedisperse_tiled8_kernel(DedisperseArgs a, uint32_t one)
{
    tiled8_tile<J, NW>(a, blockIdx.x, blockIdx.y, one);
}

// Persistent form over many series (beams): block b takes work items b,
// b + gridDim.x, ...; item i belongs to the beam with
// item_start[beam] <= i < item_start[beam + 1] and is tile
// (bx, by) = (local % nbx, local / nbx) of that beam. Each beam's arguments
// are copied to shared memory before its tiles run. TILE runs one tile.
template <typename TILE>
__device__ __forceinline__ void batch_items(const DedisperseArgs* __restrict__ args,
                                            const unsigned long long* __restrict__ item_start,
                                            const int* __restrict__ nbx, int nbeams, TILE&& tile)
{
    __shared__ DedisperseArgs s_a;
    __shared__ int s_beam;
    const unsigned long long total = item_start[nbeams];
    int cur = -1;
    for (unsigned long long item = blockIdx.x; item < total; item += gridDim.x) {
        if (threadIdx.x == 0) {
            int lo = 0, hi = nbeams - 1;  // last beam with item_start <= item
            while (lo < hi) {
                const int mid = (lo + hi + 1) / 2;
                if (item_start[mid] <= item) lo = mid;
                else hi = mid - 1;
            }
            s_beam = lo;
        }
        __syncthreads();
        const int beam = s_beam;
        if (beam != cur) {
            constexpr int NWORDS = (int)(sizeof(DedisperseArgs) / 4);
            static_assert(sizeof(DedisperseArgs) % 4 == 0, "argument block is copied as words");
            const uint32_t* src = reinterpret_cast<const uint32_t*>(args + beam);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&s_a);
            for (int w = threadIdx.x; w < NWORDS; w += blockDim.x) dst[w] = src[w];
            cur = beam;
        }
        __syncthreads();
        const unsigned long long local = item - item_start[beam];
        const int n = nbx[beam];
        tile(s_a, (int)(local % (unsigned long long)n), (size_t)(local / (unsigned long long)n));
        __syncthreads();  // shared memory is reused by the next item
    }
}

template <int J, int NW>
__global__ void __launch_bounds__(NW * 32, 1)
dedisperse_tiled8_batch_kernel(const DedisperseArgs* __restrict__ args,
                               const unsigned long long* __restrict__ item_start,
                               const int* __restrict__ nbx, int nbeams, uint32_t one)
{
    batch_items(args, item_start, nbx, nbeams,
                [&](const DedisperseArgs& a, int bx, size_t by) { tiled8_tile<J, NW>(a, bx, by, one); });
}

// ---------------------------------------------------------------------------
// K1d + K2q: the byte kernel on quad-strided rows.
//
// For a period of P words, word n of a quad-strided row holds samples n,
// n + P, n + 2P, n + 3P of the channel (byte i = sample n + i*P). A block
// tile covers output samples [t0, t0 + 4P): lane word m (0 <= m < P) of a DM
// accumulates the row's word t0 + m + d(dm, c) for every channel, whose four
// bytes are exactly the four samples t0 + m + i*P + d(dm, c). Every delay is
// therefore a whole-word offset: the rows are built once per gulp in HBM
// (four times the packed size) instead of byte-shifted copies per block and
// stage, and a stage is one window copy and one barrier. Lane l owns words
// l, l + 32, ..., so a warp's shared loads are 32 consecutive words.
// ---------------------------------------------------------------------------
// Four NBITS-bit fields (LSB first) widened to four bytes.
template <int NBITS>
__device__ __forceinline__ uint32_t widen4(uint32_t x)
{
    if constexpr (NBITS == 8) {
        return x;
    } else {
        constexpr uint32_t M = (1u << NBITS) - 1u;
        return (x & M) | (((x >> NBITS) & M) << 8) | (((x >> (2 * NBITS)) & M) << 16) |
               (((x >> (3 * NBITS)) & M) << 24);
    }
}

// K1d: quad-strided rows built straight from the time-major input. A block
// takes QD_WORDS input words of every row (QD_WORDS * 32 / NBITS channels)
// and QD_N output words n0 .. n0 + QD_N - 1: it stages the four row windows
// n0 + i*P .. n0 + i*P + QD_N - 1 (i = 0..3) in shared memory, then each
// thread turns one staged word of each window (the same 32 / NBITS channels,
// rows n + i*P) into output word n of four channels at a time (widen to
// bytes, 4x4 byte transpose). Lanes take consecutive n, so the shared reads
// (row stride QD_WORDS + 1) are conflict-free and each store is a 128-byte
// run of one channel's row. An input row is read by the four blocks whose
// windows contain it, close together in launch order (L2 hits).
constexpr int QD_WORDS = 16, QD_N = 128, QD_THREADS = 256;

template <int NBITS>
__global__ void __launch_bounds__(QD_THREADS) quad_direct_kernel(QuadDirectArgs a, int aligned)
{
    constexpr int CH = QD_WORDS * 32 / NBITS;  // channels per block
    constexpr int LOADS = 4 * QD_N * QD_WORDS / QD_THREADS;
    __shared__ uint32_t tile[4][QD_N][QD_WORDS + 1];
    const size_t n0 = (size_t)blockIdx.x * QD_N;
    const size_t w0 = (size_t)blockIdx.y * QD_WORDS;
    const size_t row_words = a.nchans * NBITS / 32;
    const size_t P = (size_t)a.period_words;

    uint32_t v[LOADS];
#pragma unroll
    for (int it = 0; it < LOADS; ++it) {
        const int idx = threadIdx.x + it * QD_THREADS;
        const int k = idx % QD_WORDS, r = (idx / QD_WORDS) % QD_N, i = idx / (QD_WORDS * QD_N);
        const size_t row = n0 + r + (size_t)i * P, wi = w0 + k;
        v[it] = 0u;
        if (row < a.rows_valid && wi < row_words) {
            const uint8_t* p = a.in + row * a.in_pitch + wi * 4;
            v[it] = aligned ? __ldg(reinterpret_cast<const uint32_t*>(p))
                            : (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) |
                                  ((uint32_t)p[3] << 24);
        }
    }
#pragma unroll
    for (int it = 0; it < LOADS; ++it) {
        const int idx = threadIdx.x + it * QD_THREADS;
        tile[idx / (QD_WORDS * QD_N)][(idx / QD_WORDS) % QD_N][idx % QD_WORDS] = v[it];
    }
    __syncthreads();

    const size_t c0 = w0 * 32 / NBITS;
    for (int item = threadIdx.x; item < (CH / 4) * QD_N; item += QD_THREADS) {
        const int r = item % QD_N, g = item / QD_N;  // output word n0 + r, channels c0 + 4g ..
        const size_t n = n0 + r, c = c0 + 4 * (size_t)g;
        if (n >= a.q_pitch_words || c >= a.nchans) continue;
        const int bit = 4 * g * NBITS, kw = bit >> 5, sh = bit & 31;
        uint32_t e[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) e[i] = widen4<NBITS>(tile[i][r][kw] >> sh);
        // word j (channel c + j) = byte j of e[0..3]
        const uint32_t a_lo = __byte_perm(e[0], e[1], 0x5140), a_hi = __byte_perm(e[0], e[1], 0x7362);
        const uint32_t b_lo = __byte_perm(e[2], e[3], 0x5140), b_hi = __byte_perm(e[2], e[3], 0x7362);
        uint32_t* dst = a.q + c * a.q_pitch_words + n;
        dst[0] = __byte_perm(a_lo, b_lo, 0x5410);
        dst[a.q_pitch_words] = __byte_perm(a_lo, b_lo, 0x7632);
        dst[2 * a.q_pitch_words] = __byte_perm(a_hi, b_hi, 0x5410);
        dst[3 * a.q_pitch_words] = __byte_perm(a_hi, b_hi, 0x7632);
    }
}

// Tile shapes of the quad-strided kernel: J words per lane (P = 32J), NW warps
// = NW DMs per block (one DM per warp).
struct Q8Shape { int J, NW; };
constexpr Q8Shape Q8_SHAPES[] = {{20, 12}, {22, 12}, {18, 12}, {16, 12}};
constexpr int Q8_NSHAPES = sizeof(Q8_SHAPES) / sizeof(Q8_SHAPES[0]);
constexpr int Q8_MAX_STAGE = 64;

// Dynamic shared memory of a quad-strided launch: the opt-in maximum less the
// static buffers (span reduction, one word per warp; channels and delays of
// two stages; for the persistent form the beam's argument block).
constexpr size_t kBatchStaticSmem = 256;
constexpr size_t quad_dynamic_smem_bytes(int nw, bool batch = false)
{
    // (64 bytes for the two stage mbarriers and alignment)
    return 227 * 1024 - 4 * (size_t)nw - 2 * 2 * Q8_MAX_STAGE * 4 - 64 - (batch ? kBatchStaticSmem : 0);
}

// Shared loads with 32-bit window addresses and immediate offsets. Volatile:
// the windows change at every stage barrier.
template <uint32_t OFF>
__device__ __forceinline__ uint32_t lds_imm(uint32_t addr)
{
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1+%2];\n" : "=r"(v) : "r"(addr), "n"(OFF));
    return v;
}

__device__ __forceinline__ uint4 lds128(uint32_t addr)
{
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"(addr));
    return v;
}

// w[k] = word (lane + 32k) of a window row, addr = row address + 4 * lane
template <int J, uint32_t... K>
__device__ __forceinline__ void lds_lane_words(uint32_t addr, uint32_t (&w)[J],
                                               std::integer_sequence<uint32_t, K...>)
{
    ((w[K] = lds_imm<128u * K>(addr)), ...);
}

template <int J, int NW>
__device__ __forceinline__ void quad8_tile(const DedisperseArgs& a, int bx, size_t by, uint32_t one, WaitCfg wc)
{
    constexpr int P = 32 * J;
    constexpr int NT = NW * 32;
    constexpr size_t BT = 4 * (size_t)P;

    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ uint32_t s_red[NW];
    __shared__ int32_t s_cl[2][Q8_MAX_STAGE];  // channel of each row, stages fetched ahead
    __shared__ float s_cdl[2][Q8_MAX_STAGE];   // its delay
    __shared__ uint64_t s_full[2];             // window copies of stage buffer b landed
    __shared__ uint64_t s_never;               // expiry test: nothing arrives on it

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i0 = bx * NW;
    const size_t t0 = by * BT;
    const int nvalid = min(NW, a.ndm - i0);
    const float dm_first = a.dms[i0];
    const float dm_last = a.dms[i0 + nvalid - 1];
    const float dm_own = a.dms[i0 + min(warp, nvalid - 1)];
    const int npad = (a.nact + 3) & ~3;  // channel list length used (padded to 4)

    // This block's window W (words per row) from its own delay span: the
    // largest (hi - lo4) over the channels, plus the P words of a lane set,
    // rounded to 16 bytes. Then as many channels per stage (a multiple of 4,
    // at most Q8_MAX_STAGE) as the launch's shared memory holds.
    // one arrival per warp and stage buffer phase (after its copies are counted)
    if (threadIdx.x == 0) {
        mbar_init(&s_full[0], NW);
        mbar_init(&s_full[1], NW);
        mbar_init(&s_never, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    uint32_t vmax = 0;
    for (int j = threadIdx.x; j < npad; j += NT) {
        const float dl = a.chan_delay[j];
        const uint32_t d0 = delay_rn(dm_first, dl), d1 = delay_rn(dm_last, dl);
        vmax = max(vmax, max(d0, d1) - (min(d0, d1) & ~3u));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vmax = max(vmax, __shfl_xor_sync(0xFFFFFFFFu, vmax, o));
    if (lane == 0) s_red[warp] = vmax;
    __syncthreads();
    vmax = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) vmax = max(vmax, s_red[w]);
    const int W = (int)((vmax + (uint32_t)P + 3u) & ~3u);
    uint32_t smem_bytes;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(smem_bytes));
    const int CS = min(Q8_MAX_STAGE, ((int)(smem_bytes / 4) / (2 * W + 4 + NW)) & ~3);
    const int nstages = (npad + CS - 1) / CS;
    const int CSW = CS * W;
    uint32_t* s_win = smem;                                        // [2][CS][W] row windows
    uint32_t* s_lo = s_win + 2 * CSW;                              // [2][CS] window start - t0
    float* s_dl = reinterpret_cast<float*>(s_lo + 2 * CS);         // [2][CS] channel delay
    uint32_t* s_off = reinterpret_cast<uint32_t*>(s_dl + 2 * CS);  // [NW][CS] per-warp row addresses

    const uint32_t win_addr = (uint32_t)__cvta_generic_to_shared(s_win);
    uint32_t* my_off = s_off + warp * CS;
    const uint32_t my_off_addr = (uint32_t)__cvta_generic_to_shared(my_off);
    const uint32_t lane4 = 4u * (uint32_t)lane;

    // Window of channel row j: words [t0 + lo4, t0 + lo4 + need), lo4 the
    // block's smallest delay rounded down to 4 words (16-byte copies), need
    // covering the largest delay plus the P words of a lane set; need <= W.
    auto stage_size = [&](int stage) { return min(CS, npad - stage * CS); };
    // channels and delays of a stage's rows into s_cl/s_cdl[stage & 1]
    auto fetch = [&](int stage) {
        const int cs = stage_size(stage);
        const size_t g = (size_t)stage * CS;
        for (int j = threadIdx.x; j < cs; j += NT) {
            cp_async4(&s_cl[stage & 1][j], a.chan_list + g + j);
            cp_async4(&s_cdl[stage & 1][j], a.chan_delay + g + j);
        }
    };
    // Lane 0 of each warp copies the warp's rows with one bulk copy each
    // (bytes counted on s_full[buf] before the copy), then arrives.
    auto prep = [&](int stage, int buf) {
        if (lane != 0) return;
        const int cs = stage_size(stage);
        for (int j = warp; j < cs; j += NW) {
            const int c = s_cl[stage & 1][j];
            const float dl = s_cdl[stage & 1][j];
            const uint32_t d0 = delay_rn(dm_first, dl), d1 = delay_rn(dm_last, dl);
            const uint32_t lo4 = min(d0, d1) & ~3u, hi = max(d0, d1);
            const int need = min(W, (int)((hi - lo4 + (uint32_t)P + 3u) & ~3u));
            const uint32_t* src = a.tr + (size_t)c * a.tr_pitch_words + t0 + lo4;
            uint32_t* dst = s_win + buf * CSW + j * W;
            mbar_expect_tx(&s_full[buf], 4u * (uint32_t)need);
            bulk_g2s(dst, src, 4u * (uint32_t)need, &s_full[buf]);
            s_lo[buf * CS + j] = lo4;
            s_dl[buf * CS + j] = dl;
        }
        mbar_arrive(&s_full[buf]);
    };

    uint32_t acc[4 * J];
    uint32_t sw[J], so[J];
#pragma unroll
    for (int k = 0; k < 4 * J; ++k) acc[k] = 0;
#pragma unroll
    for (int k = 0; k < J; ++k) sw[k] = so[k] = 0;
    auto flush = [&]() {
#pragma unroll
        for (int k = 0; k < J; ++k) {
            const uint32_t e = imad(so[k], 0xFFFFFF00u, sw[k]);  // S - 256*O
            acc[4 * k + 0] += e & 0xFFFFu;
            acc[4 * k + 2] += e >> 16;
            acc[4 * k + 1] += so[k] & 0xFFFFu;
            acc[4 * k + 3] += so[k] >> 16;
            sw[k] = so[k] = 0;
        }
    };
    // one channel pair: rows at a1, a2 (byte addresses including 4 * lane)
    auto pair = [&](uint32_t a1, uint32_t a2) {
        uint32_t w1[J], w2[J];
        lds_lane_words<J>(a1, w1, std::make_integer_sequence<uint32_t, J>{});
        lds_lane_words<J>(a2, w2, std::make_integer_sequence<uint32_t, J>{});
#pragma unroll
        for (int k = 0; k < J; ++k) {
            sw[k] = sw[k] + w1[k] + w2[k];
            so[k] = imad(__byte_perm(w1[k], 0u, 0x4341), one, so[k]);
            so[k] = imad(__byte_perm(w2[k], 0u, 0x4341), one, so[k]);
        }
    };

    if (nstages > 0) fetch(0);
    if (nstages > 1) fetch(1);
    cp_async_commit();
    asm volatile("cp.async.wait_group 0;\n" ::);
    __syncthreads();
    if (nstages > 0) prep(0, 0);
    int since_flush = 0;  // channels accumulated since the last flush
    bool failed = false;
    for (int s = 0; s < nstages; ++s) {
        const int buf = s & 1;
        const int cs = stage_size(s);
        asm volatile("cp.async.wait_group 0;\n" ::);
        bool landed = mbar_wait_bounded(&s_full[buf], ((uint32_t)s >> 1) & 1u, wc.ns);
        // expiry test: one more wait, on a barrier nothing arrives on
        if (wc.expiry_test && s == 0) landed = landed && mbar_wait_bounded(&s_never, 0u, wc.ns);
        // stage s landed; every warp is done with stage s - 1
        if (__syncthreads_or(!landed)) {
            // a copy did not complete: wait (bounded) for this stage's copies,
            // the only ones in flight, record the error and leave
            mbar_wait_bounded(&s_full[buf], ((uint32_t)s >> 1) & 1u, wc.ns);
            if (threadIdx.x == 0) atomicExch(a.err, 1u);
            failed = true;
            break;
        }
        if (s + 1 < nstages) prep(s + 1, buf ^ 1);
        if (s + 2 < nstages) fetch(s + 2);  // s_cl/s_cdl[s & 1]: prep(s) finished before the barrier
        cp_async_commit();
        // this warp's row addresses in the stage's windows
        for (int j = lane; j < cs; j += 32) {
            const uint32_t d = delay_rn(dm_own, s_dl[buf * CS + j]);
            my_off[j] = win_addr + 4u * ((uint32_t)(buf * CSW + j * W) + (d - s_lo[buf * CS + j]));
        }
        __syncwarp();

        // 16-bit lanes hold at most 256 channels of 8-bit samples
        if (since_flush + cs > T8_FLUSH_CHANNELS) {
            flush();
            since_flush = 0;
        }
#pragma unroll 1
        for (int j = 0; j < cs; j += 4) {
            const uint4 f = lds128(my_off_addr + 4u * (uint32_t)j);
            pair(f.x + lane4, f.y + lane4);
            pair(f.z + lane4, f.w + lane4);
        }
        since_flush += cs;
    }
    flush();

    if (!failed && warp < nvalid) {
        const int row = a.perm ? a.perm[i0 + warp] : i0 + warp;
        const size_t base = (size_t)row * a.out_stride;
#pragma unroll
        for (int k = 0; k < J; ++k) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const size_t t = t0 + (size_t)(lane + 32 * k) + (size_t)i * P;
                if (t < a.nsamp_out) store_out(a.out, base + t, a.out_nbits, acc[4 * k + i], a.den, a.factor);
            }
        }
    }
    // the barriers are initialised afresh by the next tile of a persistent block
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_inval(&s_full[0]);
        mbar_inval(&s_full[1]);
        mbar_inval(&s_never);
    }
}

template <int J, int NW>
__global__ void __launch_bounds__(NW * 32, 1) dedisperse_quad8_kernel(DedisperseArgs a, uint32_t one, WaitCfg wc)
{
    quad8_tile<J, NW>(a, blockIdx.x, blockIdx.y, one, wc);
}

template <int J, int NW>
__global__ void __launch_bounds__(NW * 32, 1)
dedisperse_quad8_batch_kernel(const DedisperseArgs* __restrict__ args,
                              const unsigned long long* __restrict__ item_start,
                              const int* __restrict__ nbx, int nbeams, uint32_t one, WaitCfg wc)
{
    static_assert(sizeof(DedisperseArgs) + 16 <= kBatchStaticSmem, "static shared memory of the batch form");
    batch_items(args, item_start, nbx, nbeams,
                [&](const DedisperseArgs& a, int bx, size_t by) { quad8_tile<J, NW>(a, bx, by, one, wc); });
}

template <int J, int NW>
void launch_tiled8_shape(const DedisperseArgs& a, cudaStream_t s)
{
    const size_t smem = tiled_smem_bytes(8, a.win_words, a.chan_per_stage, a.variant);
    rt::raise_smem_limit(dedisperse_tiled8_kernel<J, NW>, smem);
    dim3 grid((a.ndm + NW - 1) / NW, (unsigned)((a.nsamp_out + 128 * J - 1) / (128 * J)));
    dedisperse_tiled8_kernel<J, NW><<<grid, NW * 32, smem, s>>>(a, 1u);
    RT_CHECK(cudaGetLastError());
}

template <int V>
void launch_tiled8_variant(const DedisperseArgs& a, cudaStream_t s)
{
    launch_tiled8_shape<T8_SHAPES[V].J, T8_SHAPES[V].NW>(a, s);
}

template <int J, int NW>
void launch_quad8_shape(const DedisperseArgs& a, cudaStream_t s)
{
    // One block per SM (registers): every block may use the whole opt-in
    // shared memory for its windows; a block sizes its stages from its own
    // delay span. The plan's window (the largest span) must fit 4 channels.
    const size_t smem = quad_dynamic_smem_bytes(NW);
    if (tiled_smem_bytes(8, a.win_words, 4, a.variant) > smem)
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "quad-strided window does not fit shared memory");
    rt::raise_smem_limit(dedisperse_quad8_kernel<J, NW>, smem);
    dim3 grid((a.ndm + NW - 1) / NW, (unsigned)((a.nsamp_out + 128 * J - 1) / (128 * J)));
    dedisperse_quad8_kernel<J, NW><<<grid, NW * 32, smem, s>>>(a, 1u, wait_cfg());
    RT_CHECK(cudaGetLastError());
}

template <int V>
void launch_quad8_variant(const DedisperseArgs& a, cudaStream_t s)
{
    launch_quad8_shape<Q8_SHAPES[V].J, Q8_SHAPES[V].NW>(a, s);
}

template <int J, int NW>
void launch_tiled8_batch_shape(const BatchLaunch& b, cudaStream_t s)
{
    auto kfn = dedisperse_tiled8_batch_kernel<J, NW>;
    rt::raise_smem_limit(kfn, b.smem_bytes);
    int dev = 0, sms = 0, per_sm = 0;
    RT_CHECK(cudaGetDevice(&dev));
    RT_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    RT_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, NW * 32, b.smem_bytes));
    if (per_sm < 1) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "batch kernel does not fit on an SM");
    const unsigned long long want = (unsigned long long)sms * per_sm;
    const unsigned grid = (unsigned)std::max<unsigned long long>(1, std::min(want, b.total_items));
    kfn<<<grid, NW * 32, b.smem_bytes, s>>>(b.args, b.item_start, b.nbx, b.nbeams, 1u);
    RT_CHECK(cudaGetLastError());
}

template <int V>
void launch_tiled8_batch_variant(const BatchLaunch& b, cudaStream_t s)
{
    launch_tiled8_batch_shape<T8_SHAPES[V].J, T8_SHAPES[V].NW>(b, s);
}

template <int J, int NW>
void launch_quad8_batch_shape(const BatchLaunch& b, cudaStream_t s)
{
    auto kfn = dedisperse_quad8_batch_kernel<J, NW>;
    const size_t smem = quad_dynamic_smem_bytes(NW, true);
    if (b.smem_bytes > smem)
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "quad-strided window does not fit shared memory");
    rt::raise_smem_limit(kfn, smem);
    int dev = 0, sms = 0, per_sm = 0;
    RT_CHECK(cudaGetDevice(&dev));
    RT_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    RT_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, NW * 32, smem));
    if (per_sm < 1) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "batch kernel does not fit on an SM");
    const unsigned long long want = (unsigned long long)sms * per_sm;
    const unsigned grid = (unsigned)std::max<unsigned long long>(1, std::min(want, b.total_items));
    kfn<<<grid, NW * 32, smem, s>>>(b.args, b.item_start, b.nbx, b.nbeams, 1u, wait_cfg());
    RT_CHECK(cudaGetLastError());
}

template <int V>
void launch_quad8_batch_variant(const BatchLaunch& b, cudaStream_t s)
{
    launch_quad8_batch_shape<Q8_SHAPES[V].J, Q8_SHAPES[V].NW>(b, s);
}

template <int NBITS>
void launch_tiled_n(const DedisperseArgs& a, cudaStream_t s)
{
    if constexpr (NBITS == 8) {
        static_assert(T8_NSHAPES == 5, "dispatch below lists every shape");
        switch (a.variant) {
        case 0: launch_tiled8_variant<0>(a, s); break;
        case 1: launch_tiled8_variant<1>(a, s); break;
        case 2: launch_tiled8_variant<2>(a, s); break;
        case 3: launch_tiled8_variant<3>(a, s); break;
        case 4: launch_tiled8_variant<4>(a, s); break;
        default: DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "unknown tiled kernel variant");
        }
    } else {
        using G = TiledGeom<NBITS>;
            const size_t smem = tiled_smem_bytes(NBITS, a.win_words, a.chan_per_stage, 0);
        rt::raise_smem_limit(dedisperse_tiled_kernel<NBITS>, smem);
        dim3 grid((a.ndm + G::BD - 1) / G::BD, (unsigned)((a.nsamp_out + G::BT - 1) / G::BT));
        dedisperse_tiled_kernel<NBITS><<<grid, G::NT, smem, s>>>(a);
        RT_CHECK(cudaGetLastError());
    }
}

template <int NBITS>
void launch_plain_n(const DedisperseArgs& a, cudaStream_t s)
{
    dim3 block(8, 32);
    dim3 grid((unsigned)((a.nsamp_out + 15) / 16), (a.ndm + 31) / 32);
    dedisperse_plain_kernel<NBITS><<<grid, block, 0, s>>>(a);
    RT_CHECK(cudaGetLastError());
}

template <int NBITS>
void launch_transpose_n(const TransposeArgs& a, cudaStream_t s)
{
    using G = TrGeom<NBITS>;
    const size_t samples = a.tr_words * G::SPW;
    dim3 grid((unsigned)((samples + G::TR - 1) / G::TR), (unsigned)((a.nchans + G::TC - 1) / G::TC));
    const int aligned = ((uintptr_t)a.in % 4 == 0) && (a.in_pitch % 4 == 0);
    transpose_kernel<NBITS><<<grid, 256, 0, s>>>(a, aligned);
    RT_CHECK(cudaGetLastError());
}

}  // namespace

// Variants per input width: 8-bit 0-4 packed-row shapes (T8_SHAPES), 5-8
// quad-strided shapes (Q8_SHAPES); 1/2/4-bit 0 the generic packed-row kernel,
// 1-4 the quad-strided shapes (samples widened to bytes); 16/32-bit 0 only.
unsigned read_error_word(const unsigned* d_err, cudaStream_t s)
{
    unsigned v = 0;
    RT_CHECK(cudaMemcpyAsync(&v, d_err, sizeof(v), cudaMemcpyDeviceToHost, s));
    RT_CHECK(cudaStreamSynchronize(s));
    return v;
}

int tiled_variant_count(int nbits)
{
    return nbits == 8 ? T8_NSHAPES + Q8_NSHAPES : nbits <= 4 ? 1 + Q8_NSHAPES : 1;
}
int tiled_batch_variant_count(int nbits) { return tiled_variant_count(nbits); }

size_t tiled_batch_smem_bytes(int nbits, int win_words, int chan_per_stage, int variant)
{
    // quad-strided: every block uses the whole dynamic budget (its stage size
    // follows its own window)
    if (tiled_variant_quad(nbits, variant)) return quad_dynamic_smem_bytes(tiled_block_dms(nbits, variant), true);
    return tiled_smem_bytes(nbits, win_words, chan_per_stage, variant);
}
// Widths up to 8 bits: the quad-strided {J = 20, 12 warps} shape, the
// fastest measured on the 4096-channel, 3643-DM workload
int tiled_default_variant(int nbits) { return nbits == 8 ? T8_NSHAPES : nbits <= 4 ? 1 : 0; }

static int checked_variant(int nbits, int variant)
{
    if (variant < 0 || variant >= tiled_variant_count(nbits))
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "unknown tiled kernel variant");
    return variant;
}

// Index into Q8_SHAPES of a quad-strided variant, -1 for the others.
static int quad_shape(int nbits, int variant)
{
    checked_variant(nbits, variant);
    if (nbits == 8) return variant >= T8_NSHAPES ? variant - T8_NSHAPES : -1;
    if (nbits <= 4) return variant >= 1 ? variant - 1 : -1;
    return -1;
}

bool tiled_variant_quad(int nbits, int variant) { return quad_shape(nbits, variant) >= 0; }

int tiled_block_samples(int nbits, int variant)
{
    if (quad_shape(nbits, variant) >= 0) return 128 * tiled_lane_words(nbits, variant);
    switch (nbits) {
    case 1: return TiledGeom<1>::BT;
    case 2: return TiledGeom<2>::BT;
    case 4: return TiledGeom<4>::BT;
    case 8: return 128 * tiled_lane_words(8, variant);
    case 16: return TiledGeom<16>::BT;
    default: return TiledGeom<32>::BT;
    }
}

int tiled_block_dms(int nbits, int variant)
{
    const int q = quad_shape(nbits, variant);
    if (q >= 0) return Q8_SHAPES[q].NW;
    switch (nbits) {
    case 1: return TiledGeom<1>::BD;
    case 2: return TiledGeom<2>::BD;
    case 4: return TiledGeom<4>::BD;
    case 8: return T8_SHAPES[variant].NW;
    case 16: return TiledGeom<16>::BD;
    default: return TiledGeom<32>::BD;
    }
}

int tiled_lane_words(int nbits, int variant)
{
    const int q = quad_shape(nbits, variant);
    if (q >= 0) return Q8_SHAPES[q].J;
    switch (nbits) {
    case 1: return TiledGeom<1>::J;
    case 2: return TiledGeom<2>::J;
    case 4: return TiledGeom<4>::J;
    case 8: return T8_SHAPES[variant].J;
    case 16: return TiledGeom<16>::J;
    default: return TiledGeom<32>::J;
    }
}

size_t tiled_smem_bytes(int nbits, int win_words, int chan_per_stage, int variant)
{
    const size_t bd = (size_t)tiled_block_dms(nbits, variant);
    const size_t cs = (size_t)chan_per_stage;
    // quad-strided: two window buffers, window starts and delays per row,
    // one offset per (DM, row)
    if (tiled_variant_quad(nbits, variant)) return (2 * cs * win_words + 4 * cs + bd * cs) * 4ull;
    // 8-bit: two raw buffers plus three byte-shifted copies per stage, and
    // the per-row window lengths
    const size_t windows = nbits == 8 ? 5ull : 2ull;
    const size_t extra = nbits == 8 ? 2ull * cs : 0ull;
    return (windows * cs * win_words + 2ull * bd * cs + extra + bd) * 4ull;
}

// The opt-in maximum of dynamic shared memory per block on sm_100.
size_t tiled_max_smem_bytes() { return 227 * 1024; }

int tiled_stage_channels(int nbits, int win_words, int variant)
{
    // quad-strided: four channels per inner step
    // (quad: the budget of the persistent form, the smaller of the two)
    const bool quad = tiled_variant_quad(nbits, variant);
    const int step = quad ? 4 : 2;
    int cs = quad ? Q8_MAX_STAGE : 32;
    const size_t cap = quad ? quad_dynamic_smem_bytes(tiled_block_dms(nbits, variant), true) : tiled_max_smem_bytes();
    while (cs >= step && tiled_smem_bytes(nbits, win_words, cs, variant) > cap) cs -= step;
    return cs >= step ? cs : 0;
}

void launch_quad_direct(const QuadDirectArgs& a, cudaStream_t s)
{
    if (a.q_pitch_words % 4 != 0 || a.period_words % 4 != 0 || a.period_words <= 0)
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "quad-strided rows need a period of 4k words");
    if (a.nchans == 0 || a.q_pitch_words == 0) return;
    const size_t row_words = a.nchans * (size_t)a.nbits / 32;
    const dim3 grid((unsigned)((a.q_pitch_words + QD_N - 1) / QD_N), (unsigned)((row_words + QD_WORDS - 1) / QD_WORDS));
    if ((a.q_pitch_words + QD_N - 1) / QD_N > 0x7FFFFFFFu || grid.y > 65535u)
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "quad-strided rows too long for one launch");
    const int aligned = ((uintptr_t)a.in % 4 == 0) && (a.in_pitch % 4 == 0);
    switch (a.nbits) {
    case 1: quad_direct_kernel<1><<<grid, QD_THREADS, 0, s>>>(a, aligned); break;
    case 2: quad_direct_kernel<2><<<grid, QD_THREADS, 0, s>>>(a, aligned); break;
    case 4: quad_direct_kernel<4><<<grid, QD_THREADS, 0, s>>>(a, aligned); break;
    case 8: quad_direct_kernel<8><<<grid, QD_THREADS, 0, s>>>(a, aligned); break;
    default: DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "quad-strided rows hold samples of at most 8 bits");
    }
    RT_CHECK(cudaGetLastError());
}

void launch_transpose(const TransposeArgs& a, cudaStream_t s)
{
    switch (a.nbits) {
    case 1: launch_transpose_n<1>(a, s); break;
    case 2: launch_transpose_n<2>(a, s); break;
    case 4: launch_transpose_n<4>(a, s); break;
    case 8: launch_transpose_n<8>(a, s); break;
    case 16: launch_transpose_n<16>(a, s); break;
    case 32: launch_transpose_n<32>(a, s); break;
    default: DD_THROW(DEDISP_UNSUPPORTED_IN_NBITS);
    }
}

void launch_dedisperse_plain(const DedisperseArgs& a, cudaStream_t s)
{
    switch (a.nbits) {
    case 1: launch_plain_n<1>(a, s); break;
    case 2: launch_plain_n<2>(a, s); break;
    case 4: launch_plain_n<4>(a, s); break;
    case 8: launch_plain_n<8>(a, s); break;
    case 16: launch_plain_n<16>(a, s); break;
    case 32: launch_plain_n<32>(a, s); break;
    default: DD_THROW(DEDISP_UNSUPPORTED_IN_NBITS);
    }
}

void launch_dedisperse_tiled_batch(const BatchLaunch& b, int nbits, int variant, cudaStream_t s)
{
    if (b.total_items == 0) return;
    static_assert(T8_NSHAPES == 5 && Q8_NSHAPES == 4, "dispatch below lists every shape");
    switch (quad_shape(nbits, variant)) {
    case 0: launch_quad8_batch_variant<0>(b, s); return;
    case 1: launch_quad8_batch_variant<1>(b, s); return;
    case 2: launch_quad8_batch_variant<2>(b, s); return;
    case 3: launch_quad8_batch_variant<3>(b, s); return;
    default: break;
    }
    if (nbits != 8) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "no persistent kernel for this width and variant");
    switch (variant) {
    case 0: launch_tiled8_batch_variant<0>(b, s); break;
    case 1: launch_tiled8_batch_variant<1>(b, s); break;
    case 2: launch_tiled8_batch_variant<2>(b, s); break;
    case 3: launch_tiled8_batch_variant<3>(b, s); break;
    case 4: launch_tiled8_batch_variant<4>(b, s); break;
    default: DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "unknown tiled kernel variant");
    }
}

void launch_dedisperse_tiled(const DedisperseArgs& a, cudaStream_t s)
{
    // quad-strided rows hold bytes whatever the input width
    const int qs = quad_shape(a.nbits, a.variant);
    if (qs >= 0 && a.err == nullptr)
        DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "quad-strided launch without an error word");
    switch (qs) {
    case 0: launch_quad8_variant<0>(a, s); return;
    case 1: launch_quad8_variant<1>(a, s); return;
    case 2: launch_quad8_variant<2>(a, s); return;
    case 3: launch_quad8_variant<3>(a, s); return;
    default: break;
    }
    switch (a.nbits) {
    case 1: launch_tiled_n<1>(a, s); break;
    case 2: launch_tiled_n<2>(a, s); break;
    case 4: launch_tiled_n<4>(a, s); break;
    case 8: launch_tiled_n<8>(a, s); break;
    case 16: launch_tiled_n<16>(a, s); break;
    case 32: launch_tiled_n<32>(a, s); break;
    default: DD_THROW(DEDISP_UNSUPPORTED_IN_NBITS);
    }
}

}  // namespace kern
}  // namespace dedisp
