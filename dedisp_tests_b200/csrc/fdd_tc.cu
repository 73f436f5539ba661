// FDD phasor multiply-accumulate on the 5th-generation tensor cores
// (tcgen05, sm_100a) as a 3xBF16 complex GEMM per frequency bin.
//
// For bin k, with C real and the complex product written out,
//   Yr[dm][s] = sum_c  Pr(dm,c) Xr(c,s) - Pi(dm,c) Xi(c,s)
//   Yi[dm][s] = sum_c  Pr(dm,c) Xi(c,s) + Pi(dm,c) Xr(c,s)
// is the real GEMM  D[m][n] = sum_kk A[m][kk] B[kk][n]  with
//   A[m][2c] = Pr, A[m][2c+1] = Pi                        (M = DMs, K = 2*nact)
//   B[2c][n] = Xr(c,n), B[2c+1][n] = -Xi(c,n)             (n <  nseg)
//   B[2c][n] = Xi(c,s), B[2c+1][n] =  Xr(c,s), s = n-nseg (n >= nseg)
// and each operand is split into BF16 hi + lo parts:
//   D = Ah Bh + Ah Bl + Al Bh   (FP32 accumulation in tensor memory).
//
// Roles (one CTA per SM, 128 DMs per CTA, a range of bins per CTA):
//   warps 0-15  phasor producers: each thread owns one DM row (its TMEM
//               lane) and a quarter of every 64-channel chunk; phasors come from
//               the exact integer phase index (k*d) mod nfft and a quarter-
//               wave table of pre-split BF16 (cos, sin) pairs, and are stored
//               into tensor memory as the A operand; the same warps read the
//               accumulator of each finished bin and write Yt[k][s][dm].
//   warp 16     TMA producer for the B chunks (pre-split BF16, 128B swizzle).
//   warp 17     TMEM allocation and the single-thread MMA issuer.
// Every wait on an mbarrier is bounded; on expiry the kernel records an
// error code and winds down without waiting further.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <memory>
#include <type_traits>
#include <vector>

#include "fdd_tc.hpp"
#include "runtime.hpp"

namespace dedisp {
namespace kern {
namespace {

constexpr int TC_M = 128;              // DMs per CTA (accumulator lanes)
constexpr int TC_CHUNK = 64;           // channel padding (a multiple of both forms' A chunks)
constexpr int TC_MAX_STAGES = 6;       // B pipeline depth: as many as shared memory allows, 2..6
constexpr int TC_PRODUCER_WARPS = 16;  // 4 per TMEM lane quadrant
constexpr int TC_PARTS = TC_PRODUCER_WARPS / 4;  // producers sharing one DM row
constexpr int TC_THREADS = (TC_PRODUCER_WARPS + 2) * 32;
// Bounded mbarrier waits: give up after a.wait_ns of global time (checked
// every 16 polls) or TC_WAIT_POLLS polls, whichever comes first.
constexpr uint32_t TC_WAIT_POLLS = 1u << 28;
// Dynamic shared memory requested per CTA is at least this much so that only
// one CTA fits on an SM (each CTA allocates all 512 tensor-memory columns).
constexpr size_t TC_MIN_SMEM = 120 * 1024;
constexpr size_t TC_MAX_SMEM = kTcMaxSmem;

// Two MMA forms. Per K step of 16 reals:
//   plain (any npad <= 128): Ah Bh, Ah Bl, Al Bh as three N = npad MMAs into
//     one accumulator; 64-channel A chunks, 2 A buffers (hi 64 + lo 64
//     columns each), accumulators of 128 columns at 256 and 384;
//   fused (npad <= 80): Ah [Bh | Bl] as one N = 2 npad MMA (B hi and lo atoms
//     adjacent in shared memory), then Al Bh (N = npad) into its first npad
//     columns; the epilogue adds the two halves. Accumulators of 160 columns at
//     0 and 160, 32-channel A chunks in 3 buffers of 64 columns at 320, 384, 448.
//   deep (npad <= 64): the three-MMA form with 3 A buffers (0, 128, 256) and
//     accumulators of 64 columns at 384 and 448: half again as many phasors
//     in flight, which is what bounds the MAC when it waits on MMA
//     completions rather than on the tensor pipe.
//   fused wide (FUSED and DEEP, npad <= 32; the default there): the fused form at 64-channel
//     chunks, 3 A buffers (0, 128, 256) and accumulators of 2 npad <= 64
//     columns at 384 and 448: 16 MMAs per chunk instead of 24 (one thread
//     issues an MMA about every 30 ns whatever its N, so narrow MMAs are
//     bound by their count).
template <bool FUSED, bool DEEP = false>
struct TcForm {
    static constexpr bool NARROW = FUSED && !DEEP;        // fused at 32-channel chunks
    static constexpr int CH = NARROW ? 32 : 64;           // channels per A chunk
    static constexpr int PART_CH = CH / TC_PARTS;         // per producer thread
    static constexpr int NBUF = (FUSED || DEEP) ? 3 : 2;  // A buffers
    static constexpr uint32_t A_COLS = 2 * CH;            // hi CH + lo CH columns
    static constexpr uint32_t A_BASE = NARROW ? 320 : 0;
    static constexpr uint32_t C0 = NARROW ? 0 : DEEP ? 384 : 256, C1 = NARROW ? 160 : DEEP ? 448 : 384;
    static constexpr int KSTEPS = CH / 8;                 // K16 steps per chunk
    static constexpr int ATOMS = CH / 32;                 // 64-kk TMA atoms per split
};
constexpr int TC_FUSED_MAX_NPAD = 80;
constexpr int TC_DEEP_MAX_NPAD = 64;
constexpr int TC_MAX_ABUF = 3;

struct alignas(8) SmemBarriers {
    uint64_t b_full[TC_MAX_STAGES];
    uint64_t b_empty[TC_MAX_STAGES];
    uint64_t a_full[TC_MAX_ABUF];
    uint64_t a_empty[TC_MAX_ABUF];
    uint64_t c_full[2];
    uint64_t c_empty[2];
    uint64_t drain;
    uint64_t never;       // expiry test: nothing arrives on it
    uint64_t item_full[2];   // item index published (TMA thread)
    uint64_t item_empty[2];  // item index read (producer warps + MMA thread)
    int item[2];             // two-slot ring of this CTA's next item indices (-1: none left)
    uint32_t tmem_base;
    uint32_t abort_flag;  // a producer gave up a bounded wait (delay-table mode)
};
static_assert(sizeof(SmemBarriers) <= 256, "barriers precede the phasor table at +256 bytes");

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t* b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for phase `parity` of barrier b; false if the limit expired.
// CLUSTER: acquire at cluster scope (arrivals and stores from the other CTA
// of a pair).
template <bool CLUSTER = false>
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, uint64_t limit_ns)
{
    const uint32_t addr = smem_u32(b);
    uint64_t t0 = 0;
    for (uint32_t i = 0; i < TC_WAIT_POLLS; ++i) {
        uint32_t done;
        if constexpr (CLUSTER)
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(done)
                : "r"(addr), "r"(parity)
                : "memory");
        else
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(done)
                : "r"(addr), "r"(parity)
                : "memory");
        if (done) return true;
        if ((i & 15u) == 15u) {
            const uint64_t t = global_ns();
            if (t0 == 0) t0 = t;
            else if (t - t0 > limit_ns) return false;
        }
    }
    return false;
}

// The same wait for a whole warp, with one outcome for all its lanes (the
// tensor-memory loads and stores that follow are warp-collective).
template <bool CLUSTER = false>
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* b, uint32_t parity, uint64_t limit_ns)
{
    const bool done = mbar_wait<CLUSTER>(b, parity, limit_ns);
    return __all_sync(0xFFFFFFFFu, done);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// L2 policy for the B chunks: kept in L2 in preference to streaming data (a
// bin's chunks are read again by each of its DM tiles).
__device__ __forceinline__ uint64_t l2_evict_last_policy()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ void tma_load_4d(void* smem, const CUtensorMap* map, uint64_t* bar,
                                            int c0, int c1, int c2, int c3, uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%3, %4, %5, %6}], [%2], %7;" ::"r"(smem_u32(smem)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
        "l"(policy)
        : "memory");
}

__device__ __forceinline__ void mma_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t desc_b,
                                       uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(tmem_d),
        "r"(tmem_a), "l"(desc_b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// --- CTA pairs (cluster of 2, tcgen05 cta_group::2) -------------------------
__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// Shared::cluster address of this CTA's variable p in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank)
{
    uint32_t a;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
    return a;
}

__device__ __forceinline__ void mbar_arrive_cluster(uint32_t addr)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(addr) : "memory");
}

__device__ __forceinline__ void st_cluster_s32(uint32_t addr, int v)
{
    asm volatile("st.shared::cluster.s32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// M = 256 MMA over the pair (issued by the leader CTA): A rows 0-127 from
// the leader's tensor memory, 128-255 from the peer's (same address); B
// columns 0..N/2-1 from the leader's shared memory, the rest from the peer's
// (same offset); each CTA's accumulator holds its 128 rows x N.
__device__ __forceinline__ void mma_ts_pair(uint32_t tmem_d, uint32_t tmem_a, uint64_t desc_b, uint32_t idesc,
                                            uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(tmem_d),
        "r"(tmem_a), "l"(desc_b), "r"(idesc), "r"(accumulate));
}

// Completion of the pair's MMAs issued so far, signalled on the barrier at
// shared::cluster address `bar` (this CTA's or the peer's).
__device__ __forceinline__ void mma_commit_pair_to(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// ... on barrier `b` of the leader (mask 1) or of both CTAs (mask 3), one
// commit per CTA.
__device__ __forceinline__ void mma_commit_pair(uint64_t* b, int mask)
{
    mma_commit_pair_to(cluster_addr(b, 0));
    if (mask & 2) mma_commit_pair_to(cluster_addr(b, 1));
}

// Tile load into this CTA's shared memory whose completion counts on the
// barrier at shared::cluster address `bar` (the leader's).
__device__ __forceinline__ void tma_load_4d_pair(void* smem, const CUtensorMap* map, uint32_t bar, int c0, int c1,
                                                 int c2, int c3, uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%3, %4, %5, %6}], [%2], %7;" ::"r"(smem_u32(smem)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "l"(policy)
        : "memory");
}

// 32 consecutive 32-bit columns of this thread's lane.
// 16 consecutive 32-bit columns of this thread's lane.
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&v)[8])
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]));
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&v)[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]),
        "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]),
        "r"(v[15]));
}

__device__ __forceinline__ float tmem_ld1(uint32_t taddr)
{
    uint32_t r;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
    return __uint_as_float(r);
}

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), LBO unused (1), descriptor version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ int tc_delay(float dm, float delay, int round_delays)
{
    const float x = __fmul_rn(dm, delay);
    return round_delays ? (int)__float2uint_rn(x) : __float2int_rz(x);
}

// (re, im) -> packed bf16x2 hi parts (re low half) and lo parts
// (bf16(x - hi)).
__device__ __forceinline__ uint2 split_bf16x2(float re, float im);

// The phasor exp(+2 pi i (k d mod N) / N), split into bf16 hi/lo pairs, from
// the two-level twiddle tables in shared memory (the product the per-bin
// delay table holds). pow2: N a power of two (index by mask), else by
// Barrett reduction with nmagic = floor((2^64 - 1) / N).
__device__ __forceinline__ uint2 phasor_direct(size_t k, int d, uint32_t nfft, bool pow2, uint64_t nmagic,
                                               const float2* s_tw_lo, const float2* s_tw_hi)
{
    uint32_t idx;
    if (pow2) {
        idx = ((uint32_t)k * (uint32_t)d) & (nfft - 1u);
    } else {
        const uint32_t dn = d >= 0 ? (uint32_t)d % nfft : nfft - 1u - (uint32_t)(-(d + 1)) % nfft;
        const uint64_t p = (uint64_t)k * dn;
        uint64_t r = p - __umul64hi(p, nmagic) * (uint64_t)nfft;
        while (r >= nfft) r -= nfft;
        idx = (uint32_t)r;
    }
    const float2 h = s_tw_hi[idx >> 8], l = s_tw_lo[idx & 255u];
    const float c = __fsub_rn(__fmul_rn(h.x, l.x), __fmul_rn(h.y, l.y));
    const float sn = -__fadd_rn(__fmul_rn(h.x, l.y), __fmul_rn(h.y, l.x));
    return split_bf16x2(c, sn);
}
__device__ __forceinline__ uint2 split_bf16x2(float re, float im)
{
    const __nv_bfloat162 hi = __floats2bfloat162_rn(re, im);
    const float2 hf = __bfloat1622float2(hi);
    const __nv_bfloat162 lo = __floats2bfloat162_rn(__fsub_rn(re, hf.x), __fsub_rn(im, hf.y));
    return make_uint2(*reinterpret_cast<const uint32_t*>(&hi), *reinterpret_cast<const uint32_t*>(&lo));
}

// The MAC over a work list: item i = bins [k_begin, k_end) of DM tile `tile`
// of descriptor `desc` (its own DM list, length, B operand and tensor map,
// output and segment group); CTA b takes items b, b + G, b + 2G, ... The
// pipeline counters run on across items, so the hand-offs of consecutive
// items overlap; each item's last accumulator is read out before the next
// item starts. One plan's launch is the one-descriptor case.
// PAIR: clusters of two CTAs (cta_group::2): DM tiles of 256 rows, the
// leader's MMA thread issues M = 256 MMAs over both CTAs' tensor memory, each
// CTA loads half of every B chunk and produces the phasors of its 128 DMs;
// the leader claims the pair's items and publishes them to both CTAs.
template <bool FUSED, bool DEEP, bool PAIR>
__global__ void __launch_bounds__(TC_THREADS, 1) fdd_mac_tc_kernel(const __grid_constant__ TcParams P)
{
    using F = TcForm<FUSED, DEEP>;
    // descriptors and tensor maps live in the parameter bank (constant
    // operands, no registers); the items in global memory
    const TcMacArgs* descs = P.descs;
    const CUtensorMap* maps = P.maps;
    const TcWork* items = P.items;
    const int nitems = P.nitems;
    const TcLayout& L = P.layout;
    extern __shared__ __align__(1024) uint8_t smem_dyn[];
    // layout (from a 1024-byte aligned base, as the 128-byte swizzle needs):
    // [B stages][barriers][phasor table][twiddles lo, hi][delays][sym]; the
    // phasor table is the quarter-wave table (nfft/4 + 1 entries) or, in
    // delay-table mode (dmax >= 0), the phasors of the current bin for every
    // delay 0..dmax; each region is sized for the largest descriptor
    uint8_t* smem_raw = smem_dyn + ((1024u - (smem_u32(smem_dyn) & 1023u)) & 1023u);
    uint8_t* s_b = smem_raw;
    const int nst = L.stages;
    SmemBarriers* bars = reinterpret_cast<SmemBarriers*>(smem_raw + nst * L.stage_bytes);
    uint2* s_table = reinterpret_cast<uint2*>(reinterpret_cast<uint8_t*>(bars) + 256);
    float2* s_tw_lo = reinterpret_cast<float2*>(s_table + L.table_entries);
    float2* s_tw_hi = s_tw_lo + 256;
    float* s_delay = reinterpret_cast<float*>(s_tw_hi + L.tw_hi_entries);
    uint2* s_sym = reinterpret_cast<uint2*>(s_delay + L.nact_pad);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t crank = PAIR ? cluster_rank() : 0u;  // 0: the pair's leader
    const bool leader = crank == 0u;
    const int units = PAIR ? (int)(gridDim.x >> 1) : (int)gridDim.x;  // CTAs or pairs
    const int unit = PAIR ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
    if (unit >= nitems) return;  // whole CTA (pair) leaves before touching barriers
    const int nchunks = L.nact_pad / F::CH;
    constexpr int TILE_M = PAIR ? 2 * TC_M : TC_M;  // DMs per tile
    const int row_off = (int)crank * TC_M;         // this CTA's rows within a tile
    // arrival on the leader's barrier (this CTA's own without pairs)
    auto arrive_leader = [&](uint64_t* b) {
        if constexpr (PAIR) mbar_arrive_cluster(cluster_addr(b, 0));
        else mbar_arrive(b);
    };

    // --- set-up -------------------------------------------------------------
    for (int i = tid; i < L.nact_pad; i += blockDim.x) s_delay[i] = descs[0].delay_act[i];
    if (tid < 4) {
        // quadrant q of exp(+i theta): (re, im) = R^q (c, s); in packed
        // bf16x2 (re low half, im high half): selector swaps halves,
        // mask flips sign bits.
        const uint32_t sel[4] = {0x3210u, 0x1032u, 0x3210u, 0x1032u};
        const uint32_t neg[4] = {0u, 0x00008000u, 0x80008000u, 0x80000000u};
        s_sym[tid] = make_uint2(sel[tid], neg[tid]);
    }
    if (tid == 0) {
        for (int i = 0; i < nst; ++i) {
            mbar_init(&bars->b_full[i], 1);
            mbar_init(&bars->b_empty[i], 1);
        }
        // one arrive per producer warp (of both CTAs of a pair, on the leader's)
        constexpr uint32_t nprod = TC_PRODUCER_WARPS * (PAIR ? 2 : 1);
        for (int i = 0; i < F::NBUF; ++i) {
            mbar_init(&bars->a_full[i], nprod);
            mbar_init(&bars->a_empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&bars->c_full[i], 1);
            mbar_init(&bars->c_empty[i], nprod);
        }
        mbar_init(&bars->drain, 1);
        mbar_init(&bars->never, 1);
        for (int i = 0; i < 2; ++i) {
            mbar_init(&bars->item_full[i], 1);
            // readers of an item index: the producer warps and the MMA thread
            // (pairs: also the peer's producer warps and TMA thread)
            mbar_init(&bars->item_empty[i], PAIR ? 2 * (TC_PRODUCER_WARPS + 1) : TC_PRODUCER_WARPS + 1);
        }
        bars->abort_flag = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == TC_PRODUCER_WARPS + 1) {
        if constexpr (PAIR) {
            // the same warp of both CTAs, the same destination offset
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
                             smem_u32(&bars->tmem_base)));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::);
        } else {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
                             smem_u32(&bars->tmem_base)));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
        }
    }
    tc_fence_before();
    __syncthreads();
    // pairs: both CTAs' barriers are initialised before any remote arrival
    if constexpr (PAIR) cluster_sync_all();
    tc_fence_after();
    const uint32_t tmem = bars->tmem_base;
    bool ok = true;
    const uint64_t t_start = (P.cta_ns && tid == 0) ? global_ns() : 0;

    if (warp < TC_PRODUCER_WARPS) {
        // --- phasor producers + epilogue ------------------------------------
        // Order per bin k: (delay-table mode: rebuild the table for k), store
        // the A chunks of k, then read out the accumulator of bin k-1 while
        // the tensor cores work on k. Every producer warp passes the same
        // named barriers (bar 1) in the same order, on failure too: a warp
        // that gives up sets abort_flag and goes on to the next barrier,
        // where all of them see the flag and stop together.
        const int quad = warp & 3, part = warp >> 2;
        const uint32_t lane_addr = (uint32_t)(quad * 32) << 16;
        const int ptid = warp * 32 + lane;                      // 0..511
        volatile uint32_t* abort_flag = &bars->abort_flag;
        uint32_t g = 0;    // chunk counter (A buffers)
        int bin_iter = 0;  // bin counter (accumulators)
        int cur_desc = -1; // descriptor whose tables are in shared memory
        for (uint32_t j = 0;; ++j) {
            // item j of this CTA, as the TMA thread published it; one outcome
            // for all producers (the named barrier's OR of "gave up the wait
            // or an abort was raised"), which also orders the table reloads
            // below after every producer's reads of the previous item
            const uint32_t slot = j & 1u;
            const bool got = mbar_wait<PAIR>(&bars->item_full[slot], (j >> 1) & 1u, L.wait_ns);
            const int it = got ? *reinterpret_cast<volatile int*>(&bars->item[slot]) : -1;
            const uint32_t bad = (!got || *abort_flag) ? 1u : 0u;
            uint32_t fail;
            asm volatile(
                "{\n\t.reg .pred p, q;\n\t"
                "setp.ne.u32 p, %1, 0;\n\t"
                "bar.red.or.pred q, 1, %2, p;\n\t"
                "selp.u32 %0, 1, 0, q;\n\t}"
                : "=r"(fail)
                : "r"(bad), "n"(TC_PRODUCER_WARPS * 32)
                : "memory");
            if (fail) { ok = false; break; }
            __syncwarp();
            if (lane == 0) arrive_leader(&bars->item_empty[slot]);
            if (it < 0) break;
            const TcWork w = items[it];
            const TcMacArgs& a = descs[w.desc];  // read-only descriptor (L1)
            const uint32_t nfft = a.nfft, qn = nfft / 4;
            const bool ptab = a.dmax >= 0;
            const bool direct = !ptab && a.direct;
            const bool twl = ptab || direct;
            if (w.desc != cur_desc) {
                // this descriptor's tables (all producers are past the last
                // item's reads: barrier above)
                if (!twl) {
                    for (uint32_t i = ptid; i <= qn; i += TC_PRODUCER_WARPS * 32) s_table[i] = a.table[i];
                } else {
                    for (uint32_t i = ptid; i < 256; i += TC_PRODUCER_WARPS * 32) s_tw_lo[i] = a.tw_lo[i];
                    for (uint32_t i = ptid; i < nfft / 256; i += TC_PRODUCER_WARPS * 32) s_tw_hi[i] = a.tw_hi[i];
                }
                cur_desc = w.desc;
            }
            asm volatile("bar.sync 1, %0;" ::"n"(TC_PRODUCER_WARPS * 32) : "memory");
            const int row = quad * 32 + lane;  // this thread's DM row within a tile
            const int first_iter = bin_iter;
            const int last_tile = w.tile + w.ntile - 1;

            auto epilogue = [&](int itr, size_t kk, int m) -> bool {
                const uint32_t cb = (uint32_t)itr & 1u;
                if (!mbar_wait_warp<PAIR>(&bars->c_full[cb], ((uint32_t)itr >> 1) & 1u, L.wait_ns)) return false;
                tc_fence_after();
                const uint32_t ccol = cb ? F::C1 : F::C0;
                const uint32_t half = FUSED ? (uint32_t)a.npad : 0u;  // fused: Ah Bl columns
                const int sh = (a.nseg + TC_PARTS - 1) / TC_PARTS;
                const int s0 = min(a.nseg, part * sh), s1 = min(a.nseg, s0 + sh);
                // the row's output element offsets: Y (DM-major) or Yt (bin-major)
                float2* const yrow = a.Y ? a.Y + ((size_t)m * a.nseg_total + a.seg0) * a.y_pitch + kk
                                         : a.Yt + (kk * a.nseg_total + a.seg0) * a.ndm + m;
                const size_t ystep = a.Y ? a.y_pitch : (size_t)a.ndm;
                const bool mine = m < a.ndm;
                for (int sb = s0; sb < s1; sb += 4) {
                    const int cnt = min(4, s1 - sb);  // the same for the whole warp
                    float yr[4], yi[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        if (i < cnt) {
                            yr[i] = tmem_ld1(tmem + lane_addr + ccol + sb + i);
                            yi[i] = tmem_ld1(tmem + lane_addr + ccol + a.nseg + sb + i);
                        }
                    }
                    float zr[4], zi[4];
                    if constexpr (FUSED) {
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            if (i < cnt) {
                                zr[i] = tmem_ld1(tmem + lane_addr + ccol + half + sb + i);
                                zi[i] = tmem_ld1(tmem + lane_addr + ccol + half + a.nseg + sb + i);
                            }
                        }
                    }
                    tmem_wait_ld();
                    if constexpr (FUSED) {
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            yr[i] += zr[i];
                            yi[i] += zi[i];
                        }
                    }
                    if (mine) {
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            if (i < cnt) __stcs(yrow + (size_t)(sb + i) * ystep, make_float2(yr[i], yi[i]));
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) arrive_leader(&bars->c_empty[cb]);
                return true;
            };

            const uint32_t nmask = nfft - 1u, qshift = (uint32_t)(31 - __clz((int)max(qn, 1u)));
            const bool pow2n = (nfft & nmask) == 0u;
            bool aborted = false;
            // k == k_end: only the read-out of the item's last bin (one call
            // site of the epilogue keeps it inlined once)
            // Per bin: (delay-table mode) the table, then every DM tile of the
            // item, each one (bin, tile) pair with its own accumulator: the
            // table is built once per bin for all tiles.
            for (size_t k = w.k_begin; k <= w.k_end; ++k) {
                const bool tail = k == w.k_end;
                if (tail) {
                    if (ok && bin_iter > first_iter) ok = epilogue(bin_iter - 1, k - 1, last_tile * TILE_M + row_off + row);
                    if (!ok) *abort_flag = 1u;
                    break;
                }
                if (ptab) {
                    // All producers are done with the previous bin's table, and
                    // every abort raised before this point is visible to all.
                    asm volatile("bar.sync 1, %0;" ::"n"(TC_PRODUCER_WARPS * 32) : "memory");
                    if (*abort_flag) { aborted = true; break; }
                    // idx = (k d) mod N for d = ptid, ptid + S, ... (S = 512 threads),
                    // stepped by (k S) mod N: exact for any N (N < 2^31)
                    constexpr uint32_t S = TC_PRODUCER_WARPS * 32;
                    uint32_t idx = (uint32_t)(((uint64_t)k * (uint64_t)ptid) % nfft);
                    const uint32_t step = (uint32_t)(((uint64_t)k * S) % nfft);
                    for (int d = ptid; d <= a.dmax; d += S, idx = (idx + step >= nfft) ? idx + step - nfft : idx + step) {
                        // exp(+2 pi i idx / N) = conj(tw_hi[idx >> 8] * tw_lo[idx & 255])
                        const float2 h = s_tw_hi[idx >> 8], l = s_tw_lo[idx & 255u];
                        const float c = __fsub_rn(__fmul_rn(h.x, l.x), __fmul_rn(h.y, l.y));
                        const float sn = -__fadd_rn(__fmul_rn(h.x, l.y), __fmul_rn(h.y, l.x));
                        s_table[d] = split_bf16x2(c, sn);
                    }
                    asm volatile("bar.sync 1, %0;" ::"n"(TC_PRODUCER_WARPS * 32) : "memory");
                } else if (!ok) {
                    break;
                }
                for (int t = w.tile; t < w.tile + w.ntile; ++t) {
                if (ok) {
                    const int m = t * TILE_M + row_off + row;
                    const float dm = a.dms[min(m, a.ndm - 1)];
                    for (int ch = 0; ch < nchunks; ++ch, ++g) {
                        const uint32_t buf = g % F::NBUF, use = g / F::NBUF;
                        // the phasors first: their gathers overlap the MMAs still
                        // reading this A buffer
                        constexpr int TC_PART_CH = F::PART_CH;
                        uint32_t hi[TC_PART_CH], lo[TC_PART_CH];
                        const int c0 = ch * F::CH + part * TC_PART_CH;
                        if (ptab) {
                            // delays of the 16 channels (4 vector loads); the table
                            // covers 0..dmax, the largest delay over the plan's DMs and
                            // channels computed on the host with the same float
                            // operations, so the unsigned clamp is only a guard
                            const float4* sd4 = reinterpret_cast<const float4*>(s_delay + c0);
                            const uint32_t dmax = (uint32_t)a.dmax;
                            const bool rn = a.round_delays != 0;
                            if (!a.hybrid) {
#pragma unroll
                                for (int q = 0; q < TC_PART_CH / 4; ++q) {
                                    const float4 v4 = sd4[q];
                                    const float dl[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
                                    for (int i = 0; i < 4; ++i) {
                                        const float x = __fmul_rn(dm, dl[i]);
                                        const float y = rn ? __fadd_rn(x, 8388608.0f) : __fadd_rz(x, 8388608.0f);
                                        const uint2 v = s_table[min(__float_as_uint(y) - 0x4B000000u, dmax)];
                                        hi[4 * q + i] = v.x;
                                        lo[4 * q + i] = v.y;
                                    }
                                }
                            } else {
                                // the table covers delays 0..dmax; larger ones are
                                // computed from the twiddle tables
#pragma unroll
                                for (int q = 0; q < TC_PART_CH / 4; ++q) {
                                    const float4 v4 = sd4[q];
                                    const float dl[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
                                    for (int i = 0; i < 4; ++i) {
                                        const float x = __fmul_rn(dm, dl[i]);
                                        const float y = rn ? __fadd_rn(x, 8388608.0f) : __fadd_rz(x, 8388608.0f);
                                        const uint32_t d = __float_as_uint(y) - 0x4B000000u;
                                        const uint2 v = d <= dmax ? s_table[d]
                                                                  : phasor_direct(k, (int)d, nfft, pow2n, a.nmagic,
                                                                                  s_tw_lo, s_tw_hi);
                                        hi[4 * q + i] = v.x;
                                        lo[4 * q + i] = v.y;
                                    }
                                }
                            }
                        } else if (direct) {
#pragma unroll
                            for (int i = 0; i < TC_PART_CH; ++i) {
                                const int d = tc_delay(dm, s_delay[c0 + i], a.round_delays);
                                const uint2 v = phasor_direct(k, d, nfft, pow2n, a.nmagic, s_tw_lo, s_tw_hi);
                                hi[i] = v.x;
                                lo[i] = v.y;
                            }
                        } else {
#pragma unroll
                            for (int i = 0; i < TC_PART_CH; ++i) {
                                const int d = tc_delay(dm, s_delay[c0 + i], a.round_delays);
                                const uint32_t idx = ((uint32_t)k * (uint32_t)d) & nmask;
                                const uint32_t q = idx >> qshift, r = idx & (qn - 1u);
                                const uint2 t = s_table[r];
                                const uint2 sy = s_sym[q];
                                hi[i] = __byte_perm(t.x, 0u, sy.x) ^ sy.y;
                                lo[i] = __byte_perm(t.y, 0u, sy.x) ^ sy.y;
                            }
                        }
                        if (!mbar_wait_warp<PAIR>(&bars->a_empty[buf], (use & 1u) ^ 1u, L.wait_ns)) { ok = false; break; }
                        tc_fence_after();
                        const uint32_t acol = F::A_BASE + buf * F::A_COLS;
                        if constexpr (TC_PART_CH == 8) {
                            tmem_st8(tmem + lane_addr + acol + part * TC_PART_CH, hi);
                            tmem_st8(tmem + lane_addr + acol + F::CH + part * TC_PART_CH, lo);
                        } else {
                            tmem_st16(tmem + lane_addr + acol + part * TC_PART_CH, hi);
                            tmem_st16(tmem + lane_addr + acol + F::CH + part * TC_PART_CH, lo);
                        }
                        tmem_wait_st();
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) arrive_leader(&bars->a_full[buf]);
                    }
                }
                // the previous pair's read-out overlaps this pair's MMAs
                if (ok && bin_iter > first_iter)
                    ok = epilogue(bin_iter - 1, t > w.tile ? k : k - 1,
                                  (t > w.tile ? t - 1 : last_tile) * TILE_M + row_off + row);
                if (!ok) *abort_flag = 1u;  // the others stop at the next barrier
                ++bin_iter;
                }
            }
            if (aborted) ok = false;
            if (!ok) *abort_flag = 1u;
        }
    } else if (warp == TC_PRODUCER_WARPS) {
        // --- TMA producer ------------------------------------------------------
        if (lane == 0) {
            uint32_t g = 0;
            uint32_t st = 0, st_phase = 0;  // B stage of chunk g (g % nst) and its use parity
            const uint64_t b_policy = l2_evict_last_policy();
            // this CTA's items: blockIdx.x first, then the next unclaimed item
            // of the list (longest first) each time one is done, published to
            // the other roles through the two-slot ring
            for (uint32_t j = 0; ok; ++j) {
                const uint32_t slot = j & 1u;
                int it;
                if (!PAIR || leader) {
                    it = j == 0 ? unit : units + (int)atomicAdd(P.next_item, 1u);
                    if (it >= nitems) it = -1;
                    if (!mbar_wait<PAIR>(&bars->item_empty[slot], ((j >> 1) & 1u) ^ 1u, L.wait_ns)) { ok = false; break; }
                    bars->item[slot] = it;
                    mbar_arrive(&bars->item_full[slot]);
                    if constexpr (PAIR) {
                        // the peer's copy of the slot; the release of the remote
                        // arrival orders the store before it
                        st_cluster_s32(cluster_addr(&bars->item[slot], 1), it);
                        mbar_arrive_cluster(cluster_addr(&bars->item_full[slot], 1));
                    }
                } else {
                    // the peer: the index its leader published
                    if (!mbar_wait<PAIR>(&bars->item_full[slot], (j >> 1) & 1u, L.wait_ns)) { ok = false; break; }
                    it = *reinterpret_cast<volatile int*>(&bars->item[slot]);
                    mbar_arrive_cluster(cluster_addr(&bars->item_empty[slot], 0));
                }
                if (it < 0) break;
                const TcWork w = items[it];
                const CUtensorMap* bmap = maps + w.desc;
                // B rows this CTA loads (pairs: its half of the MMA's N) and
                // one 64-kk atom of one split of them
                const uint32_t rows = (uint32_t)descs[w.desc].npad / (PAIR ? 2u : 1u);
                const uint32_t atom_bytes = rows * 128u;
                const int n0 = (int)(crank * rows);
                for (size_t kt = (size_t)w.k_begin * w.ntile; kt < (size_t)w.k_end * w.ntile && ok; ++kt) {
                    const size_t k = kt / (size_t)w.ntile;  // every tile of bin k reads bin k's B
                    for (int ch = 0; ch < nchunks; ++ch, ++g) {
                        if (!mbar_wait<PAIR>(&bars->b_empty[st], st_phase ^ 1u, L.wait_ns)) { ok = false; break; }
                        // the leader's barrier counts both halves of a pair's chunk
                        if (!PAIR || leader)
                            mbar_expect_tx(&bars->b_full[st], (PAIR ? 2u : 1u) * 2u * F::ATOMS * atom_bytes);
                        uint8_t* dst = s_b + st * L.stage_bytes;
                        // coordinates: (kk, n, split, bin); atoms in the order
                        // (atom, split), so each atom's hi and lo rows are adjacent
                        for (int at = 0; at < F::ATOMS; ++at)
                            for (int sp = 0; sp < 2; ++sp) {
                                if constexpr (PAIR)
                                    tma_load_4d_pair(dst + (at * 2 + sp) * atom_bytes, bmap,
                                                     cluster_addr(&bars->b_full[st], 0),
                                                     ch * (2 * F::CH) + at * 64, n0, sp, (int)k, b_policy);
                                else
                                    tma_load_4d(dst + (at * 2 + sp) * atom_bytes, bmap, &bars->b_full[st],
                                                ch * (2 * F::CH) + at * 64, 0, sp, (int)k, b_policy);
                            }
                        if (++st == (uint32_t)nst) {
                            st = 0;
                            st_phase ^= 1u;
                        }
                    }
                }
            }
            // do not leave while loads are in flight: wait for the last stages
            // (a pair's leader: both CTAs' loads count on its barriers; the
            // peer stays resident until the pair's closing cluster barrier)
            if (!PAIR || leader) {
                const uint32_t issued = g;
                for (uint32_t j = (issued > (uint32_t)nst ? issued - nst : 0); j < issued; ++j)
                    mbar_wait<PAIR>(&bars->b_full[j % nst], (j / nst) & 1u, L.wait_ns);
            }
        }
    } else {
        // --- MMA issuer (a pair's leader only) ----------------------------------
        if (lane == 0 && (!PAIR || leader)) {
            uint32_t g = 0;
            uint32_t st = 0, st_phase = 0;   // B stage of chunk g (g % nst) and its use parity
            uint32_t buf = 0, a_phase = 0;   // A buffer of chunk g (g % NBUF) and its use parity
            int bin_iter = 0;
            const uint64_t desc_s0 = sw128_desc(smem_u32(s_b));  // descriptor of stage 0's first atom
            for (uint32_t j = 0; ok; ++j) {
                const uint32_t slot = j & 1u;
                if (!mbar_wait<PAIR>(&bars->item_full[slot], (j >> 1) & 1u, L.wait_ns)) { ok = false; break; }
                const int it = *reinterpret_cast<volatile int*>(&bars->item[slot]);
                mbar_arrive(&bars->item_empty[slot]);
                if (it < 0) break;
                const TcWork w = items[it];
                const uint32_t npad = (uint32_t)descs[w.desc].npad;
                // one atom (this CTA's B rows x 128 bytes) in descriptor units
                const uint32_t atom16 = (npad / (PAIR ? 2u : 1u)) * 8u;
                const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((npad >> 3) << 17) |
                                       ((uint32_t)(TILE_M >> 4) << 24);
                const uint32_t idesc2 = (1u << 4) | (1u << 7) | (1u << 10) | (((2u * npad) >> 3) << 17) |
                                        ((uint32_t)(TILE_M >> 4) << 24);
                for (size_t kt = (size_t)w.k_begin * w.ntile; kt < (size_t)w.k_end * w.ntile && ok; ++kt, ++bin_iter) {
                    const uint32_t cb = (uint32_t)bin_iter & 1u;
                    if (!mbar_wait<PAIR>(&bars->c_empty[cb], (((uint32_t)bin_iter >> 1) & 1u) ^ 1u, L.wait_ns)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t dcol = tmem + (cb ? F::C1 : F::C0);
                    for (int ch = 0; ch < nchunks; ++ch, ++g) {
                        if (!mbar_wait<PAIR>(&bars->a_full[buf], a_phase, L.wait_ns)) { ok = false; break; }
                        if (!mbar_wait<PAIR>(&bars->b_full[st], st_phase, L.wait_ns)) { ok = false; break; }
                        // expiry test: one more wait, on a barrier nothing arrives on
                        if (L.wait_test && g == 0 && !mbar_wait<PAIR>(&bars->never, 0u, L.wait_ns)) { ok = false; break; }
                        tc_fence_after();
                        const uint32_t acol = tmem + F::A_BASE + buf * F::A_COLS;
                        // descriptors by adding offsets (16-byte units) to the low
                        // word: shared addresses stay below 2^18, so the 14-bit
                        // address field never carries
                        const uint64_t d0 = desc_s0 + (uint64_t)((st * L.stage_bytes) >> 4);
#pragma unroll
                        for (int s = 0; s < F::KSTEPS; ++s) {
                            const uint32_t at = (uint32_t)s >> 2, sub = (uint32_t)s & 3u;
                            const uint64_t bh = d0 + (uint64_t)(at * 2u * atom16 + sub * 2u);
                            const uint32_t ah = acol + s * 8, al = acol + F::CH + s * 8;
                            const uint32_t first = (s == 0 && ch == 0) ? 0u : 1u;
                            if constexpr (FUSED) {
                                // [Bh | Bl]: the lo atom follows the hi atom (2 npad rows)
                                mma_ts(dcol, ah, bh, idesc2, first);
                                mma_ts(dcol, al, bh, idesc, 1u);
                            } else if constexpr (PAIR) {
                                const uint64_t bl = bh + (uint64_t)atom16;
                                mma_ts_pair(dcol, ah, bh, idesc, first);
                                mma_ts_pair(dcol, ah, bl, idesc, 1u);
                                mma_ts_pair(dcol, al, bh, idesc, 1u);
                            } else {
                                const uint64_t bl = bh + (uint64_t)atom16;
                                mma_ts(dcol, ah, bh, idesc, first);
                                mma_ts(dcol, ah, bl, idesc, 1u);
                                mma_ts(dcol, al, bh, idesc, 1u);
                            }
                        }
                        if constexpr (PAIR) {
                            mma_commit_pair(&bars->a_empty[buf], 3);
                            mma_commit_pair(&bars->b_empty[st], 3);
                        } else {
                            mma_commit(&bars->a_empty[buf]);
                            mma_commit(&bars->b_empty[st]);
                        }
                        if (++buf == (uint32_t)F::NBUF) {
                            buf = 0;
                            a_phase ^= 1u;
                        }
                        if (++st == (uint32_t)nst) {
                            st = 0;
                            st_phase ^= 1u;
                        }
                    }
                    if (!ok) break;
                    if constexpr (PAIR) mma_commit_pair(&bars->c_full[cb], 3);
                    else mma_commit(&bars->c_full[cb]);
                }
            }
            // all issued MMAs complete before the accumulator memory goes away
            if constexpr (PAIR) mma_commit_pair(&bars->drain, 1);
            else mma_commit(&bars->drain);
            mbar_wait<PAIR>(&bars->drain, 0, L.wait_ns);
        }
    }
    if (!ok) atomicExch(L.err, 1u);

    tc_fence_before();
    __syncthreads();
    // pairs: neither CTA leaves (nor frees tensor memory) while the other may
    // still arrive on its barriers or the leader's MMAs read its memory
    if constexpr (PAIR) cluster_sync_all();
    tc_fence_after();
    if (P.cta_ns && tid == 0) P.cta_ns[blockIdx.x] = global_ns() - t_start;
    if (warp == TC_PRODUCER_WARPS + 1) {
        if constexpr (PAIR) asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, 512;" ::"r"(tmem));
        else asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
    }
}

__device__ __forceinline__ uint32_t bf16x2_bits(float lo_half, float hi_half)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo_half, hi_half);  // .x low, .y high
    return *reinterpret_cast<const uint32_t*>(&v);
}

// B operand from the spectra: Bsplit[k][split][n][kk] bf16, n < 2 nseg,
// kk < 2*nact_pad (hi = bf16(v), lo = bf16(v - hi)); killmask applied.
// Element pairs (kk = 2j, 2j+1) are written as one 32-bit word.
__global__ void __launch_bounds__(256) fdd_prep_b_kernel(const float2* X, size_t bin_pitch, int nseg,
                                                         size_t nbins, const int32_t* chan,
                                                         const float* km, int nact, int nact_pad,
                                                         int npad, uint32_t* B, BinMap map, int seg0,
                                                         int nseg_total)
{
    // segments seg0 .. seg0 + nseg - 1 of X rows c * nseg_total + s
    // one block per (tile of 32 row positions of X, channel tile of 32),
    // looping over n; position p holds bin pbin(p) (BinMap order)
    auto pbin = [&](size_t p) -> size_t {
        return (map.Q <= 1 || p >= map.M) ? p : (size_t)map.Q * (p & (map.P - 1)) + p / map.P;
    };
    __shared__ float2 tile[32][33];
    const size_t k0 = (size_t)blockIdx.x * 32;
    const int j0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const size_t words_row = (size_t)nact_pad;  // 2*nact_pad bf16 per row
    // B holds the 2*nseg real rows of each bin; the MMA's rows up to npad are
    // zeros that the tensor-map load fills in (out-of-bounds fill)
    const size_t nrow = 2 * (size_t)nseg;
    // the next segment's loads are issued before this segment's stores
    float2 nv[4];
    auto load = [&](int s) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int j = j0 + ty + 8 * i;
            const size_t k = k0 + tx;
            nv[i] = (j < nact && k < nbins) ? X[((size_t)chan[j] * nseg_total + seg0 + s) * bin_pitch + k]
                                            : make_float2(0.f, 0.f);
        }
    };
    load(0);
    for (int s = 0; s < nseg; ++s) {
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int j = j0 + ty + 8 * i;
            const float w = j < nact ? km[j] : 0.f;
            tile[ty + 8 * i][tx] = make_float2(nv[i].x * w, nv[i].y * w);
        }
        if (s + 1 < nseg) load(s + 1);
        __syncthreads();
        for (int r = ty; r < 32; r += 8) {
            if (k0 + r >= nbins || j0 + tx >= nact_pad) continue;
            const size_t k = pbin(k0 + r);
            const int j = j0 + tx;
            const float2 v = tile[tx][r];
            // real-output column s: (Xr, -Xi); imaginary-output column
            // nseg + s: (Xi, Xr); element 2j in the low half, 2j+1 high
            const float vals[2][2] = {{v.x, -v.y}, {v.y, v.x}};
#pragma unroll
            for (int part = 0; part < 2; ++part) {
                const int n = part * nseg + s;
                const float a0 = vals[part][0], a1 = vals[part][1];
                const float h0 = __bfloat162float(__float2bfloat16_rn(a0));
                const float h1 = __bfloat162float(__float2bfloat16_rn(a1));
                B[((k * 2 + 0) * nrow + n) * words_row + j] = bf16x2_bits(h0, h1);
                B[((k * 2 + 1) * nrow + n) * words_row + j] = bf16x2_bits(a0 - h0, a1 - h1);
            }
        }
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    // initialised once, thread-safely (a failed lookup throws and is retried
    // by the next call)
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        RT_CHECK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (!p || q != cudaDriverEntryPointSuccess)
            DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "cuTensorMapEncodeTiled unavailable");
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

}  // namespace

size_t tc_b_bytes(size_t nbins, int nact_pad, int nseg)
{
    return nbins * 2 * (2 * (size_t)nseg) * 2 * (size_t)nact_pad * sizeof(__nv_bfloat16);
}

int tc_pad_channels(int nact) { return ((nact + TC_CHUNK - 1) / TC_CHUNK) * TC_CHUNK; }
int tc_pad_n(int nseg) { return ((2 * nseg + 15) / 16) * 16; }
bool tc_quarter_mode_fits(unsigned nfft, int nact_pad, int npad)
{
    if (nfft < 256 || (nfft & (nfft - 1)) != 0) return false;  // quarter-wave indexing needs a power of two
    return tc_smem_bytes(nfft, nact_pad, npad, -1, 2, false) <= TC_MAX_SMEM;
}

void launch_fdd_prep_b(const float2* X, size_t bin_pitch, int nseg, size_t nbins,
                       const int32_t* chan, const float* km, int nact, int nact_pad, int npad,
                       void* B, const BinMap& map, int seg0, int nseg_total, cudaStream_t s)
{
    // every word of B is written (zeros for padding rows and channels)
    dim3 grid((unsigned)((nbins + 31) / 32), (unsigned)((nact_pad + 31) / 32));
    fdd_prep_b_kernel<<<grid, 256, 0, s>>>(X, bin_pitch, nseg, nbins, chan, km, nact, nact_pad, npad,
                                           static_cast<uint32_t*>(B), map, seg0, nseg_total);
    RT_CHECK(cudaGetLastError());
}

std::vector<uint2> tc_quarter_table(unsigned nfft)
{
    // exp(+2 pi i r / nfft), r = 0..nfft/4, split into bf16 hi + lo parts
    // (re in the low half of each packed word, im in the high half).
    auto bf16_bits = [](double x) -> uint32_t {
        const float f = (float)x;
        uint32_t u;
        std::memcpy(&u, &f, 4);
        const uint32_t rounding = 0x7FFFu + ((u >> 16) & 1u);  // round to nearest even
        return ((u + rounding) >> 16) & 0xFFFFu;
    };
    auto bf16_val = [](uint32_t b) -> double {
        const uint32_t u = b << 16;
        float f;
        std::memcpy(&f, &u, 4);
        return (double)f;
    };
    const unsigned qn = nfft / 4;
    std::vector<uint2> t(qn + 1);
    for (unsigned r = 0; r <= qn; ++r) {
        const double th = 2.0 * 3.14159265358979323846 * (double)r / (double)nfft;
        const double c = std::cos(th), s = std::sin(th);
        const uint32_t ch = bf16_bits(c), sh = bf16_bits(s);
        const uint32_t cl = bf16_bits(c - bf16_val(ch)), sl = bf16_bits(s - bf16_val(sh));
        t[r] = make_uint2(ch | (sh << 16), cl | (sl << 16));
    }
    return t;
}

// Dynamic shared memory of fdd_mac_tc_kernel: base alignment, the B stages
// (three-MMA form, the larger), barriers, the phasor table and the two
// twiddle tables (float2 tables padded to even counts, 16-byte aligned), the
// channel delays and the abort flag.
size_t tc_layout_bytes(int npad, size_t table_entries, size_t hi_entries, int nact_pad, int stages)
{
    const size_t stage = 4ull * (size_t)npad * 128ull;
    const size_t need = 1024 + (size_t)stages * stage + 256 +
                        (((table_entries + 1) & ~(size_t)1) + 256 + ((hi_entries + 1) & ~(size_t)1)) * 8 +
                        (size_t)nact_pad * 4 + 4 * 8;
    return std::max(need, TC_MIN_SMEM);
}

size_t tc_smem_bytes(unsigned nfft, int nact_pad, int npad, int dmax, int stages, bool direct)
{
    // one descriptor: table mode: dmax + 1 phasors and the twiddle tables;
    // direct mode: the twiddle tables; quarter-wave mode: nfft/4 + 1 phasors
    const size_t table = dmax >= 0 ? (size_t)dmax + 1 : direct ? 0 : (size_t)nfft / 4 + 1;
    const size_t hi = (dmax >= 0 || direct) ? (size_t)nfft / 256 : 0;
    return tc_layout_bytes(npad, table, hi, nact_pad, stages);
}

int tc_table_capacity(int npad, size_t hi_entries, int nact_pad)
{
    // largest entry count t (= cap + 1) whose layout fits: bytes grow with t
    size_t lo = 0, hi = TC_MAX_SMEM / 8;
    if (tc_layout_bytes(npad, 1, hi_entries, nact_pad, 2) > TC_MAX_SMEM) return -1;
    lo = 1;
    while (lo < hi) {
        const size_t mid = (lo + hi + 1) / 2;
        if (tc_layout_bytes(npad, mid, hi_entries, nact_pad, 2) <= TC_MAX_SMEM) lo = mid;
        else hi = mid - 1;
    }
    return (int)lo - 1;
}

int tc_table_cap_limit()
{
    const char* v = std::getenv("DEDISP_TC_TABLE_CAP");
    if (!v || !*v) return INT_MAX;
    const long x = std::strtol(v, nullptr, 10);
    return x < 0 ? -1 : (int)std::min<long>(x, INT_MAX);
}

TcSource tc_choose_source(int dmax, unsigned nfft, int table_cap, bool quarter_fits)
{
    TcSource s;
    if (dmax >= 0 && dmax <= table_cap) {
        s.dmax = dmax;  // every delay from the per-bin table
        return s;
    }
    const bool twiddles = nfft % 256 == 0 && table_cap >= 0;  // room for the twiddle tables
    // relative cost per phasor: table gather 1, quarter-wave gather 1.3,
    // direct 2.5 (a reduction, two twiddle loads, a complex product)
    double best = 1e30;
    if (quarter_fits) best = 1.3;
    if (twiddles && dmax >= 0 && dmax < (1 << 22) && table_cap >= 1024) {
        // share of (DM, channel) delays inside the table when both the DMs and
        // the channel delays spread evenly from zero: c (1 - ln c)
        const double c = (double)(table_cap + 1) / (double)(dmax + 1);
        const double cov = c * (1.0 - std::log(c));
        const double cost = cov + 2.5 * (1.0 - cov);
        if (cost < best) {
            best = cost;
            s.dmax = table_cap;
            s.hybrid = 1;
        }
    }
    if (best > 2.5 && twiddles) {
        s.direct = 1;
        best = 2.5;
    }
    if (best > 2.5) s.dmax = -2;  // no source fits
    return s;
}

int tc_stages(unsigned nfft, int nact_pad, int npad, int dmax, bool direct)
{
    int st = TC_MAX_STAGES;
    while (st > 2 && tc_smem_bytes(nfft, nact_pad, npad, dmax, st, direct) > TC_MAX_SMEM) --st;
    return st;
}

bool tc_direct_mode_fits(unsigned nfft, int nact_pad, int npad)
{
    return nfft % 256 == 0 && tc_smem_bytes(nfft, nact_pad, npad, -1, 2, true) <= TC_MAX_SMEM;
}

void tc_encode_map(void* map_out, const TcMacArgs& a, const void* B, bool pair)
{
    // Tensor map over Bsplit[bin][split][n][kk]: dims (kk, n, split, bin).
    CUtensorMap* map = static_cast<CUtensorMap*>(map_out);
    // (kk, n < 2 nseg stored rows, split, bin); the box's npad rows past the
    // stored ones read as zero (out-of-bounds fill), the count is the full box
    const cuuint64_t nrow = 2 * (cuuint64_t)a.nseg;
    const cuuint64_t dims[4] = {(cuuint64_t)(2 * a.nact_pad), nrow, 2, (cuuint64_t)a.nbins};
    const cuuint64_t strides[3] = {(cuuint64_t)(2 * a.nact_pad) * 2, (cuuint64_t)(2 * a.nact_pad) * 2 * nrow,
                                   (cuuint64_t)(2 * a.nact_pad) * 2 * nrow * 2};
    // pairs: each CTA loads half of the MMA's rows
    const cuuint32_t box[4] = {64, (cuuint32_t)(pair ? a.npad / 2 : a.npad), 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = encode_fn()(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(B),
                                   dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                   CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "cuTensorMapEncodeTiled failed");
}

bool tc_pair_mode(const std::vector<TcMacArgs>& descs)
{
    // DEDISP_TC_PAIR=1 asks for pairs wherever they fit. Not the default:
    // a pair issues one M = 256 MMA where two CTAs issue two M = 128 ones, at
    // the same rate per SM, so only the halved B loads per CTA remain (config
    // 2: 38.9 against 40.5 ms; one segment: 1129 against 1078 ms; per-beam
    // config-3 plans 2.5 % slower)
    const char* e = std::getenv("DEDISP_TC_PAIR");
    if (!e || std::atoi(e) != 1) return false;
    const char* form = std::getenv("DEDISP_TC_FORM");
    if (form && (std::atoi(form) == 1 || std::atoi(form) == 3)) return false;  // no paired fused forms
    for (const TcMacArgs& a : descs)
        if ((2 * a.nseg + 31) / 32 * 32 > 128) return false;
    return tc_sm_count() >= 2;
}

TcMacArgs tc_finish_args(const TcMacArgs& a, bool pair)
{
    TcMacArgs ka = a;
    if (ka.nseg_total <= 0) ka.nseg_total = ka.nseg;
    // pairs: the M = 256 MMA takes N in multiples of 32 (16 rows per CTA)
    if (pair) ka.npad = (std::max(ka.npad, 2 * ka.nseg) + 31) / 32 * 32;
    if (ka.nseg > kTcMaxSeg || ka.seg0 + ka.nseg > ka.nseg_total || ka.npad < 2 * ka.nseg ||
        ka.npad % 16 != 0 || ka.npad > 128 || ka.nact_pad % TC_CHUNK != 0 || ka.nfft % 256 != 0)
        DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "tensor-core MAC: bad shape");
    // Barrett constant floor((2^64 - 1) / N) for (k d) mod N in direct mode
    ka.nmagic = ~0ull / (unsigned long long)ka.nfft;
    return ka;
}

TcLayout tc_layout(const std::vector<TcMacArgs>& descs, unsigned* err, bool pair)
{
    if (descs.empty()) DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "tensor-core MAC: no descriptors");
    TcLayout L{};
    int npad = 16;
    size_t table = 0, hi = 0;
    for (const TcMacArgs& a : descs) {
        npad = std::max(npad, a.npad);
        const size_t t = a.dmax >= 0 ? (size_t)a.dmax + 1 : a.direct ? 0 : (size_t)a.nfft / 4 + 1;
        table = std::max(table, t);
        if (a.dmax >= 0 || a.direct) hi = std::max(hi, (size_t)a.nfft / 256);
        if (a.nact_pad != descs[0].nact_pad)
            DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "tensor-core MAC: descriptors differ in channels");
    }
    // MMA form: the three-MMA form unless DEDISP_TC_FORM=1 asks for the fused
    // form (which needs npad <= 80; its 32-channel chunks double the hand-offs
    // per channel: config 2 41.6 against 40.5 ms), kept selectable
    const char* form = std::getenv("DEDISP_TC_FORM");
    L.pair = pair ? 1 : 0;
    const int fsel = form ? std::atoi(form) : 0;
    // the fused form at 64-channel chunks wherever npad <= 32 (DEDISP_TC_FORM=1
    // or 2 select the others): 16 MMAs per chunk instead of 24; measured
    // 4491 -> 4101 ms of MAC over the first 12 config-3 beams (reference
    // segments), 1077 -> 872 ms for the config-2 whole-series spectrum
    const bool wide = !pair && (fsel == 0 || fsel == 3) && npad <= 32;
    L.fused = (wide || (!pair && fsel == 1 && npad <= TC_FUSED_MAX_NPAD)) ? 1 : 0;
    // three A buffers when the accumulators fit in 64 columns (DEDISP_TC_FORM=2
    // keeps two, for comparison); the wide fused form always has three
    L.deep = (wide || (!L.fused && npad <= TC_DEEP_MAX_NPAD && fsel != 2)) ? 1 : 0;
    // a stage: 2 splits x (CH / 64 atoms) x the CTA's B rows x 128 bytes
    L.stage_bytes = ((L.fused && !L.deep) ? 2u : 4u) * (uint32_t)(pair ? npad / 2 : npad) * 128u;
    L.table_entries = (uint32_t)((table + 1) & ~(size_t)1);  // keep the float2 tables 16-byte aligned
    L.tw_hi_entries = (uint32_t)((hi + 1) & ~(size_t)1);
    L.nact_pad = descs[0].nact_pad;
    // the fused form's stages are half as large: the same formula at npad / 2
    auto bytes = [&](int st) {
        return tc_layout_bytes((int)(L.stage_bytes / 512u), L.table_entries, L.tw_hi_entries, L.nact_pad, st);
    };
    int st = TC_MAX_STAGES;
    while (st > 2 && bytes(st) > TC_MAX_SMEM) --st;
    if (bytes(st) > TC_MAX_SMEM)
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "tensor-core MAC: tables do not fit shared memory");
    L.stages = st;
    L.smem_bytes = bytes(st);
    L.wait_ns = rt::wait_limit_ns();
    L.wait_test = rt::wait_expiry_test() ? 1 : 0;
    L.err = err;
    return L;
}

std::vector<TcWork> tc_work_items(const std::vector<TcMacArgs>& descs, int ctas)
{
    // An item is a bin range of one descriptor over all its DM tiles (the
    // per-bin phasor table is built once for every tile). With CTA pairs the
    // units are pairs and the tiles 256 DMs.
    const bool pair = tc_pair_mode(descs);
    const int tile_m = pair ? 2 * TC_M : TC_M;
    ctas = std::max(pair ? ctas / 2 : ctas, 1);
    std::vector<TcWork> items;
    if (descs.size() == 1) {
        // one descriptor: at most `ctas` equal items, CTA b takes item b
        const TcMacArgs& a = descs[0];
        const int ntiles = (a.ndm + tile_m - 1) / tile_m;
        const size_t parts = std::max<size_t>(1, std::min<size_t>(a.nbins, (size_t)ctas));
        for (size_t p = 0; p < parts; ++p) {
            const size_t k0 = a.nbins * p / parts, k1 = a.nbins * (p + 1) / parts;
            if (k0 < k1) items.push_back(TcWork{0, 0, ntiles, (unsigned)k0, (unsigned)k1});
        }
        return items;
    }
    // Several descriptors (a batch of beams): items of about 1/32 of a CTA's
    // share of an estimated cost per bin (tiles x chunks x (phasor source +
    // columns)), listed longest first. CTA b starts with item b and then
    // claims the next unclaimed item whenever it finishes one, so the
    // estimate only orders the list and the tail is at most one small item.
    auto cost_per_bin = [&](const TcMacArgs& a) {
        const double ntiles = (double)((a.ndm + tile_m - 1) / tile_m);
        const double phasor = a.dmax >= 0 ? (a.hybrid ? 1.8 : 1.0) : a.direct ? 2.5 : 1.3;
        return ntiles * (double)(a.nact_pad / TC_CHUNK) * (phasor + (double)a.npad / 48.0);
    };
    double total = 0;
    for (const TcMacArgs& a : descs) total += cost_per_bin(a) * (double)a.nbins;
    // (8 items per CTA left 10 % of tail on the first 12 config-3 beams, 32 and
    // 64 under 2 %)
    const double per = std::max(1e-9, total / (32.0 * ctas));
    std::vector<std::pair<double, TcWork>> parts;
    for (size_t d = 0; d < descs.size(); ++d) {
        const TcMacArgs& a = descs[d];
        const double cb = cost_per_bin(a);
        const int ntiles = (a.ndm + tile_m - 1) / tile_m;
        const size_t n = std::max<size_t>(1, std::min<size_t>(a.nbins, (size_t)std::ceil(cb * (double)a.nbins / per)));
        for (size_t p = 0; p < n; ++p) {
            const size_t k0 = a.nbins * p / n, k1 = a.nbins * (p + 1) / n;
            if (k0 < k1) parts.push_back({cb * (double)(k1 - k0), TcWork{(int)d, 0, ntiles, (unsigned)k0, (unsigned)k1}});
        }
    }
    std::stable_sort(parts.begin(), parts.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    for (const auto& pw : parts) items.push_back(pw.second);
    return items;
}

size_t tc_work_bytes(size_t nitems) { return nitems * sizeof(TcWork) + 256; }

int tc_sm_count()
{
    int dev = 0, sms = 148;
    RT_CHECK(cudaGetDevice(&dev));
    RT_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return sms;
}

void tc_prepare_list(TcParams& P, const std::vector<TcMacArgs>& descs_in, const std::vector<const void*>& Bs,
                     const std::vector<TcWork>& items, unsigned* err, void* d_items, size_t items_bytes,
                     cudaStream_t s)
{
    if (descs_in.empty() || descs_in.size() != Bs.size() || descs_in.size() > (size_t)kTcMaxDesc)
        DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "tensor-core MAC: 1 to 48 descriptors per launch");
    const bool pair = tc_pair_mode(descs_in);
    const int tile_m = pair ? 2 * TC_M : TC_M;
    std::vector<TcMacArgs> descs;
    for (size_t d = 0; d < descs_in.size(); ++d) {
        descs.push_back(tc_finish_args(descs_in[d], pair));
        P.descs[d] = descs.back();
        tc_encode_map(&P.maps[d], descs.back(), Bs[d], pair);
    }
    P.ndesc = (int)descs.size();
    if (tc_work_bytes(items.size()) > items_bytes)
        DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "tensor-core MAC: work buffer too small");
    for (const TcWork& w : items)
        if (w.desc < 0 || w.desc >= P.ndesc || w.k_end > descs[w.desc].nbins || w.k_begin > w.k_end ||
            w.tile < 0 || w.ntile < 1 || (w.tile + w.ntile - 1) * tile_m >= descs[w.desc].ndm)
            DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "tensor-core MAC: bad work item");
    // pageable source: the call returns once the bytes are staged
    if (!items.empty())
        RT_CHECK(cudaMemcpyAsync(d_items, items.data(), items.size() * sizeof(TcWork), cudaMemcpyHostToDevice, s));
    P.items = static_cast<const TcWork*>(d_items);
    P.nitems = (int)items.size();
    P.next_item = reinterpret_cast<unsigned*>(static_cast<uint8_t*>(d_items) +
                                              (items.size() * sizeof(TcWork) + 15) / 16 * 16);
    P.layout = tc_layout(descs, err, pair);
}

void launch_fdd_mac_tc_list(const TcParams& P, cudaStream_t s)
{
    if (P.nitems <= 0) return;
    RT_CHECK(cudaMemsetAsync(P.next_item, 0, sizeof(unsigned), s));
    if (P.layout.pair) {
        auto kern = P.layout.deep ? fdd_mac_tc_kernel<false, true, true> : fdd_mac_tc_kernel<false, false, true>;
        rt::raise_smem_limit(kern, P.layout.smem_bytes);
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.blockDim = dim3(TC_THREADS);
        cfg.dynamicSmemBytes = P.layout.smem_bytes;
        cfg.stream = s;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        // as many pairs as can be resident at once (one CTA per SM)
        int pairs = tc_sm_count() / 2;
        cfg.gridDim = dim3((unsigned)(2 * pairs));
        int resident = 0;
        if (cudaOccupancyMaxActiveClusters(&resident, kern, &cfg) == cudaSuccess && resident > 0)
            pairs = std::min(pairs, resident);
        else
            (void)cudaGetLastError();
        pairs = std::max(1, std::min(pairs, P.nitems));
        cfg.gridDim = dim3((unsigned)(2 * pairs));
        RT_CHECK(cudaLaunchKernelEx(&cfg, kern, P));
        RT_CHECK(cudaGetLastError());
        return;
    }
    auto kern = P.layout.fused  ? (P.layout.deep ? fdd_mac_tc_kernel<true, true, false>
                                                 : fdd_mac_tc_kernel<true, false, false>)
                : P.layout.deep ? fdd_mac_tc_kernel<false, true, false>
                                : fdd_mac_tc_kernel<false, false, false>;
    rt::raise_smem_limit(kern, P.layout.smem_bytes);
    const int grid = std::min(P.nitems, tc_sm_count());
    kern<<<grid, TC_THREADS, P.layout.smem_bytes, s>>>(P);
    RT_CHECK(cudaGetLastError());
}

int tc_form_code(const TcLayout& L)
{
    return L.fused ? (L.deep ? 5 : 1) : L.pair ? (L.deep ? 4 : 3) : L.deep ? 2 : 0;
}

int launch_fdd_mac_tc(const TcMacArgs& a, const void* B, void* d_items, size_t items_bytes, cudaStream_t s)
{
    const std::vector<TcMacArgs> descs{tc_finish_args(a, false)};
    const std::vector<TcWork> items = tc_work_items(descs, tc_sm_count());
    std::unique_ptr<TcParams> P(new TcParams());
    tc_prepare_list(*P, descs, {B}, items, a.err, d_items, items_bytes, s);
    launch_fdd_mac_tc_list(*P, s);
    return tc_form_code(P->layout);
}

}  // namespace kern
}  // namespace dedisp
