// Allocation-free time-domain dedispersion.
//
// Some callers cannot call cudaMalloc: real-time pipelines that forbid
// allocation once they have started (an allocation can block on the driver
// for an unbounded time), and hosts whose device memory is owned by another
// allocator (a framework pool or a fixed memory budget). For them this file provides one extra C entry
// point that performs the same computation as TDDPlan::execute with
// DEDISP_DEVICE_POINTERS (K1 transpose + tiled K2 kernel) but never allocates
// device memory. Its scratch -- the channel-major copy of the input and the
// small per-call tables -- lives in file-scope __device__ arrays of a fixed
// maximum size, which every GPU that loads the library holds until exit.
//
// The host code obtains the device address of each array with
// cudaGetSymbolAddress, once per device, on the first call made with that
// device current; that first call should therefore come before any stream
// capture. All calls share the arrays: two calls that overlap on the GPU
// (from different host threads or streams) race on them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "dedisp_b200.h"
#include "errors.hpp"
#include "host_math.hpp"
#include "runtime.hpp"
#include "tdd_kernels.hpp"

namespace {

// Stated maximum sizes of the allocation-free path.
constexpr size_t kScratchWords = (size_t)16 << 20;  // 64 MiB channel-major input
constexpr size_t kMaxDms = 16384;
constexpr size_t kMaxChans = 8192;
constexpr size_t kListPad = 64;

}  // namespace

// Scratch and per-call tables of the allocation-free path (file scope).
static __device__ __align__(256) uint32_t g_noalloc_scratch[kScratchWords];
static __device__ __align__(256) float g_noalloc_dms[kMaxDms];
static __device__ __align__(256) int32_t g_noalloc_perm[kMaxDms];
static __device__ __align__(256) float g_noalloc_delays[kMaxChans + 1];
static __device__ __align__(256) int32_t g_noalloc_chan[kMaxChans + kListPad];

namespace {

struct DeviceSymbols {
    bool ready = false;
    uint32_t* scratch = nullptr;
    float* dms = nullptr;
    int32_t* perm = nullptr;
    float* delays = nullptr;
    int32_t* chan = nullptr;
};

constexpr int kMaxDevices = 64;
DeviceSymbols g_symbols[kMaxDevices];
std::mutex g_symbols_mutex;

thread_local std::string t_noalloc_msg;

dedisp_error fail(dedisp_error code, const char* msg)
{
    t_noalloc_msg = msg;
    return code;
}

// Resolves the device addresses of the arrays for the current device, which
// must be the device of `stream` (the arrays' addresses differ per device).
dedisp_error symbols_for_current_device(cudaStream_t stream, DeviceSymbols** out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(DEDISP_INVALID_DEVICE_INDEX, "no usable current CUDA device");
    if (stream) {
        int sdev = -1;
        if (cudaStreamGetDevice(stream, &sdev) != cudaSuccess) {
            cudaGetLastError();
            return fail(DEDISP_INVALID_DEVICE_INDEX, "cannot query the stream's device");
        }
        if (sdev != dev)
            return fail(DEDISP_INVALID_DEVICE_INDEX, "the stream belongs to another device than the current one");
    }
    std::lock_guard<std::mutex> lock(g_symbols_mutex);
    DeviceSymbols& s = g_symbols[dev];
    if (!s.ready) {
        if (cudaGetSymbolAddress((void**)&s.scratch, g_noalloc_scratch) != cudaSuccess ||
            cudaGetSymbolAddress((void**)&s.dms, g_noalloc_dms) != cudaSuccess ||
            cudaGetSymbolAddress((void**)&s.perm, g_noalloc_perm) != cudaSuccess ||
            cudaGetSymbolAddress((void**)&s.delays, g_noalloc_delays) != cudaSuccess ||
            cudaGetSymbolAddress((void**)&s.chan, g_noalloc_chan) != cudaSuccess) {
            cudaGetLastError();
            return fail(DEDISP_INTERNAL_GPU_ERROR, "cudaGetSymbolAddress failed");
        }
        s.ready = true;
    }
    *out = &s;
    return DEDISP_NO_ERROR;
}

size_t round_up(size_t a, size_t b) { return (a + b - 1) / b * b; }

bool valid_nbits(size_t n) { return n == 1 || n == 2 || n == 4 || n == 8 || n == 16 || n == 32; }

}  // namespace

extern "C" dedisp_error dedisp_b200_tdd_execute_noalloc(
    dedisp_size nchans, dedisp_float dt, dedisp_float f0, dedisp_float df,
    const dedisp_float* dm_list, dedisp_size dm_count, const dedisp_bool* killmask,
    dedisp_size nsamps, const dedisp_byte* d_in, dedisp_size in_nbits, dedisp_size in_stride,
    dedisp_byte* d_out, dedisp_size out_nbits, dedisp_size out_stride, void* stream)
{
    using namespace dedisp;
    t_noalloc_msg.clear();  // the message describes this call's failure only
    if (!dm_list || !d_in || !d_out) return fail(DEDISP_INVALID_POINTER, "NULL pointer");
    if (dm_count == 0) return fail(DEDISP_NO_DM_LIST_SET, "empty DM list");
    if (!valid_nbits(in_nbits) || (nchans * in_nbits) % 32 != 0)
        return fail(DEDISP_UNSUPPORTED_IN_NBITS, "unsupported in_nbits for this channel count");
    if (out_nbits != 8 && out_nbits != 16 && out_nbits != 32)
        return fail(DEDISP_UNSUPPORTED_OUT_NBITS, "unsupported out_nbits");
    if (nchans == 0 || nchans > kMaxChans)
        return fail(DEDISP_NCHANS_EXCEEDS_LIMIT, "nchans exceeds the 8192-channel limit");
    if (dm_count > kMaxDms)
        return fail(DEDISP_MEM_ALLOC_FAILED, "dm_count exceeds the 16384-DM limit of the "
                                             "allocation-free path");

    // Host set-up with the reference arithmetic (delay table, max delay).
    std::vector<float> delays(nchans);
    hostmath::delay_table(nchans, dt, f0, df, delays.data());
    const size_t max_delay = hostmath::max_delay(dm_list[dm_count - 1], delays[nchans - 1]);
    const size_t ob = out_nbits / 8;
    if (in_stride < nchans * in_nbits / 8) return fail(DEDISP_INVALID_STRIDE, "in_stride too small");
    if (nsamps < max_delay) return fail(DEDISP_TOO_FEW_NSAMPS, "nsamps < max delay");
    const size_t nsamp_out = nsamps - max_delay;
    if (out_stride < nsamp_out * ob || out_stride % ob != 0)
        return fail(DEDISP_INVALID_STRIDE, "out_stride too small or not a multiple of the sample size");
    if (nsamp_out == 0) return DEDISP_NO_ERROR;

    // Active channels: this path runs the tiled kernel, which needs a 0/1 mask.
    std::vector<int32_t> chan;
    for (size_t c = 0; c < nchans; ++c) {
        const int km = killmask ? killmask[c] : 1;
        if (km != 0 && km != 1)
            return fail(DEDISP_UNKNOWN_ERROR, "killmask values other than 0/1 are not supported "
                                              "by the allocation-free path");
        if (km) chan.push_back((int32_t)c);
    }
    const int nact = (int)chan.size();

    // DMs in ascending order with the output row of each slot.
    std::vector<int32_t> perm(dm_count);
    std::iota(perm.begin(), perm.end(), 0);
    auto key = [&](int32_t i) { return std::isnan(dm_list[i]) ? -INFINITY : dm_list[i]; };
    std::stable_sort(perm.begin(), perm.end(), [&](int32_t a, int32_t b) { return key(a) < key(b); });
    std::vector<float> dms(dm_count);
    for (size_t i = 0; i < dm_count; ++i) dms[i] = dm_list[perm[i]];

    uint32_t tmax = 0;
    for (int j = 0; j < nact; ++j) {
        const float dl = delays[chan[j]];
        tmax = std::max(tmax, std::max(hostmath::delay_rn(dms.front(), dl),
                                       hostmath::delay_rn(dms.back(), dl)));
    }
    const int nbits = (int)in_nbits;
    const size_t spw = 32 / nbits;
    const size_t bd = (size_t)kern::tiled_block_dms(nbits, 0);
    const size_t bt = (size_t)kern::tiled_block_samples(nbits, 0);
    const size_t J = (size_t)kern::tiled_lane_words(nbits, 0);
    uint32_t span = 0;
    for (size_t t = 0; t < dm_count; t += bd) {
        const float f = dms[t], l = dms[std::min(t + bd, (size_t)dm_count) - 1];
        for (int j = 0; j < nact; ++j) {
            const float dl = delays[chan[j]];
            const uint32_t a = hostmath::delay_rn(f, dl), b = hostmath::delay_rn(l, dl);
            span = std::max(span, a > b ? a - b : b - a);
        }
    }
    const size_t win = round_up((span + 4 * spw - 1) / spw + 32 * J + 1, 4);
    if (win > ((size_t)1 << 26)) return fail(DEDISP_UNKNOWN_ERROR, "DM spacing too wide for the tiled kernel");
    const int cs = kern::tiled_stage_channels(nbits, (int)win, 0);
    if (cs < 2) return fail(DEDISP_UNKNOWN_ERROR, "DM spacing too wide for the tiled kernel");
    const int nstages = std::max(1, (nact + cs - 1) / cs);
    if ((size_t)nstages * cs > kMaxChans + kListPad)
        return fail(DEDISP_NCHANS_EXCEEDS_LIMIT, "channel list exceeds the static table");
    chan.resize((size_t)nstages * cs, (int32_t)nchans);

    const size_t pitch = round_up((round_up(nsamp_out, bt) + tmax + spw - 1) / spw + win + 8, 32);
    if ((nchans + 1) * pitch > kScratchWords)
        return fail(DEDISP_MEM_ALLOC_FAILED,
                    "input too large for the 64 MiB allocation-free scratch: (nchans+1) x "
                    "(nsamps - max_delay + max delay) samples must fit");

    DeviceSymbols* sym = nullptr;
    const dedisp_error se = symbols_for_current_device(static_cast<cudaStream_t>(stream), &sym);
    if (se != DEDISP_NO_ERROR) return se;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    delays.push_back(0.f);  // the all-zero padding channel
    try {
        // Stream-ordered copies into the static tables (pageable sources are
        // staged by the driver before these calls return).
        RT_CHECK(cudaMemcpyAsync(sym->dms, dms.data(), dm_count * 4, cudaMemcpyHostToDevice, st));
        RT_CHECK(cudaMemcpyAsync(sym->perm, perm.data(), dm_count * 4, cudaMemcpyHostToDevice, st));
        RT_CHECK(cudaMemcpyAsync(sym->delays, delays.data(), delays.size() * 4,
                                 cudaMemcpyHostToDevice, st));
        RT_CHECK(cudaMemcpyAsync(sym->chan, chan.data(), chan.size() * 4, cudaMemcpyHostToDevice, st));
        // The padding channel row must read as zero; the transpose rewrites
        // every other word of the rows it uses.
        RT_CHECK(cudaMemsetAsync(sym->scratch + nchans * pitch, 0, pitch * 4, st));
        kern::TransposeArgs ta{d_in, in_stride, std::min(nsamps, nsamp_out + tmax), nchans, nbits,
                               sym->scratch, pitch, 0, pitch};
        kern::launch_transpose(ta, st);
        kern::DedisperseArgs da{};
        da.tr = sym->scratch;
        da.tr_pitch_words = pitch;
        da.nbits = nbits;
        da.nchans = nchans;
        da.chan_list = sym->chan;
        da.nact = nact;
        da.nstages = nstages;
        da.km_vals = nullptr;  // the tiled kernel reads no per-channel multipliers (0/1 mask)
        da.delay_table = sym->delays;
        da.dms = sym->dms;
        da.perm = sym->perm;
        da.ndm = (int)dm_count;
        da.nsamp_out = nsamp_out;
        da.out = d_out;
        da.out_stride = out_stride / ob;
        da.out_nbits = (int)out_nbits;
        const float in_range = (float)(nbits == 32 ? 0xFFFFFFFFu : ((1u << nbits) - 1u));
        da.den = in_range * (float)nchans;
        da.factor = 3.f * 1024.f / 255.f / 16.f;
        da.win_words = (int)win;
        da.chan_per_stage = cs;
        kern::launch_dedisperse_tiled(da, st);
        // The host tables above are only guaranteed to have been consumed
        // once the stream reaches this point.
        RT_CHECK(cudaStreamSynchronize(st));
    } catch (const Error& e) {
        return fail(e.code(), e.what());
    } catch (...) {
        return fail(DEDISP_UNKNOWN_ERROR, "unexpected exception");
    }
    return DEDISP_NO_ERROR;
}

extern "C" const char* dedisp_b200_noalloc_last_message(void) { return t_noalloc_msg.c_str(); }
