// TDD execution engine (see tdd_engine.hpp).
#include "tdd_engine.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>

#include "host_math.hpp"
#include "tdd_kernels.hpp"

namespace dedisp {
namespace detail {

namespace {
constexpr int kMaxOutGroups = 8;                   // DM groups for D2H overlap

size_t round_up(size_t a, size_t b) { return (a + b - 1) / b * b; }
}  // namespace

// Everything derived from (DM list, killmask, DM range, nbits, kernel choice).
struct TddEngine::Setup {
    unsigned long version = ~0ul;
    size_t first = ~(size_t)0, count = ~(size_t)0;
    int nbits = -1;
    TddKernel kernel = TddKernel::Auto;
    int variant = -1;

    bool tiled = false;
    bool quad = false;           // 8-bit kernel on quad-strided rows
    int period = 0;              // quad: P, words per lane set
    int nact = 0;
    int win_words = 0;
    int chan_per_stage = 0;
    int nstages = 0;
    uint32_t tmax = 0;           // largest delay of the range over active channels
    bool identity = true;        // DM range already ascending
    std::vector<int32_t> chan_list;
    std::vector<uint32_t> km_vals;
    std::vector<float> dms;      // ascending (tiled) or in list order (plain)
    std::vector<int32_t> perm;   // output row of each slot
};

TddEngine::TddEngine(GpuState& gpu) : m_gpu(gpu), m_setup(new Setup()) {}
TddEngine::~TddEngine()
{
    if (m_gpu.has_device) {
        rt::DeviceGuard g(m_gpu.device);
        cudaStreamSynchronize(m_gpu.stream());
        if (m_gpu.d2h) cudaStreamSynchronize(m_gpu.d2h->get());
        if (m_gpu.h2d) cudaStreamSynchronize(m_gpu.h2d->get());
    }
}

rt::Event& TddEngine::event(size_t i)
{
    while (m_events.size() <= i) m_events.emplace_back(new rt::Event(false));
    return *m_events[i];
}

void TddEngine::prepare(const TddView& v, const TddCall& c)
{
    Setup& s = *m_setup;
    // variants are numbered per input width; one outside the width's range
    // (or -1) selects the width's default
    const int eff_variant = (variant >= 0 && variant < kern::tiled_variant_count(c.in_nbits))
                                ? variant
                                : kern::tiled_default_variant(c.in_nbits);
    if (s.version == v.version && s.first == c.first_dm && s.count == c.dm_count &&
        s.nbits == c.in_nbits && s.kernel == kernel && s.variant == eff_variant)
        return;

    Setup n;
    n.version = v.version;
    n.first = c.first_dm;
    n.count = c.dm_count;
    n.nbits = c.in_nbits;
    n.kernel = kernel;
    n.variant = eff_variant;

    // Active channels (killmask != 0) and their multipliers. The reference
    // multiplies every sample by its killmask value (dedisperse_kernel.cuh:
    // 177-179); 0/1 masks let the tiled kernel skip channels and multiplies.
    bool general = false;
    for (size_t ch = 0; ch < v.nchans; ++ch) {
        const int32_t km = v.killmask[ch];
        if (km == 0) continue;
        if (km != 1) general = true;
        n.chan_list.push_back((int32_t)ch);
        n.km_vals.push_back((uint32_t)km);
    }
    n.nact = (int)n.chan_list.size();

    // DM range in ascending order (NaN sorts first: its delay is 0).
    const float* src = v.dms + c.first_dm;
    std::vector<int32_t> order(c.dm_count);
    std::iota(order.begin(), order.end(), 0);
    auto key = [&](int32_t i) {
        const float d = src[i];
        return std::isnan(d) ? -INFINITY : d;
    };
    n.identity = std::is_sorted(order.begin(), order.end(),
                                [&](int32_t a, int32_t b) { return key(a) < key(b); });
    if (!n.identity)
        std::stable_sort(order.begin(), order.end(),
                         [&](int32_t a, int32_t b) { return key(a) < key(b); });
    n.dms.resize(c.dm_count);
    for (size_t i = 0; i < c.dm_count; ++i) n.dms[i] = src[order[i]];
    if (!n.identity) n.perm = order;

    // Largest delay: d(dm, c) is monotonic in dm, so the extreme DMs bound it.
    const float dlo = n.dms.front(), dhi = n.dms.back();
    for (int j = 0; j < n.nact; ++j) {
        const float dl = v.delays[n.chan_list[j]];
        n.tmax = std::max(n.tmax, std::max(hostmath::delay_rn(dlo, dl), hostmath::delay_rn(dhi, dl)));
    }

    n.tiled = (kernel != TddKernel::Plain) && !general;
    if (n.tiled) {
        const int bd = kern::tiled_block_dms(c.in_nbits, n.variant);
        const int spw = 32 / c.in_nbits;
        const int J = kern::tiled_lane_words(c.in_nbits, n.variant);
        uint32_t span = 0;
        for (size_t t = 0; t < c.dm_count; t += bd) {
            const float f = n.dms[t], l = n.dms[std::min(t + bd, (size_t)c.dm_count) - 1];
            for (int j = 0; j < n.nact; ++j) {
                const float dl = v.delays[n.chan_list[j]];
                const uint32_t a = hostmath::delay_rn(f, dl), b = hostmath::delay_rn(l, dl);
                span = std::max(span, a > b ? a - b : b - a);
            }
        }
        // quad-strided rows: a 1-sample delay is a 1-word offset, the window
        // is the lane set (P words) plus the span plus the 16-byte rounding
        n.quad = kern::tiled_variant_quad(c.in_nbits, n.variant);
        n.period = 32 * J;
        const size_t w = n.quad ? (size_t)span + 3 + (size_t)n.period
                                : (span + 4 * (size_t)spw - 1) / spw + 32 * (size_t)J + 1;
        n.win_words = (int)round_up(w, 4);
        const int cs = w > ((size_t)1 << 26) ? 0 : kern::tiled_stage_channels(c.in_nbits, n.win_words, n.variant);
        if (cs < 2) {
            n.tiled = false;
        } else {
            n.chan_per_stage = cs;
            n.nstages = std::max(1, (n.nact + cs - 1) / cs);
        }
    }
    if (kernel == TddKernel::Tiled && !n.tiled)
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "tiled kernel unavailable for this killmask/DM list");

    std::vector<int32_t> chan(n.chan_list);
    if (n.tiled) chan.resize((size_t)n.nstages * n.chan_per_stage, (int32_t)v.nchans);
    if (chan.empty()) chan.push_back((int32_t)v.nchans);
    // delay of each list entry (the padding channel's is 0)
    std::vector<float> cdl(chan.size());
    for (size_t j = 0; j < chan.size(); ++j) cdl[j] = chan[j] < (int32_t)v.nchans ? v.delays[chan[j]] : 0.f;

    cudaStream_t st = m_gpu.stream();
    m_chan.reserve(chan.size() * 4);
    RT_CHECK(cudaMemcpyAsync(m_chan.get(), chan.data(), chan.size() * 4, cudaMemcpyHostToDevice, st));
    m_cdl.reserve(cdl.size() * 4);
    RT_CHECK(cudaMemcpyAsync(m_cdl.get(), cdl.data(), cdl.size() * 4, cudaMemcpyHostToDevice, st));
    std::vector<uint32_t> km(n.km_vals);
    if (km.empty()) km.push_back(0);
    m_km.reserve(km.size() * 4);
    RT_CHECK(cudaMemcpyAsync(m_km.get(), km.data(), km.size() * 4, cudaMemcpyHostToDevice, st));
    m_dms.reserve(n.dms.size() * 4);
    RT_CHECK(cudaMemcpyAsync(m_dms.get(), n.dms.data(), n.dms.size() * 4, cudaMemcpyHostToDevice, st));
    if (!n.identity) {
        m_perm.reserve(n.perm.size() * 4);
        RT_CHECK(cudaMemcpyAsync(m_perm.get(), n.perm.data(), n.perm.size() * 4,
                                 cudaMemcpyHostToDevice, st));
    }
    // The host vectors must outlive the asynchronous copies.
    RT_CHECK(cudaStreamSynchronize(st));
    *m_setup = std::move(n);
}

void TddEngine::execute(const TddView& v, const TddCall& c)
{
    m_gpu.require_device();
    rt::DeviceGuard guard(m_gpu.device);
    stats = TddStats();

    const size_t nsamp_out = c.nsamps - v.max_delay;
    if (nsamp_out == 0 || c.dm_count == 0) return;
    prepare(v, c);
    const Setup& s = *m_setup;
    stats.tiled = s.tiled;

    const bool dev_in = (c.flags & DEDISP_DEVICE_POINTERS) != 0;
    const bool dev_out = dev_in;
    const int nbits = c.in_nbits;
    const size_t spw = 32 / nbits;
    const size_t ob = (size_t)c.out_nbits / 8;
    const size_t row_bytes = v.nchans * nbits / 8;
    const size_t ndm = c.dm_count;
    if (dev_out && c.out_stride % ob != 0)
        DD_THROW_MSG(DEDISP_INVALID_STRIDE, "device output stride must be a multiple of the sample size");

    const size_t bt = s.tiled ? (size_t)kern::tiled_block_samples(nbits, s.variant) : 16;
    const size_t win = s.tiled ? (size_t)s.win_words : 0;

    // Gulp size: the user cap, the grid limit, then device memory. With more
    // than one gulp the input rows and the output rows of a gulp have two
    // buffers each, so that gulp g+1's host-to-device copy and gulp g-1's
    // device-to-host copy run while gulp g is dedispersed.
    const size_t gulp_default = dev_in && dev_out ? kDefaultGulp : kHostDefaultGulp;
    size_t G = std::min(nsamp_out, gulp_set && gulp_size ? gulp_size : gulp_default);
    G = std::min(G, (size_t)65535 * bt);
    if (G < nsamp_out && G > bt) G = G / bt * bt;  // whole time tiles in every gulp but the last
    auto pitch_for = [&](size_t g) {
        return round_up((round_up(g, bt) + s.tmax + spw - 1) / spw + win + 8, 32);
    };
    // quad-strided rows: the tile windows read up to word
    // (tiles - 1) * bt + tmax + P + 2 of a row
    const bool quad = s.tiled && s.quad;
    auto qpitch_for = [&](size_t g) { return round_up(round_up(g, bt) + s.tmax + s.period + 4, 32); };
    auto nbuf_for = [&](size_t g) -> size_t { return nsamp_out > g ? 2 : 1; };
    auto in_bytes_for = [&](size_t g) { return round_up(g + s.tmax, 128) * row_bytes; };
    // quad-strided rows are built straight from the input rows (K1d); the
    // channel-major packed copy exists only for the other forms
    auto bytes_for = [&](size_t g) {
        size_t b = quad ? (v.nchans + 1) * qpitch_for(g) * 4 : (v.nchans + 1) * pitch_for(g) * 4;
        if (!dev_out) b += nbuf_for(g) * ndm * g * ob;
        if (!dev_in) b += nbuf_for(g) * in_bytes_for(g);
        return b;
    };
    size_t free_b = 0, total_b = 0;
    RT_CHECK(cudaMemGetInfo(&free_b, &total_b));
    const size_t avail = free_b + m_tr.capacity() + m_q.capacity() + m_out[0].capacity() + m_out[1].capacity() +
                         m_stage[0].capacity() + m_stage[1].capacity();
    while (G > bt && bytes_for(G) > avail / 100 * 90) G = round_up(G / 2, bt);
    if (bytes_for(G) > avail) DD_THROW(DEDISP_MEM_ALLOC_FAILED);

    const size_t nbuf = nbuf_for(G);
    const size_t pitch = pitch_for(G);
    if (!quad) m_tr.reserve((v.nchans + 1) * pitch * 4);
    const size_t qpitch = quad ? qpitch_for(G) : 0;
    if (quad) m_q.reserve((v.nchans + 1) * qpitch * 4);
    for (size_t b = 0; b < nbuf; ++b) {
        if (!dev_out) m_out[b].reserve(ndm * G * ob);
        if (!dev_in) m_stage[b].reserve(in_bytes_for(G));
    }

    cudaStream_t ex = m_gpu.stream();
    cudaStream_t h2d = m_gpu.h2d->get();
    cudaStream_t d2h = m_gpu.d2h->get();
    uint32_t* tr = m_tr.get<uint32_t>();
    if (quad) {
        m_err.reserve(sizeof(unsigned));
        RT_CHECK(cudaMemsetAsync(m_err.get(), 0, sizeof(unsigned), ex));
    }

    const float in_range = (float)(nbits == 32 ? 0xFFFFFFFFu : ((1u << nbits) - 1u));
    const float den = in_range * (float)v.nchans;
    const float factor = 3.f * 1024.f / 255.f / 16.f;

    // The last gulp's K2 runs per group of DM slots whose output rows are
    // contiguous, so that its device-to-host copy starts group by group
    // (every other gulp's copy already overlaps the next gulp's kernels, and
    // each extra launch ends with a partly filled wave).
    const size_t bd = s.tiled ? (size_t)kern::tiled_block_dms(nbits, s.variant) : 32;
    const size_t ntile = (ndm + bd - 1) / bd;
    const size_t ngroups_last = (!dev_out && s.identity) ? std::min<size_t>(kMaxOutGroups, ntile) : 1;

    // Gulps (first output sample, samples). With host input and several
    // gulps the first is a quarter of G: its input copy is the one that no
    // kernel hides, and the next gulp's copy runs during its kernels.
    std::vector<std::pair<size_t, size_t>> gulps;
    for (size_t g0 = 0; g0 < nsamp_out;) {
        size_t gc = std::min(G, nsamp_out - g0);
        if (g0 == 0 && !dev_in && gc < nsamp_out && G >= 4 * bt) gc = round_up(G / 4, bt);
        gulps.emplace_back(g0, gc);
        g0 += gc;
    }

    std::unique_ptr<rt::Event> t_a, t_b, t_c;
    if (record_timing) {
        t_a.reset(new rt::Event(true));
        t_b.reset(new rt::Event(true));
        t_c.reset(new rt::Event(true));
    }

    size_t ev = 0;
    rt::Event* ev_in_free[2] = {&event(ev++), &event(ev++)};   // K1 has read input buffer b
    rt::Event* ev_out_free[2] = {&event(ev++), &event(ev++)};  // D2H has read output buffer b
    bool in_used[2] = {false, false}, out_used[2] = {false, false};

    for (size_t gi = 0; gi < gulps.size(); ++gi) {
        const size_t g0 = gulps[gi].first, gc = gulps[gi].second;
        const bool last = gi + 1 == gulps.size();
        const size_t ngroups = last ? ngroups_last : 1;
        const size_t b = gi % nbuf;
        const size_t rows_need = gc + s.tmax;
        const size_t rows_avail = std::min(rows_need, c.nsamps - g0);

        if (t_a && g0 == 0) t_a->record(ex);
        // Padding channel row (all zero).
        if (quad) RT_CHECK(cudaMemsetAsync(m_q.get<uint32_t>() + v.nchans * qpitch, 0, qpitch * 4, ex));
        else RT_CHECK(cudaMemsetAsync(tr + v.nchans * pitch, 0, pitch * 4, ex));

        // K1 (channel-major packed) or K1d (quad-strided rows) from the
        // gulp's input rows, zero past the data.
        const uint8_t* rows = c.in + g0 * c.in_stride;
        size_t rows_pitch = c.in_stride;
        if (!dev_in) {
            // the whole gulp's rows into input buffer b, on the copy stream
            if (in_used[b]) RT_CHECK(cudaStreamWaitEvent(h2d, *ev_in_free[b], 0));
            RT_CHECK(cudaMemcpy2DAsync(m_stage[b].get(), row_bytes, rows, c.in_stride, row_bytes, rows_avail,
                                       cudaMemcpyHostToDevice, h2d));
            rt::Event& ready = event(ev++);
            ready.record(h2d);
            RT_CHECK(cudaStreamWaitEvent(ex, ready, 0));
            rows = m_stage[b].get<uint8_t>();
            rows_pitch = row_bytes;
        }
        if (quad) {
            kern::QuadDirectArgs qa{rows, rows_pitch, rows_avail, v.nchans, nbits, m_q.get<uint32_t>(), qpitch,
                                    s.period};
            kern::launch_quad_direct(qa, ex);
        } else {
            kern::TransposeArgs ta{rows, rows_pitch, rows_avail, v.nchans, nbits, tr, pitch, 0, pitch};
            kern::launch_transpose(ta, ex);
        }
        ++stats.launches;
        if (!dev_in) {
            ev_in_free[b]->record(ex);
            in_used[b] = true;
        }
        if (t_b && g0 == 0) t_b->record(ex);

        // K2 per DM group.
        if (!dev_out && out_used[b]) RT_CHECK(cudaStreamWaitEvent(ex, *ev_out_free[b], 0));
        const size_t out_elems_stride = dev_out ? c.out_stride / ob : gc;
        uint8_t* out_base = dev_out ? c.out + g0 * ob : m_out[b].get<uint8_t>();
        std::vector<std::pair<size_t, size_t>> groups;
        for (size_t gr = 0; gr < ngroups; ++gr) {
            const size_t t0 = ntile * gr / ngroups, t1 = ntile * (gr + 1) / ngroups;
            const size_t s0 = t0 * bd, s1 = std::min(ndm, t1 * bd);
            if (s0 >= s1) continue;
            groups.emplace_back(s0, s1);
            kern::DedisperseArgs da{};
            da.tr = quad ? m_q.get<uint32_t>() : tr;
            da.tr_pitch_words = quad ? qpitch : pitch;
            da.nbits = nbits;
            da.nchans = v.nchans;
            da.chan_list = m_chan.get<int32_t>();
            da.nact = s.nact;
            da.nstages = s.nstages;
            da.km_vals = m_km.get<uint32_t>();
            da.delay_table = m_gpu.delay_table.get<float>();
            da.chan_delay = m_cdl.get<float>();
            da.dms = m_dms.get<float>() + s0;
            da.ndm = (int)(s1 - s0);
            da.nsamp_out = gc;
            da.out_stride = out_elems_stride;
            da.out_nbits = c.out_nbits;
            da.den = den;
            da.factor = factor;
            da.win_words = s.win_words;
            da.chan_per_stage = s.chan_per_stage;
            da.variant = s.variant;
            da.err = m_err.get<unsigned>();
            if (s.identity) {
                da.perm = nullptr;
                da.out = out_base + s0 * out_elems_stride * ob;
            } else {
                da.perm = m_perm.get<int32_t>() + s0;
                da.out = out_base;
            }
            if (s.tiled) kern::launch_dedisperse_tiled(da, ex);
            else kern::launch_dedisperse_plain(da, ex);
            ++stats.launches;
            if (!dev_out) event(ev + groups.size() - 1).record(ex);
        }
        if (t_c && last) t_c->record(ex);

        // D2H per group into the caller's rows (column offset g0).
        if (!dev_out) {
            for (size_t gr = 0; gr < groups.size(); ++gr) {
                const size_t s0 = groups[gr].first, s1 = groups[gr].second;
                const size_t r0 = s.identity ? s0 : 0, nrow = s.identity ? s1 - s0 : ndm;
                RT_CHECK(cudaStreamWaitEvent(d2h, event(ev + gr), 0));
                if (!s.identity && gr + 1 < groups.size()) continue;
                RT_CHECK(cudaMemcpy2DAsync(c.out + r0 * c.out_stride + g0 * ob, c.out_stride,
                                           m_out[b].get<uint8_t>() + r0 * gc * ob, gc * ob, gc * ob,
                                           nrow, cudaMemcpyDeviceToHost, d2h));
            }
            ev += groups.size();
            ev_out_free[b]->record(d2h);
            out_used[b] = true;
        }
    }

    const bool async = (c.flags & DEDISP_ASYNC) && dev_in;
    if (!async) {
        RT_CHECK(cudaStreamSynchronize(ex));
        if (!dev_out) RT_CHECK(cudaStreamSynchronize(d2h));
        if (quad && kern::read_error_word(m_err.get<unsigned>(), ex))
            DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "a staged window copy did not complete");
    }
    if (record_timing) {
        RT_CHECK(cudaEventSynchronize(*t_c));
        RT_CHECK(cudaEventElapsedTime(&stats.transpose_ms, *t_a, *t_b));
        RT_CHECK(cudaEventElapsedTime(&stats.kernel_ms, *t_b, *t_c));
    }
}

}  // namespace detail
}  // namespace dedisp
