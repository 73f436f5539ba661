// Batched multi-beam TDD (see batch.hpp).
#include "batch.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

#include "dedisp_b200.h"
#include "errors.hpp"
#include "host_math.hpp"

namespace dedisp {
namespace detail {

namespace {
size_t round_up(size_t a, size_t b) { return (a + b - 1) / b * b; }
constexpr size_t kTuneSamples = 8192;  // leading samples per beam timed by autotune()
constexpr int kMaxStageChannels = 32;
}  // namespace

struct TddBatch::BeamState {
    BatchBeamSpec spec;
    std::vector<float> sorted;   // ascending DMs (NaN first)
    std::vector<int32_t> perm;   // output row of each sorted slot; empty: identity
    size_t max_delay = 0;        // reference rule: last DM of the list x last channel
    size_t nout = 0;
    uint32_t tmax = 0;           // largest delay over active channels and DMs
    size_t dm_off = 0;           // offset in the concatenated device DM / perm arrays
};

struct TddBatch::Layout {
    BatchShape shape;
    bool tiled = false;
    bool persistent = false;
    std::vector<kern::DedisperseArgs> args;   // host copy (device pointers)
    std::vector<size_t> tr_off;               // words into the workspace
    std::vector<size_t> pitch;                // words per channel row
    bool quad = false;                        // quad-strided rows (8-bit quad variants)
    int period = 0;                           // quad: P words
    std::vector<size_t> q_off;                // quad: rows' offset in the workspace (words)
    std::vector<size_t> qpitch;               // quad: words per row
    uint32_t* ws = nullptr;                   // workspace the args point into (upload)
    std::vector<int> nbx;
    std::vector<unsigned long long> start;    // nbeams + 1
    std::vector<size_t> units;                // DM trials x samples covered per beam
    size_t smem = 0;
    size_t ws_words = 0;
};

TddBatch::TddBatch(size_t nchans, float dt, float f0, float df, int in_nbits, int out_nbits,
                   int device)
    : m_nchans(nchans), m_nbits(in_nbits), m_out_nbits(out_nbits), m_device(device)
{
    if (nchans == 0) DD_THROW_MSG(DEDISP_INVALID_PLAN, "nchans must be positive");
    if (in_nbits != 1 && in_nbits != 2 && in_nbits != 4 && in_nbits != 8 && in_nbits != 16 &&
        in_nbits != 32)
        DD_THROW(DEDISP_UNSUPPORTED_IN_NBITS);
    if (out_nbits != 8 && out_nbits != 16 && out_nbits != 32) DD_THROW(DEDISP_UNSUPPORTED_OUT_NBITS);
    if ((nchans * (size_t)in_nbits) % 32 != 0)
        DD_THROW_MSG(DEDISP_INVALID_STRIDE, "nchans * in_nbits must be a multiple of 32");
    if (nchans > 8192) DD_THROW(DEDISP_NCHANS_EXCEEDS_LIMIT);
    m_shape.variant = kern::tiled_default_variant(in_nbits);
    m_delays.assign(nchans + 1, 0.f);
    hostmath::delay_table(nchans, dt, f0, df, m_delays.data());
    set_killmask(nullptr);
    rt::DeviceGuard g(m_device);
    for (auto& e : m_ev) e.reset(new rt::Event(true));
    m_d_delay.reserve(m_delays.size() * 4);
    m_d_err.reserve(sizeof(unsigned));
    RT_CHECK(cudaMemset(m_d_err.get(), 0, sizeof(unsigned)));
    RT_CHECK(cudaMemcpy(m_d_delay.get(), m_delays.data(), m_delays.size() * 4, cudaMemcpyHostToDevice));
}

TddBatch::~TddBatch()
{
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != m_device) cudaSetDevice(m_device);
    cudaDeviceSynchronize();
    drop_graph();
}

void TddBatch::drop_graph()
{
    if (m_exec) cudaGraphExecDestroy(m_exec);
    if (m_graph) cudaGraphDestroy(m_graph);
    m_exec = nullptr;
    m_graph = nullptr;
}

void TddBatch::set_killmask(const int32_t* killmask)
{
    m_km.assign(m_nchans, 1);
    if (killmask) std::copy(killmask, killmask + m_nchans, m_km.begin());
    m_chan.clear();
    m_kmv.clear();
    m_general_mask = false;
    for (size_t c = 0; c < m_nchans; ++c) {
        if (m_km[c] == 0) continue;
        if (m_km[c] != 1) m_general_mask = true;
        m_chan.push_back((int32_t)c);
        m_kmv.push_back((uint32_t)m_km[c]);
    }
    // Channel list padded with the all-zero row `nchans` up to any stage size.
    std::vector<int32_t> padded(m_chan);
    padded.resize(round_up(std::max<size_t>(m_chan.size(), 1), kMaxStageChannels) + kMaxStageChannels,
                  (int32_t)m_nchans);
    std::vector<float> cdl(padded.size());  // delay of each list entry
    for (size_t j = 0; j < padded.size(); ++j) cdl[j] = m_delays[padded[j]];
    rt::DeviceGuard g(m_device);
    m_d_chan.reserve(padded.size() * 4);
    RT_CHECK(cudaMemcpy(m_d_chan.get(), padded.data(), padded.size() * 4, cudaMemcpyHostToDevice));
    m_d_cdl.reserve(cdl.size() * 4);
    RT_CHECK(cudaMemcpy(m_d_cdl.get(), cdl.data(), cdl.size() * 4, cudaMemcpyHostToDevice));
    m_d_kmv.reserve(std::max<size_t>(m_kmv.size(), 1) * 4);
    if (!m_kmv.empty())
        RT_CHECK(cudaMemcpy(m_d_kmv.get(), m_kmv.data(), m_kmv.size() * 4, cudaMemcpyHostToDevice));
    // beams depend on the active channels (largest delay)
    if (!m_beams.empty()) {
        std::vector<BatchBeamSpec> specs;
        for (auto& b : m_beams) specs.push_back(b.spec);
        set_beams(std::move(specs));
    }
    m_dirty = true;
}

void TddBatch::set_beams(std::vector<BatchBeamSpec> beams)
{
    const size_t ob = (size_t)m_out_nbits / 8;
    const size_t row_bytes = m_nchans * (size_t)m_nbits / 8;
    std::vector<BeamState> st(beams.size());
    size_t dm_total = 0;
    for (size_t b = 0; b < beams.size(); ++b) {
        BatchBeamSpec& s = beams[b];
        BeamState& t = st[b];
        if (!s.in || !s.out) DD_THROW_MSG(DEDISP_INVALID_POINTER, "beam input/output pointer is null");
        if (s.dms.empty()) DD_THROW(DEDISP_NO_DM_LIST_SET);
        if (s.in_stride < row_bytes) DD_THROW(DEDISP_INVALID_STRIDE);
        t.max_delay = hostmath::max_delay(s.dms.back(), m_delays[m_nchans - 1]);
        if (s.nsamps < t.max_delay) DD_THROW(DEDISP_TOO_FEW_NSAMPS);
        t.nout = s.nsamps - t.max_delay;
        if (s.out_stride < t.nout * ob || s.out_stride % ob != 0) DD_THROW(DEDISP_INVALID_STRIDE);
        std::vector<int32_t> order(s.dms.size());
        std::iota(order.begin(), order.end(), 0);
        auto key = [&](int32_t i) { return std::isnan(s.dms[i]) ? -INFINITY : s.dms[i]; };
        const bool identity =
            std::is_sorted(order.begin(), order.end(), [&](int32_t x, int32_t y) { return key(x) < key(y); });
        if (!identity)
            std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return key(x) < key(y); });
        t.sorted.resize(s.dms.size());
        for (size_t i = 0; i < s.dms.size(); ++i) t.sorted[i] = s.dms[order[i]];
        if (!identity) t.perm = order;
        for (int32_t c : m_chan) {
            const float dl = m_delays[c];
            t.tmax = std::max(t.tmax, std::max(hostmath::delay_rn(t.sorted.front(), dl),
                                               hostmath::delay_rn(t.sorted.back(), dl)));
        }
        t.dm_off = dm_total;
        dm_total += s.dms.size();
        t.spec = std::move(s);
    }
    rt::DeviceGuard g(m_device);
    std::vector<float> dms(std::max<size_t>(dm_total, 1), 0.f);
    std::vector<int32_t> perm(std::max<size_t>(dm_total, 1), 0);
    for (auto& t : st) {
        std::copy(t.sorted.begin(), t.sorted.end(), dms.begin() + t.dm_off);
        std::copy(t.perm.begin(), t.perm.end(), perm.begin() + t.dm_off);
    }
    m_d_dms.reserve(dms.size() * 4);
    m_d_perm.reserve(perm.size() * 4);
    RT_CHECK(cudaMemcpy(m_d_dms.get(), dms.data(), dms.size() * 4, cudaMemcpyHostToDevice));
    RT_CHECK(cudaMemcpy(m_d_perm.get(), perm.data(), perm.size() * 4, cudaMemcpyHostToDevice));
    m_beams = std::move(st);
    m_dirty = true;
}

void TddBatch::set_shape(const BatchShape& shape)
{
    const int nv = kern::tiled_batch_variant_count(m_nbits);
    if (shape.variant < 0 || shape.variant >= nv) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "unknown tile-shape variant");
    if (shape.chan_per_stage < 0 || shape.chan_per_stage > kMaxStageChannels || shape.chan_per_stage % 2)
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "channels per stage must be even and at most 32");
    m_shape = shape;
    m_dirty = true;
}

size_t TddBatch::max_delay(size_t beam) const { return m_beams.at(beam).max_delay; }
size_t TddBatch::nsamp_out(size_t beam) const { return m_beams.at(beam).nout; }

TddBatch::Layout TddBatch::make_layout(const BatchShape& shape, size_t tile_limit) const
{
    Layout L;
    L.shape = shape;
    const int nb = m_nbits, v = shape.variant;
    const int spw = 32 / nb;
    const bool want_tiled = !m_general_mask;
    const size_t bd = (size_t)kern::tiled_block_dms(nb, v);
    const size_t bt = (size_t)kern::tiled_block_samples(nb, v);
    const int J = kern::tiled_lane_words(nb, v);
    const bool quad = want_tiled && kern::tiled_variant_quad(nb, v);
    const size_t nbeams = m_beams.size();
    L.args.resize(nbeams);
    L.tr_off.resize(nbeams);
    L.pitch.resize(nbeams);
    L.q_off.assign(nbeams, 0);
    L.qpitch.assign(nbeams, 0);
    L.period = 32 * J;
    L.nbx.resize(nbeams);
    L.units.resize(nbeams);
    L.start.assign(nbeams + 1, 0);
    // Tiled layout first; any beam whose window does not fit shared memory
    // sends the whole batch to the plain kernel.
    std::vector<int> W(nbeams, 0), CS(nbeams, 0);
    bool tiled = want_tiled;
    for (size_t b = 0; b < nbeams && tiled; ++b) {
        const BeamState& t = m_beams[b];
        uint32_t span = 0;
        for (size_t i = 0; i < t.sorted.size(); i += bd) {
            const float f = t.sorted[i], l = t.sorted[std::min(i + bd, t.sorted.size()) - 1];
            for (int32_t c : m_chan) {
                const uint32_t x = hostmath::delay_rn(f, m_delays[c]), y = hostmath::delay_rn(l, m_delays[c]);
                span = std::max(span, x > y ? x - y : y - x);
            }
        }
        // quad-strided rows: a 1-sample delay is a 1-word offset
        const size_t w = quad ? round_up((size_t)span + 3 + 32 * (size_t)J, 4)
                              : round_up((span + 4 * (size_t)spw - 1) / spw + 32 * (size_t)J + 1, 4);
        const int fit = w > ((size_t)1 << 26) ? 0 : kern::tiled_stage_channels(nb, (int)w, v);
        if (fit < 2) { tiled = false; break; }
        W[b] = (int)w;
        CS[b] = shape.chan_per_stage > 0 ? std::min(shape.chan_per_stage, fit) : fit;
    }
    L.tiled = tiled;
    L.persistent = tiled && (nb == 8 || quad);
    L.quad = tiled && quad;
    const size_t ubt = tiled ? bt : 16, ubd = tiled ? bd : 32;
    const float in_range = (float)(nb == 32 ? 0xFFFFFFFFu : ((1u << nb) - 1u));
    size_t off = 0;
    for (size_t b = 0; b < nbeams; ++b) {
        const BeamState& t = m_beams[b];
        const size_t win = tiled ? (size_t)W[b] : 0;
        L.pitch[b] = round_up((round_up(std::max<size_t>(t.nout, 1), ubt) + t.tmax + spw - 1) / spw + win + 8, 32);
        // quad-strided rows are built straight from the input (K1d); the
        // channel-major packed copy exists only for the other forms
        L.tr_off[b] = off;
        if (!L.quad) off += round_up((m_nchans + 1) * L.pitch[b], 64);
        if (L.quad) {
            // the tile windows read up to word (tiles - 1) * bt + tmax + P + 2
            L.qpitch[b] = round_up(round_up(std::max<size_t>(t.nout, 1), ubt) + t.tmax + L.period + 4, 32);
            L.q_off[b] = off;
            off += round_up((m_nchans + 1) * L.qpitch[b], 64);
        }
        kern::DedisperseArgs& a = L.args[b];
        a = kern::DedisperseArgs{};
        a.tr_pitch_words = L.quad ? L.qpitch[b] : L.pitch[b];
        a.nbits = nb;
        a.nchans = m_nchans;
        a.nact = (int)m_chan.size();
        a.ndm = (int)t.sorted.size();
        a.nsamp_out = t.nout;
        a.out_stride = t.spec.out_stride / ((size_t)m_out_nbits / 8);
        a.out_nbits = m_out_nbits;
        a.den = in_range * (float)m_nchans;
        a.factor = 3.f * 1024.f / 255.f / 16.f;
        a.win_words = tiled ? W[b] : 0;
        a.chan_per_stage = tiled ? CS[b] : 0;
        a.nstages = tiled ? std::max(1, ((int)m_chan.size() + CS[b] - 1) / CS[b]) : 0;
        a.variant = tiled ? v : 0;
        const size_t nbx = (t.sorted.size() + ubd - 1) / ubd;
        size_t nby = (t.nout + ubt - 1) / ubt;
        size_t covered = t.nout;
        if (tile_limit) {
            nby = std::min(nby, (tile_limit + ubt - 1) / ubt);
            covered = std::min(t.nout, nby * ubt);
        }
        L.nbx[b] = (int)nbx;
        L.units[b] = t.sorted.size() * covered;
        L.start[b + 1] = L.start[b] + (unsigned long long)(nbx * nby);
        if (tiled) L.smem = std::max(L.smem, kern::tiled_batch_smem_bytes(nb, W[b], CS[b], v));
    }
    L.ws_words = off;
    return L;
}

size_t TddBatch::workspace_bytes() const
{
    size_t words = 0;
    for (int v = 0; v < kern::tiled_batch_variant_count(m_nbits); ++v) {
        BatchShape s;
        s.variant = v;
        words = std::max(words, make_layout(s, 0).ws_words);
    }
    return std::max<size_t>(words, 64) * 4;
}

void TddBatch::set_workspace(void* ptr, size_t bytes)
{
    if (ptr && bytes < workspace_bytes()) DD_THROW_MSG(DEDISP_MEM_ALLOC_FAILED, "workspace too small");
    m_ext_ws = ptr;
    m_ext_ws_bytes = ptr ? bytes : 0;
    m_dirty = true;
}

uint8_t* TddBatch::workspace_base()
{
    if (m_ext_ws) return static_cast<uint8_t*>(m_ext_ws);
    m_own_ws.reserve(workspace_bytes());
    return m_own_ws.get<uint8_t>();
}

void TddBatch::upload(Layout& L)
{
    rt::DeviceGuard g(m_device);
    uint32_t* ws = reinterpret_cast<uint32_t*>(workspace_base());
    std::vector<kern::DedisperseArgs> args(L.args);
    for (size_t b = 0; b < m_beams.size(); ++b) {
        const BeamState& t = m_beams[b];
        kern::DedisperseArgs& a = args[b];
        a.tr = ws + (L.quad ? L.q_off[b] : L.tr_off[b]);
        a.chan_list = m_d_chan.get<int32_t>();
        a.chan_delay = m_d_cdl.get<float>();
        a.km_vals = m_d_kmv.get<uint32_t>();
        a.delay_table = m_d_delay.get<float>();
        a.dms = m_d_dms.get<float>() + t.dm_off;
        a.perm = t.perm.empty() ? nullptr : m_d_perm.get<int32_t>() + t.dm_off;
        a.out = t.spec.out;
        a.err = m_d_err.get<unsigned>();
    }
    L.args = args;
    L.ws = ws;
    const size_t nb = std::max<size_t>(m_beams.size(), 1);
    m_d_args.reserve(nb * sizeof(kern::DedisperseArgs));
    m_d_start.reserve((nb + 1) * sizeof(unsigned long long));
    m_d_nbx.reserve(nb * sizeof(int));
    if (!m_beams.empty()) {
        RT_CHECK(cudaMemcpy(m_d_args.get(), args.data(), args.size() * sizeof(kern::DedisperseArgs),
                            cudaMemcpyHostToDevice));
        RT_CHECK(cudaMemcpy(m_d_nbx.get(), L.nbx.data(), L.nbx.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    RT_CHECK(cudaMemcpy(m_d_start.get(), L.start.data(), L.start.size() * sizeof(unsigned long long),
                        cudaMemcpyHostToDevice));
}

void TddBatch::enqueue(cudaStream_t s, const Layout& L, bool timing)
{
    int launches = 0;
    if (timing) m_ev[0]->record(s);  // never inside a stream capture (see execute)
    if (L.quad) RT_CHECK(cudaMemsetAsync(m_d_err.get(), 0, sizeof(unsigned), s));
    for (size_t b = 0; b < m_beams.size(); ++b) {
        const BeamState& t = m_beams[b];
        if (t.nout == 0) continue;
        uint32_t* ws = L.ws;
        const size_t rows = std::min(t.nout + t.tmax, t.spec.nsamps);
        if (L.quad) {
            // K1d: quad-strided rows and the zero padding row
            uint32_t* q = ws + L.q_off[b];
            RT_CHECK(cudaMemsetAsync(q + m_nchans * L.qpitch[b], 0, L.qpitch[b] * 4, s));
            kern::QuadDirectArgs qa{t.spec.in, t.spec.in_stride, rows, m_nchans, m_nbits, q, L.qpitch[b],
                                    L.period};
            kern::launch_quad_direct(qa, s);
        } else {
            uint32_t* tr = ws + L.tr_off[b];
            RT_CHECK(cudaMemsetAsync(tr + m_nchans * L.pitch[b], 0, L.pitch[b] * 4, s));
            kern::TransposeArgs ta{t.spec.in, t.spec.in_stride, rows, m_nchans, m_nbits, tr, L.pitch[b], 0,
                                   L.pitch[b]};
            kern::launch_transpose(ta, s);
        }
        ++launches;
    }
    if (timing) m_ev[1]->record(s);
    if (L.persistent) {
        kern::BatchLaunch bl{m_d_args.get<kern::DedisperseArgs>(), m_d_start.get<unsigned long long>(),
                             m_d_nbx.get<int>(), (int)m_beams.size(), L.start.back(), L.smem};
        kern::launch_dedisperse_tiled_batch(bl, m_nbits, L.shape.variant, s);
        ++launches;
    } else {
        for (size_t b = 0; b < m_beams.size(); ++b) {
            if (m_beams[b].nout == 0) continue;
            if (L.tiled) kern::launch_dedisperse_tiled(L.args[b], s);
            else kern::launch_dedisperse_plain(L.args[b], s);
            ++launches;
        }
    }
    if (timing) m_ev[2]->record(s);
    last_launches = launches;
}

void TddBatch::sync(cudaStream_t stream)
{
    rt::DeviceGuard g(m_device);
    RT_CHECK(cudaStreamSynchronize(stream));
    if (kern::read_error_word(m_d_err.get<unsigned>(), stream))
        DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "a staged window copy did not complete");
}

BatchShape TddBatch::autotune(cudaStream_t stream)
{
    rt::DeviceGuard g(m_device);
    if (m_beams.empty()) return m_shape;
    std::vector<BatchShape> cands;
    const int nv = m_general_mask ? 1 : kern::tiled_batch_variant_count(m_nbits);
    for (int v = 0; v < nv; ++v)
        for (int cs : {0, 24, 16}) {
            // quad-strided blocks size their stages themselves
            if (cs && kern::tiled_variant_quad(m_nbits, v)) continue;
            BatchShape s;
            s.variant = v;
            s.chan_per_stage = cs;
            cands.push_back(s);
        }
    double best = std::numeric_limits<double>::infinity();
    BatchShape best_shape = m_shape;
    std::vector<int> fit_cs;  // stage sizes of the current variant's largest-fit layout
    for (const BatchShape& c : cands) {
        Layout L = make_layout(c, kTuneSamples);
        std::vector<int> cs;
        for (auto& a : L.args) cs.push_back(a.chan_per_stage);
        if (c.chan_per_stage == 0) fit_cs = cs;
        else if (cs == fit_cs) continue;  // same stage sizes as the largest fit: already timed
        upload(L);
        float ms = 0.f;
        for (int rep = 0; rep < 2; ++rep) {
            enqueue(stream, L, true);
            RT_CHECK(cudaEventSynchronize(m_ev[2]->get()));
            RT_CHECK(cudaEventElapsedTime(&ms, m_ev[1]->get(), m_ev[2]->get()));
        }
        double units = 0;
        for (size_t u : L.units) units += (double)u;
        const double cost = ms / std::max(units, 1.0);
        if (cost < best) {
            best = cost;
            best_shape = c;
        }
        if (!L.tiled) break;  // plain form: nothing to tune
    }
    m_shape = best_shape;
    m_dirty = true;
    return m_shape;
}

void TddBatch::execute(cudaStream_t stream, bool use_graph)
{
    rt::DeviceGuard g(m_device);
    if (m_beams.empty()) return;
    if (m_dirty || !m_layout) {
        drop_graph();
        m_layout.reset(new Layout(make_layout(m_shape, 0)));
        upload(*m_layout);
        m_dirty = false;
    }
    if (!use_graph) {
        enqueue(stream, *m_layout, record_timing);
    } else {
        // The graph holds no event records (elapsed time between events
        // recorded by graph nodes is not available); with timing on, events
        // bracket the whole graph launch instead.
        if (!m_exec) {
            rt::Stream cap;
            RT_CHECK(cudaStreamBeginCapture(cap.get(), cudaStreamCaptureModeRelaxed));
            try {
                enqueue(cap.get(), *m_layout, false);
            } catch (...) {
                cudaGraph_t gph = nullptr;
                cudaStreamEndCapture(cap.get(), &gph);
                if (gph) cudaGraphDestroy(gph);
                throw;
            }
            RT_CHECK(cudaStreamEndCapture(cap.get(), &m_graph));
            RT_CHECK(cudaGraphInstantiate(&m_exec, m_graph, 0));
            m_graph_launches = last_launches;
        }
        if (record_timing) m_ev[1]->record(stream);
        RT_CHECK(cudaGraphLaunch(m_exec, stream));
        if (record_timing) m_ev[2]->record(stream);
        last_launches = m_graph_launches;
    }
    if (record_timing) {
        RT_CHECK(cudaEventSynchronize(m_ev[2]->get()));
        if (m_layout->quad && kern::read_error_word(m_d_err.get<unsigned>(), stream))
            DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "a staged window copy did not complete");
        if (use_graph) last_k1_ms = -1.f;  // transposes are inside the graph
        else RT_CHECK(cudaEventElapsedTime(&last_k1_ms, m_ev[0]->get(), m_ev[1]->get()));
        RT_CHECK(cudaEventElapsedTime(&last_k2_ms, m_ev[1]->get(), m_ev[2]->get()));
    }
}

}  // namespace detail
}  // namespace dedisp

// ---------------------------------------------------------------------------
// C interface (include/dedisp_b200.h). Errors are returned with their
// specific code; dedisp_b200_last_error is not involved.
// ---------------------------------------------------------------------------
struct dedisp_b200_batch_struct {
    std::unique_ptr<dedisp::detail::TddBatch> b;
};

namespace dedisp {
void note_last_error(dedisp_error code, const char* msg);
}

namespace {
template <typename F>
dedisp_error batch_call(dedisp_b200_batch batch, F&& fn)
{
    if (!batch || !batch->b) return DEDISP_INVALID_PLAN;
    try {
        fn(*batch->b);
        return DEDISP_NO_ERROR;
    } catch (const dedisp::Error& e) {
        dedisp::note_last_error(e.code(), e.what());
        return e.code();
    } catch (const std::exception& e) {
        dedisp::note_last_error(DEDISP_UNKNOWN_ERROR, e.what());
        return DEDISP_UNKNOWN_ERROR;
    } catch (...) {
        return DEDISP_UNKNOWN_ERROR;
    }
}
}  // namespace

extern "C" {

dedisp_error dedisp_b200_batch_create(dedisp_b200_batch* batch, dedisp_size nchans, dedisp_float dt,
                                      dedisp_float f0, dedisp_float df, dedisp_size in_nbits,
                                      dedisp_size out_nbits, int device)
{
    if (!batch) return DEDISP_INVALID_POINTER;
    *batch = nullptr;
    try {
        auto* h = new dedisp_b200_batch_struct;
        try {
            h->b.reset(new dedisp::detail::TddBatch(nchans, dt, f0, df, (int)in_nbits, (int)out_nbits, device));
        } catch (...) {
            delete h;
            throw;
        }
        *batch = h;
        return DEDISP_NO_ERROR;
    } catch (const dedisp::Error& e) {
        dedisp::note_last_error(e.code(), e.what());
        return e.code();
    } catch (...) {
        return DEDISP_UNKNOWN_ERROR;
    }
}

void dedisp_b200_batch_destroy(dedisp_b200_batch batch)
{
    try {
        delete batch;
    } catch (...) {
    }
}

dedisp_error dedisp_b200_batch_set_killmask(dedisp_b200_batch batch, const dedisp_bool* killmask)
{
    return batch_call(batch, [&](dedisp::detail::TddBatch& b) {
        b.set_killmask(reinterpret_cast<const int32_t*>(killmask));
    });
}

dedisp_error dedisp_b200_batch_set_beams(dedisp_b200_batch batch, const dedisp_b200_beam* beams,
                                         dedisp_size nbeams)
{
    if (nbeams && !beams) return DEDISP_INVALID_POINTER;
    return batch_call(batch, [&](dedisp::detail::TddBatch& b) {
        std::vector<dedisp::detail::BatchBeamSpec> v(nbeams);
        for (size_t i = 0; i < nbeams; ++i) {
            const dedisp_b200_beam& s = beams[i];
            if (s.dm_count && !s.dm_list) DD_THROW(DEDISP_INVALID_POINTER);
            v[i].in = s.in;
            v[i].in_stride = s.in_stride;
            v[i].nsamps = s.nsamps;
            v[i].dms.assign(s.dm_list, s.dm_list + s.dm_count);
            v[i].out = s.out;
            v[i].out_stride = s.out_stride;
        }
        b.set_beams(std::move(v));
    });
}

dedisp_size dedisp_b200_batch_workspace_size(dedisp_b200_batch batch)
{
    dedisp_size n = 0;
    if (batch_call(batch, [&](dedisp::detail::TddBatch& b) { n = b.workspace_bytes(); }) != DEDISP_NO_ERROR)
        return 0;
    return n;
}

dedisp_error dedisp_b200_batch_set_workspace(dedisp_b200_batch batch, void* d_workspace, dedisp_size bytes)
{
    return batch_call(batch, [&](dedisp::detail::TddBatch& b) { b.set_workspace(d_workspace, bytes); });
}

int dedisp_b200_batch_variant_count(dedisp_size in_nbits)
{
    return dedisp::kern::tiled_batch_variant_count((int)in_nbits);
}

dedisp_error dedisp_b200_batch_set_shape(dedisp_b200_batch batch, int variant, int chan_per_stage)
{
    return batch_call(batch, [&](dedisp::detail::TddBatch& b) {
        dedisp::detail::BatchShape s;
        s.variant = variant;
        s.chan_per_stage = chan_per_stage;
        b.set_shape(s);
    });
}

dedisp_error dedisp_b200_batch_autotune(dedisp_b200_batch batch, void* stream, int* variant,
                                        int* chan_per_stage)
{
    return batch_call(batch, [&](dedisp::detail::TddBatch& b) {
        const dedisp::detail::BatchShape s = b.autotune(static_cast<cudaStream_t>(stream));
        if (variant) *variant = s.variant;
        if (chan_per_stage) *chan_per_stage = s.chan_per_stage;
    });
}

dedisp_error dedisp_b200_batch_execute(dedisp_b200_batch batch, void* stream, int use_graph)
{
    return batch_call(batch, [&](dedisp::detail::TddBatch& b) {
        b.execute(static_cast<cudaStream_t>(stream), use_graph != 0);
    });
}

dedisp_error dedisp_b200_batch_sync(dedisp_b200_batch batch, void* stream)
{
    return batch_call(batch, [&](dedisp::detail::TddBatch& b) { b.sync(static_cast<cudaStream_t>(stream)); });
}

dedisp_error dedisp_b200_batch_set_timing(dedisp_b200_batch batch, int enable)
{
    return batch_call(batch, [&](dedisp::detail::TddBatch& b) { b.record_timing = enable != 0; });
}

dedisp_error dedisp_b200_batch_get_timing(dedisp_b200_batch batch, float* transpose_ms,
                                          float* dedisperse_ms, int* launches)
{
    return batch_call(batch, [&](dedisp::detail::TddBatch& b) {
        if (transpose_ms) *transpose_ms = b.last_k1_ms;
        if (dedisperse_ms) *dedisperse_ms = b.last_k2_ms;
        if (launches) *launches = b.last_launches;
    });
}

dedisp_size dedisp_b200_batch_max_delay(dedisp_b200_batch batch, dedisp_size beam)
{
    dedisp_size n = 0;
    if (batch_call(batch, [&](dedisp::detail::TddBatch& b) { n = b.max_delay(beam); }) != DEDISP_NO_ERROR)
        return 0;
    return n;
}

}  // extern "C"
