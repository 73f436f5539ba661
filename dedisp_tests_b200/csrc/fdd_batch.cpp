// Batched multi-beam FDD (see fdd_batch.hpp).
#include "fdd_batch.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "dedisp_b200.h"
#include "host_math.hpp"

namespace dedisp {
namespace detail {

namespace {
size_t round_up(size_t a, size_t b) { return (a + b - 1) / b * b; }
constexpr size_t kAlign = 256;
}  // namespace

struct FddBatch::Beam {
    FddBeamSpec spec;
    size_t max_delay = 0, nout = 0;
    FddGeometry g;
    bool qpath = false;
    kern::BinMap bmap;
    size_t bin_pitch = 0, x_len = 0, seg_stride = 0;
    int dmax = -1;      // largest delay index (trunc), -1 if a DM is negative
    kern::TcSource src;  // phasor source of the tensor-core MAC
    int npad = 0, ngroups = 0;
    size_t b_bytes = 0;  // one segment group's B operand
    size_t off_b = 0, off_yt = 0;
    rt::DeviceBuffer dms, tw_lo, tw_hi, qtable, wq;
};

FddBatch::FddBatch(size_t nchans, float dt, float f0, float df, int in_nbits, int device)
    : m_nchans(nchans), m_nbits(in_nbits), m_device(device), m_dt(dt)
{
    if (nchans == 0) DD_THROW_MSG(DEDISP_INVALID_PLAN, "nchans must be positive");
    if (in_nbits != 1 && in_nbits != 2 && in_nbits != 4 && in_nbits != 8 && in_nbits != 16 && in_nbits != 32)
        DD_THROW(DEDISP_UNSUPPORTED_IN_NBITS);
    if ((nchans * (size_t)in_nbits) % 8 != 0) DD_THROW(DEDISP_INVALID_STRIDE);
    m_delays.assign(nchans, 0.f);
    hostmath::delay_table(nchans, dt, f0, df, m_delays.data());
    m_km.assign(nchans, 1);
    rt::DeviceGuard g(m_device);
    for (auto& e : m_ev) e.reset(new rt::Event(true));
    m_err.reserve(sizeof(unsigned));
    RT_CHECK(cudaMemset(m_err.get(), 0, sizeof(unsigned)));
}

FddBatch::~FddBatch()
{
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != m_device) cudaSetDevice(m_device);
    cudaDeviceSynchronize();
    drop_graph();
}

void FddBatch::drop_graph()
{
    if (m_exec) cudaGraphExecDestroy(m_exec);
    if (m_graph) cudaGraphDestroy(m_graph);
    m_exec = nullptr;
    m_graph = nullptr;
}

void FddBatch::set_killmask(const int32_t* killmask)
{
    for (size_t c = 0; c < m_nchans; ++c) m_km[c] = killmask ? killmask[c] : 1;
    m_dirty = true;
}

void FddBatch::set_beams(std::vector<FddBeamSpec> beams)
{
    if (beams.empty()) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "a batch needs at least one beam");
    std::vector<std::unique_ptr<Beam>> bs;
    for (auto& spec : beams) {
        if (!spec.in || !spec.out) DD_THROW(DEDISP_INVALID_POINTER);
        if (spec.dms.empty()) DD_THROW(DEDISP_NO_DM_LIST_SET);
        if (spec.in_stride < m_nchans * (size_t)m_nbits / 8) DD_THROW(DEDISP_INVALID_STRIDE);
        std::unique_ptr<Beam> b(new Beam());
        b->spec = std::move(spec);
        b->max_delay = hostmath::max_delay(b->spec.dms.back(), m_delays[m_nchans - 1]);
        if (b->spec.nsamps < b->max_delay) DD_THROW(DEDISP_TOO_FEW_NSAMPS);
        b->nout = b->spec.nsamps - b->max_delay;
        if (b->spec.out_stride < b->nout * sizeof(float) || b->spec.out_stride % sizeof(float))
            DD_THROW(DEDISP_INVALID_STRIDE);
        bs.push_back(std::move(b));
    }
    m_beams = std::move(bs);
    m_dirty = true;
    plan();
}

size_t FddBatch::max_delay(size_t beam) const
{
    if (beam >= m_beams.size()) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "beam index out of range");
    return m_beams[beam]->max_delay;
}

int FddBatch::phasor_source(size_t beam) const
{
    if (beam >= m_beams.size()) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "beam index out of range");
    const Beam& b = *m_beams[beam];
    if (b.nout == 0 || m_nact == 0) return -1;
    return b.src.hybrid ? 2 : b.src.dmax >= 0 ? 0 : b.src.direct ? 3 : 1;
}

size_t FddBatch::nsamp_out(size_t beam) const
{
    if (beam >= m_beams.size()) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "beam index out of range");
    return m_beams[beam]->nout;
}

void FddBatch::plan()
{
    m_nact = 0;
    for (int32_t k : m_km) m_nact += k != 0;
    m_nact_pad = kern::tc_pad_channels(std::max(m_nact, 1));
    size_t shared = 0, scratch = 0, per_beam = 0;
    for (auto& bp : m_beams) {
        Beam& b = *bp;
        b.off_b = b.off_yt = 0;
        if (b.nout == 0) continue;
        FddOptions opt;
        opt.segmented = 1;
        opt.output = FddOutput::TimeSeries;
        opt.precision = FddPrecision::BF16x3;
        opt.segment_nfft = m_segment_nfft;
        b.g = fdd_geometry(opt, b.spec.nsamps, b.max_delay, b.spec.dms.size(), (size_t)std::max(m_nact, 1));
        const size_t nfft = b.g.nfft, nseg = b.g.nchunk, nbins = b.g.nbins;
        const bool pow2 = (nfft & (nfft - 1)) == 0;
        b.qpath = !(pow2 && nfft >= 512 && nfft <= (size_t)kern::kMaxFft);
        if (b.qpath && !kern::fftq_length(nfft)) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "unsupported FFT length");
        b.bmap = b.qpath ? kern::fdd_binmap(nfft) : kern::BinMap{8192u, 1u, nfft / 2};
        b.bin_pitch = round_up(nbins, 32);
        b.seg_stride = b.g.nsamp_good;
        b.x_len = round_up((nseg - 1) * b.seg_stride + nfft, 32);
        const size_t ndm = b.spec.dms.size();
        // largest delay index over DMs and active channels (reference trunc rule)
        long dmax = 0;
        bool ok = true;
        for (float d : b.spec.dms) {
            if (!(d >= 0.f)) { ok = false; break; }
            for (size_t c = 0; c < m_nchans; ++c)
                if (m_km[c]) dmax = std::max<long>(dmax, hostmath::delay_trunc(d, m_delays[c]));
        }
        b.dmax = (ok && dmax < (1l << 30)) ? (int)dmax : -1;
        b.ngroups = (int)((nseg + kern::kTcMaxSeg - 1) / kern::kTcMaxSeg);
        b.npad = kern::tc_pad_n((int)std::min<size_t>(nseg, kern::kTcMaxSeg));
        const int cap = std::min(kern::tc_table_capacity(b.npad, nfft / 256, m_nact_pad), kern::tc_table_cap_limit());
        b.src = kern::tc_choose_source(b.dmax, (unsigned)nfft, cap,
                                       kern::tc_quarter_mode_fits((unsigned)nfft, m_nact_pad, b.npad));
        if (b.src.dmax == -2) DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "tensor-core MAC: transform length too large");
        b.b_bytes = round_up(kern::tc_b_bytes(nbins, m_nact_pad, (int)std::min<size_t>(nseg, kern::kTcMaxSeg)),
                             kAlign);
        const size_t yt = round_up(nbins * nseg * ndm * sizeof(float2), kAlign);
        b.off_b = per_beam;
        b.off_yt = per_beam + (size_t)b.ngroups * b.b_bytes;
        per_beam = b.off_yt + yt;
        // unpack + spectra before the MAC, DM-major spectra after it: the same region
        const size_t xb = round_up(m_nchans * b.x_len * sizeof(float), kAlign);
        const size_t Xb = round_up(m_nchans * nseg * b.bin_pitch * sizeof(float2), kAlign);
        const size_t Yb = round_up(ndm * nseg * b.bin_pitch * sizeof(float2), kAlign);
        shared = std::max(shared, std::max(xb + Xb, Yb));
        const size_t rows = std::max(m_nchans, ndm) * nseg;
        const size_t sc = b.qpath ? rows * (nfft / 2) : kern::fft_scratch_elems((int)nfft, rows);
        scratch = std::max(scratch, round_up(sc * sizeof(float2), kAlign));
    }
    // The MAC's shared-memory layout is the union of the beams' tables. When
    // they do not fit together, every beam's source is chosen again for the
    // room left beside all beams' twiddle tables (a shorter per-bin table with
    // the larger delays computed, the quarter-wave table if it fits, or every
    // phasor computed): then the union fits by construction.
    int npad_u = 16;
    size_t hi_all = 0;
    for (auto& bp : m_beams) {
        if (bp->nout == 0) continue;
        npad_u = std::max(npad_u, bp->npad);
        if (bp->g.nfft % 256 == 0) hi_all = std::max(hi_all, bp->g.nfft / 256);
    }
    auto union_bytes = [&]() {
        size_t table = 0, hi = 0;
        for (auto& bp : m_beams) {
            const Beam& b = *bp;
            if (b.nout == 0) continue;
            const size_t t = b.src.dmax >= 0 ? (size_t)b.src.dmax + 1 : b.src.direct ? 0 : b.g.nfft / 4 + 1;
            table = std::max(table, t);
            if (b.src.dmax >= 0 || b.src.direct) hi = std::max(hi, b.g.nfft / 256);
        }
        return kern::tc_layout_bytes(npad_u, table, hi, m_nact_pad, 2);
    };
    if (union_bytes() > kern::kTcMaxSmem) {
        const int cap = std::min(kern::tc_table_capacity(npad_u, hi_all, m_nact_pad), kern::tc_table_cap_limit());
        for (auto& bp : m_beams) {
            Beam& b = *bp;
            if (b.nout == 0) continue;
            const unsigned n = (unsigned)b.g.nfft;
            const bool quarter = cap >= 0 && (size_t)n / 4 <= (size_t)cap && kern::tc_quarter_mode_fits(n, m_nact_pad, b.npad);
            b.src = kern::tc_choose_source(b.dmax, n, cap, quarter);
            if (b.src.dmax == -2)
                DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "tensor-core MAC: the beams' tables do not fit");
        }
        if (union_bytes() > kern::kTcMaxSmem)
            DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "tensor-core MAC: the beams' tables do not fit");
    }
    m_shared_bytes = shared;
    m_scratch_off = shared;
    m_scratch_bytes = scratch;
    const size_t base = shared + scratch;
    for (auto& bp : m_beams) {
        if (bp->nout == 0) continue;
        bp->off_b += base;
        bp->off_yt += base;
    }
    m_ws_bytes = base + per_beam;
}

size_t FddBatch::workspace_bytes() const { return m_ws_bytes; }

void FddBatch::set_workspace(void* ptr, size_t bytes)
{
    if (ptr && bytes < workspace_bytes()) DD_THROW_MSG(DEDISP_MEM_ALLOC_FAILED, "workspace too small");
    m_ext_ws = ptr;
    m_ext_ws_bytes = bytes;
    m_dirty = true;
}

uint8_t* FddBatch::workspace_base()
{
    if (m_ext_ws) return static_cast<uint8_t*>(m_ext_ws);
    m_own_ws.reserve(workspace_bytes());
    return m_own_ws.get<uint8_t>();
}

void FddBatch::upload()
{
    rt::DeviceGuard guard(m_device);
    uint8_t* ws = workspace_base();
    // active channels, their killmask multipliers and delays (padded)
    std::vector<int32_t> chan;
    std::vector<float> km, dl;
    for (size_t c = 0; c < m_nchans; ++c) {
        if (!m_km[c]) continue;
        chan.push_back((int32_t)c);
        km.push_back((float)m_km[c]);
        dl.push_back(m_delays[c]);
    }
    chan.resize(std::max<size_t>(chan.size(), 1), 0);
    km.resize(chan.size(), 0.f);
    dl.resize((size_t)m_nact_pad, 0.f);
    m_chan.reserve(chan.size() * 4);
    m_kmv.reserve(km.size() * 4);
    m_delay_pad.reserve(dl.size() * 4);
    RT_CHECK(cudaMemcpy(m_chan.get(), chan.data(), chan.size() * 4, cudaMemcpyHostToDevice));
    RT_CHECK(cudaMemcpy(m_kmv.get(), km.data(), km.size() * 4, cudaMemcpyHostToDevice));
    RT_CHECK(cudaMemcpy(m_delay_pad.get(), dl.data(), dl.size() * 4, cudaMemcpyHostToDevice));
    {
        std::vector<float2> lo, hi;
        kern::make_twiddle_tables(16384, lo, hi);
        m_twp_lo.reserve(lo.size() * sizeof(float2));
        m_twp_hi.reserve(hi.size() * sizeof(float2));
        RT_CHECK(cudaMemcpy(m_twp_lo.get(), lo.data(), lo.size() * sizeof(float2), cudaMemcpyHostToDevice));
        RT_CHECK(cudaMemcpy(m_twp_hi.get(), hi.data(), hi.size() * sizeof(float2), cudaMemcpyHostToDevice));
    }
    std::vector<kern::TcMacArgs> descs;
    std::vector<const void*> Bs;
    for (auto& bp : m_beams) {
        Beam& b = *bp;
        if (b.nout == 0) continue;
        const size_t ndm = b.spec.dms.size();
        b.dms.reserve(ndm * 4);
        RT_CHECK(cudaMemcpy(b.dms.get(), b.spec.dms.data(), ndm * 4, cudaMemcpyHostToDevice));
        std::vector<float2> lo, hi;
        kern::make_twiddle_tables(b.g.nfft, lo, hi);
        b.tw_lo.reserve(lo.size() * sizeof(float2));
        b.tw_hi.reserve(hi.size() * sizeof(float2));
        RT_CHECK(cudaMemcpy(b.tw_lo.get(), lo.data(), lo.size() * sizeof(float2), cudaMemcpyHostToDevice));
        RT_CHECK(cudaMemcpy(b.tw_hi.get(), hi.data(), hi.size() * sizeof(float2), cudaMemcpyHostToDevice));
        if (b.src.dmax < 0 && !b.src.direct) {
            const std::vector<uint2> t = kern::tc_quarter_table((unsigned)b.g.nfft);
            b.qtable.reserve(t.size() * sizeof(uint2));
            RT_CHECK(cudaMemcpy(b.qtable.get(), t.data(), t.size() * sizeof(uint2), cudaMemcpyHostToDevice));
        }
        if (b.qpath) {
            const std::vector<float2> w = kern::fftq_wq_table(b.bmap.Q);
            b.wq.reserve(w.size() * sizeof(float2));
            RT_CHECK(cudaMemcpy(b.wq.get(), w.data(), w.size() * sizeof(float2), cudaMemcpyHostToDevice));
        }
        const size_t nseg = b.g.nchunk;
        for (int gi = 0; gi < b.ngroups; ++gi) {
            kern::TcMacArgs a;
            a.Yt = reinterpret_cast<float2*>(ws + b.off_yt);
            a.Y = nullptr;
            a.y_pitch = b.bin_pitch;
            a.dms = b.dms.get<float>();
            a.delay_act = m_delay_pad.get<float>();
            a.table = b.qtable.get<uint2>();
            a.tw_lo = b.tw_lo.get<float2>();
            a.tw_hi = b.tw_hi.get<float2>();
            a.err = m_err.get<unsigned>();
            a.nact_pad = m_nact_pad;
            a.ndm = (int)ndm;
            a.seg0 = gi * kern::kTcMaxSeg;
            a.nseg = (int)std::min<size_t>(nseg - (size_t)a.seg0, kern::kTcMaxSeg);
            a.nseg_total = (int)nseg;
            a.npad = b.npad;
            a.nbins = b.g.nbins;
            a.nfft = (unsigned)b.g.nfft;
            a.round_delays = 0;
            a.dmax = b.src.dmax;
            a.direct = b.src.direct;
            a.hybrid = b.src.hybrid;
            descs.push_back(a);
            Bs.push_back(ws + b.off_b + (size_t)gi * b.b_bytes);
        }
    }
    if (descs.size() > (size_t)kern::kTcMaxDesc)
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "a batch holds at most 48 beam segment groups");
    // Segment groups of at most 32 MMA columns take the wide fused form, the
    // others the three-MMA form: a launch for each class present (a launch's
    // form follows its widest descriptor).
    std::vector<kern::TcMacArgs> cls_descs[2];
    std::vector<const void*> cls_bs[2];
    for (size_t d = 0; d < descs.size(); ++d) {
        const int c = descs[d].npad <= 32 ? 0 : 1;
        cls_descs[c].push_back(descs[d]);
        cls_bs[c].push_back(Bs[d]);
    }
    for (int c = 0; c < 2; ++c) {
        m_params[c].reset();
        if (cls_descs[c].empty()) continue;
        m_params[c].reset(new kern::TcParams());
        const std::vector<kern::TcWork> items = kern::tc_work_items(cls_descs[c], kern::tc_sm_count());
        const size_t ib = kern::tc_work_bytes(items.size());
        m_items[c].reserve(ib);
        kern::tc_prepare_list(*m_params[c], cls_descs[c], cls_bs[c], items, m_err.get<unsigned>(), m_items[c].get(),
                              ib, nullptr);
    }
    RT_CHECK(cudaDeviceSynchronize());
}

void FddBatch::enqueue(cudaStream_t s, bool timing)
{
    uint8_t* ws = workspace_base();
    float* x = reinterpret_cast<float*>(ws);
    float2* scratch = reinterpret_cast<float2*>(ws + m_scratch_off);
    int launches = 0;
    if (timing) m_ev[0]->record(s);
    RT_CHECK(cudaMemsetAsync(m_err.get(), 0, sizeof(unsigned), s));
    const float scale = (float)(1.0 / (double)m_nchans);
    const kern::TwiddleTable twp{m_twp_lo.get<float2>(), m_twp_hi.get<float2>(), 16384};
    for (auto& bp : m_beams) {
        Beam& b = *bp;
        if (b.nout == 0) continue;
        const size_t nseg = b.g.nchunk;
        float2* X = reinterpret_cast<float2*>(ws + round_up(m_nchans * b.x_len * sizeof(float), kAlign));
        const kern::TwiddleTable tw{b.tw_lo.get<float2>(), b.tw_hi.get<float2>(), (unsigned)b.g.nfft};
        kern::launch_fdd_unpack(b.spec.in, b.spec.in_stride, m_nbits, b.spec.nsamps, m_nchans, scale, x, b.x_len,
                                b.x_len, s);
        if (b.qpath)
            kern::launch_fft_r2c_q(x, b.x_len, m_nchans, nseg, b.seg_stride, b.g.nfft, X, b.bin_pitch, tw, twp,
                                   b.wq.get<float2>(), scratch, s);
        else
            kern::launch_fft_r2c(x, b.x_len, m_nchans, nseg, b.seg_stride, (int)b.g.nfft, X, b.bin_pitch, tw,
                                 scratch, s);
        launches += 2;
        for (int gi = 0; gi < b.ngroups; ++gi) {
            const int s0 = gi * kern::kTcMaxSeg;
            const int ns = (int)std::min<size_t>(nseg - (size_t)s0, kern::kTcMaxSeg);
            kern::launch_fdd_prep_b(X, b.bin_pitch, ns, b.g.nbins, m_chan.get<int32_t>(), m_kmv.get<float>(),
                                    m_nact, m_nact_pad, b.npad, ws + b.off_b + (size_t)gi * b.b_bytes, b.bmap,
                                    s0, (int)nseg, s);
            ++launches;
        }
    }
    if (timing) m_ev[1]->record(s);
    for (int c = 0; c < 2; ++c) {
        kern::TcParams* P = m_params[c].get();
        if (m_nact == 0 || !P || P->nitems <= 0) continue;
        if (timing) m_cta_ns[c].reserve((size_t)kern::tc_sm_count() * sizeof(unsigned long long));
        P->cta_ns = timing ? m_cta_ns[c].get<unsigned long long>() : nullptr;
        kern::launch_fdd_mac_tc_list(*P, s);
        P->cta_ns = nullptr;
        ++launches;
    }
    if (timing) m_ev[2]->record(s);
    for (auto& bp : m_beams) {
        Beam& b = *bp;
        if (b.nout == 0) continue;
        const size_t nseg = b.g.nchunk, ndm = b.spec.dms.size();
        float2* Yt = reinterpret_cast<float2*>(ws + b.off_yt);
        float2* Y = reinterpret_cast<float2*>(ws);
        float* out = reinterpret_cast<float*>(b.spec.out);
        const kern::TwiddleTable tw{b.tw_lo.get<float2>(), b.tw_hi.get<float2>(), (unsigned)b.g.nfft};
        if (m_nact == 0) RT_CHECK(cudaMemsetAsync(Yt, 0, b.g.nbins * nseg * ndm * sizeof(float2), s));
        kern::launch_fdd_to_dmmajor(Yt, nseg, ndm, b.g.nbins, Y, b.bin_pitch, b.bmap, s);
        const size_t ostride = b.spec.out_stride / sizeof(float);
        if (b.qpath)
            kern::launch_fft_c2r_q(Y, b.bin_pitch, ndm, nseg, b.g.nfft, out, ostride, b.g.nsamp_good, b.nout, tw,
                                   twp, b.wq.get<float2>(), scratch, s);
        else
            kern::launch_fft_c2r(Y, b.bin_pitch, ndm, nseg, (int)b.g.nfft, out, ostride, b.g.nsamp_good, b.nout,
                                 tw, scratch, s);
        launches += 2;
    }
    if (timing) m_ev[3]->record(s);
    last_launches = launches;
}

void FddBatch::execute(cudaStream_t stream, bool use_graph)
{
    rt::DeviceGuard g(m_device);
    if (m_beams.empty()) return;
    if (m_dirty) {
        drop_graph();
        plan();
        upload();
        m_dirty = false;
    }
    if (!use_graph) {
        enqueue(stream, record_timing);
    } else {
        if (!m_exec) {
            rt::Stream cap;
            RT_CHECK(cudaStreamBeginCapture(cap.get(), cudaStreamCaptureModeRelaxed));
            try {
                enqueue(cap.get(), false);
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
        RT_CHECK(cudaEventSynchronize(use_graph ? m_ev[2]->get() : m_ev[3]->get()));
        if (kern::read_error_word(m_err.get<unsigned>(), stream))
            DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "tensor-core MAC pipeline wait expired");
        if (use_graph) {
            last_prep_ms = last_post_ms = -1.f;
            RT_CHECK(cudaEventElapsedTime(&last_mac_ms, m_ev[1]->get(), m_ev[2]->get()));
        } else {
            RT_CHECK(cudaEventElapsedTime(&last_prep_ms, m_ev[0]->get(), m_ev[1]->get()));
            RT_CHECK(cudaEventElapsedTime(&last_mac_ms, m_ev[1]->get(), m_ev[2]->get()));
            RT_CHECK(cudaEventElapsedTime(&last_post_ms, m_ev[2]->get(), m_ev[3]->get()));
            // the launches run one after the other: sums of their slowest
            // and of their mean CTA times
            last_cta_max_ms = last_cta_mean_ms = 0.f;
            for (int c = 0; c < 2; ++c) {
                const kern::TcParams* P = m_params[c].get();
                if (m_nact == 0 || !P || P->nitems <= 0) continue;
                const int n = std::min(P->nitems, kern::tc_sm_count());
                std::vector<unsigned long long> ns((size_t)n);
                RT_CHECK(cudaMemcpy(ns.data(), m_cta_ns[c].get(), ns.size() * sizeof(ns[0]), cudaMemcpyDeviceToHost));
                double sum = 0, mx = 0;
                for (unsigned long long v : ns) {
                    sum += (double)v;
                    mx = std::max(mx, (double)v);
                }
                last_cta_max_ms += (float)(mx * 1e-6);
                last_cta_mean_ms += (float)(sum / n * 1e-6);
            }
        }
    }
}

void FddBatch::sync(cudaStream_t stream)
{
    rt::DeviceGuard g(m_device);
    RT_CHECK(cudaStreamSynchronize(stream));
    if (kern::read_error_word(m_err.get<unsigned>(), stream))
        DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "tensor-core MAC pipeline wait expired");
}

}  // namespace detail
}  // namespace dedisp

// ---------------------------------------------------------------------------
// C interface (include/dedisp_b200.h). Errors are returned with their
// specific code (and noted for dedisp_b200_last_error).
// ---------------------------------------------------------------------------
struct dedisp_b200_fdd_batch_struct {
    std::unique_ptr<dedisp::detail::FddBatch> b;
};

namespace dedisp {
void note_last_error(dedisp_error code, const char* msg);
}

namespace {
template <typename F>
dedisp_error fdd_batch_call(dedisp_b200_fdd_batch batch, F&& fn)
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

dedisp_error dedisp_b200_fdd_batch_create(dedisp_b200_fdd_batch* batch, dedisp_size nchans, dedisp_float dt,
                                          dedisp_float f0, dedisp_float df, dedisp_size in_nbits, int device)
{
    if (!batch) return DEDISP_INVALID_POINTER;
    *batch = nullptr;
    try {
        auto* h = new dedisp_b200_fdd_batch_struct;
        try {
            h->b.reset(new dedisp::detail::FddBatch(nchans, dt, f0, df, (int)in_nbits, device));
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

void dedisp_b200_fdd_batch_destroy(dedisp_b200_fdd_batch batch)
{
    try {
        delete batch;
    } catch (...) {
    }
}

dedisp_error dedisp_b200_fdd_batch_set_killmask(dedisp_b200_fdd_batch batch, const dedisp_bool* killmask)
{
    return fdd_batch_call(batch, [&](dedisp::detail::FddBatch& b) {
        b.set_killmask(reinterpret_cast<const int32_t*>(killmask));
    });
}

dedisp_error dedisp_b200_fdd_batch_set_beams(dedisp_b200_fdd_batch batch, const dedisp_b200_beam* beams,
                                             dedisp_size nbeams)
{
    if (!beams && nbeams) return DEDISP_INVALID_POINTER;
    return fdd_batch_call(batch, [&](dedisp::detail::FddBatch& b) {
        std::vector<dedisp::detail::FddBeamSpec> specs;
        for (dedisp_size i = 0; i < nbeams; ++i) {
            const dedisp_b200_beam& s = beams[i];
            if (!s.dm_list || s.dm_count == 0) DD_THROW(DEDISP_NO_DM_LIST_SET);
            dedisp::detail::FddBeamSpec sp;
            sp.in = s.in;
            sp.in_stride = s.in_stride;
            sp.nsamps = s.nsamps;
            sp.dms.assign(s.dm_list, s.dm_list + s.dm_count);
            sp.out = s.out;
            sp.out_stride = s.out_stride;
            specs.push_back(std::move(sp));
        }
        b.set_beams(std::move(specs));
    });
}

dedisp_size dedisp_b200_fdd_batch_workspace_size(dedisp_b200_fdd_batch batch)
{
    dedisp_size n = 0;
    if (fdd_batch_call(batch, [&](dedisp::detail::FddBatch& b) { n = b.workspace_bytes(); }) != DEDISP_NO_ERROR)
        return 0;
    return n;
}

dedisp_error dedisp_b200_fdd_batch_set_workspace(dedisp_b200_fdd_batch batch, void* d_workspace,
                                                 dedisp_size bytes)
{
    return fdd_batch_call(batch, [&](dedisp::detail::FddBatch& b) { b.set_workspace(d_workspace, bytes); });
}

dedisp_error dedisp_b200_fdd_batch_execute(dedisp_b200_fdd_batch batch, void* stream, int use_graph)
{
    return fdd_batch_call(batch, [&](dedisp::detail::FddBatch& b) {
        b.execute(static_cast<cudaStream_t>(stream), use_graph != 0);
    });
}

dedisp_error dedisp_b200_fdd_batch_sync(dedisp_b200_fdd_batch batch, void* stream)
{
    return fdd_batch_call(batch, [&](dedisp::detail::FddBatch& b) { b.sync(static_cast<cudaStream_t>(stream)); });
}

dedisp_error dedisp_b200_fdd_batch_set_timing(dedisp_b200_fdd_batch batch, int enable)
{
    return fdd_batch_call(batch, [&](dedisp::detail::FddBatch& b) { b.record_timing = enable != 0; });
}

dedisp_error dedisp_b200_fdd_batch_get_timing(dedisp_b200_fdd_batch batch, float* prep_ms, float* mac_ms,
                                              float* post_ms, int* launches)
{
    return fdd_batch_call(batch, [&](dedisp::detail::FddBatch& b) {
        if (prep_ms) *prep_ms = b.last_prep_ms;
        if (mac_ms) *mac_ms = b.last_mac_ms;
        if (post_ms) *post_ms = b.last_post_ms;
        if (launches) *launches = b.last_launches;
    });
}

dedisp_error dedisp_b200_fdd_batch_set_segment_nfft(dedisp_b200_fdd_batch batch, dedisp_size segment_nfft)
{
    return fdd_batch_call(batch, [&](dedisp::detail::FddBatch& b) { b.set_segment_nfft(segment_nfft); });
}

dedisp_error dedisp_b200_fdd_batch_get_mac_balance(dedisp_b200_fdd_batch batch, float* cta_max_ms,
                                                   float* cta_mean_ms)
{
    return fdd_batch_call(batch, [&](dedisp::detail::FddBatch& b) {
        if (cta_max_ms) *cta_max_ms = b.last_cta_max_ms;
        if (cta_mean_ms) *cta_mean_ms = b.last_cta_mean_ms;
    });
}

int dedisp_b200_fdd_batch_phasor_source(dedisp_b200_fdd_batch batch, dedisp_size beam)
{
    int v = -1;
    if (fdd_batch_call(batch, [&](dedisp::detail::FddBatch& b) { v = b.phasor_source(beam); }) != DEDISP_NO_ERROR)
        return -1;
    return v;
}

dedisp_size dedisp_b200_fdd_batch_max_delay(dedisp_b200_fdd_batch batch, dedisp_size beam)
{
    dedisp_size n = 0;
    if (fdd_batch_call(batch, [&](dedisp::detail::FddBatch& b) { n = b.max_delay(beam); }) != DEDISP_NO_ERROR)
        return 0;
    return n;
}

}  // extern "C"
