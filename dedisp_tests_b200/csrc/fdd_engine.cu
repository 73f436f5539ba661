// FDD execution engine: unpack -> real FFT per (channel, segment) ->
// bin-major -> phasor MAC -> spectrum output, or DM-major -> inverse real
// FFT with stitching (src/fdd/FDDGPUPlan.cpp:58-706 whole series,
// :725-1271 segmented).
#include "fdd_engine.hpp"

#include <algorithm>
#include <cmath>
#include <vector>

#include "fdd_kernels.hpp"
#include "fdd_tc.hpp"
#include "host_math.hpp"

namespace dedisp {
namespace detail {

namespace {
size_t round_up(size_t a, size_t b) { return (a + b - 1) / b * b; }
}  // namespace

struct FddEngine::Impl {
    rt::DeviceBuffer in, x, X, Xt, Yt, Y, out, tw_lo, tw_hi, dms, chan, km, delay_act;
    // tensor-core form
    rt::DeviceBuffer B, delay_pad, qtable, err, tcwork;
    rt::DeviceBuffer fft_tmp;  // four-step FFT scratch (nfft > 32768)
    rt::DeviceBuffer twp_lo, twp_hi, wq;  // transforms of 16384 Q points: 16384-point table, W_Q
    unsigned wq_n = 0;
    unsigned qtable_n = 0;
    int delay_pad_n = -1;
    unsigned tw_n = 0;
    unsigned long version = ~0ul;
    unsigned long pad_version = ~0ul;
    unsigned long dmax_version = ~0ul;
    int dmax_round = -1;
    int dmax = -1;               // largest delay index, -1 if any DM is negative or NaN
    int nact = 0;
    std::vector<float> delays_active;
};

FddEngine::FddEngine(GpuState& gpu) : m_gpu(gpu), m_impl(new Impl()) {}
FddEngine::~FddEngine()
{
    if (m_gpu.has_device) {
        rt::DeviceGuard g(m_gpu.device);
        cudaStreamSynchronize(m_gpu.stream());
    }
}

void FddEngine::execute(const FddOptions& opt, const FddView& v, const FddCall& c)
{
    m_gpu.require_device();
    rt::DeviceGuard guard(m_gpu.device);
    Impl& m = *m_impl;
    stats = ExecTiming();

    size_t nlive = 0;  // channels the killmask keeps (automatic segment length)
    for (size_t i = 0; i < v.nchans; ++i) nlive += (!v.killmask || v.killmask[i]) ? 1 : 0;
    const FddGeometry g = fdd_geometry(opt, c.nsamps, v.max_delay, v.ndm, std::max<size_t>(1, nlive));
    // Power-of-two lengths up to 2^20: one-CTA or four-step transforms;
    // other multiples of 16384 (the whole-series rule) and longer lengths:
    // the 16384 Q-point transforms (spectra in the BinMap order).
    const bool pow2 = (g.nfft & (g.nfft - 1)) == 0;
    const bool qpath = !(pow2 && g.nfft >= 512 && g.nfft <= (size_t)kern::kMaxFft);
    if (qpath && !kern::fftq_length(g.nfft))
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR,
                     "FDD transform length must be a power of two in 512..2^20 or a multiple of 16384");
    const kern::BinMap bmap = qpath ? kern::fdd_binmap(g.nfft) : kern::BinMap{8192u, 1u, g.nfft / 2};
    const bool dev = (c.flags & DEDISP_DEVICE_POINTERS) != 0;
    cudaStream_t st = m_gpu.stream();
    const size_t nchans = v.nchans, ndm = v.ndm, nseg = g.nchunk;
    const size_t nbins = g.nbins;
    const size_t bin_pitch = round_up(nbins, 32);
    const size_t seg_stride = g.segmented ? g.nsamp_good : 0;
    const size_t x_len = round_up((nseg - 1) * seg_stride + g.nfft, 32);
    const size_t in_stride = nchans * (size_t)c.in_nbits / 8;

    // Per-plan state: active channels, killmask multipliers, DM list.
    if (m.version != v.version) {
        std::vector<int32_t> chan;
        std::vector<float> km, dl;
        for (size_t i = 0; i < nchans; ++i) {
            if (v.killmask[i] == 0) continue;
            chan.push_back((int32_t)i);
            km.push_back((float)v.killmask[i]);
            dl.push_back(v.delays[i]);
        }
        m.nact = (int)chan.size();
        const size_t n = std::max<size_t>(1, chan.size());
        chan.resize(n, 0);
        km.resize(n, 0.f);
        dl.resize(n, 0.f);
        m.chan.reserve(n * 4);
        m.km.reserve(n * 4);
        m.delay_act.reserve(n * 4);
        m.dms.reserve(ndm * 4);
        RT_CHECK(cudaMemcpy(m.chan.get(), chan.data(), n * 4, cudaMemcpyHostToDevice));
        RT_CHECK(cudaMemcpy(m.km.get(), km.data(), n * 4, cudaMemcpyHostToDevice));
        RT_CHECK(cudaMemcpy(m.delay_act.get(), dl.data(), n * 4, cudaMemcpyHostToDevice));
        RT_CHECK(cudaMemcpy(m.dms.get(), v.dms, ndm * 4, cudaMemcpyHostToDevice));
        m.delays_active.assign(dl.begin(), dl.begin() + m.nact);
        m.version = v.version;
    }
    const bool use_tc = opt.precision == FddPrecision::BF16x3 && m.nact > 0;
    // Twiddles W_N^t = exp(-2 pi i t / N) as hi[t >> 8] * lo[t & 255].
    if (m.tw_n != g.nfft) {
        const unsigned n = (unsigned)g.nfft;
        std::vector<float2> lo(256), hi(n / 256);
        for (unsigned l = 0; l < 256; ++l) {
            const double a = -2.0 * 3.14159265358979323846 * (double)l / (double)n;
            lo[l] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        for (unsigned h = 0; h < n / 256; ++h) {
            const double a = -2.0 * 3.14159265358979323846 * (double)h * 256.0 / (double)n;
            hi[h] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        m.tw_lo.reserve(256 * sizeof(float2));
        m.tw_hi.reserve(hi.size() * sizeof(float2));
        RT_CHECK(cudaMemcpy(m.tw_lo.get(), lo.data(), 256 * sizeof(float2), cudaMemcpyHostToDevice));
        RT_CHECK(cudaMemcpy(m.tw_hi.get(), hi.data(), hi.size() * sizeof(float2),
                            cudaMemcpyHostToDevice));
        m.tw_n = n;
    }
    kern::TwiddleTable tw{m.tw_lo.get<float2>(), m.tw_hi.get<float2>(), (unsigned)g.nfft};
    kern::TwiddleTable twp{nullptr, nullptr, 16384};
    if (qpath) {
        if (!m.twp_lo.get()) {
            std::vector<float2> lo(256), hi(16384 / 256);
            for (unsigned l = 0; l < 256; ++l) {
                const double a = -2.0 * 3.14159265358979323846 * (double)l / 16384.0;
                lo[l] = make_float2((float)std::cos(a), (float)std::sin(a));
            }
            for (unsigned h = 0; h < hi.size(); ++h) {
                const double a = -2.0 * 3.14159265358979323846 * (double)h * 256.0 / 16384.0;
                hi[h] = make_float2((float)std::cos(a), (float)std::sin(a));
            }
            m.twp_lo.reserve(lo.size() * sizeof(float2));
            m.twp_hi.reserve(hi.size() * sizeof(float2));
            RT_CHECK(cudaMemcpy(m.twp_lo.get(), lo.data(), lo.size() * sizeof(float2), cudaMemcpyHostToDevice));
            RT_CHECK(cudaMemcpy(m.twp_hi.get(), hi.data(), hi.size() * sizeof(float2), cudaMemcpyHostToDevice));
        }
        twp = kern::TwiddleTable{m.twp_lo.get<float2>(), m.twp_hi.get<float2>(), 16384};
        if (m.wq_n != bmap.Q) {
            const std::vector<float2> w = kern::fftq_wq_table(bmap.Q);
            m.wq.reserve(w.size() * sizeof(float2));
            RT_CHECK(cudaMemcpy(m.wq.get(), w.data(), w.size() * sizeof(float2), cudaMemcpyHostToDevice));
            m.wq_n = bmap.Q;
        }
    }

    // Buffers.
    const uint8_t* d_in = c.in;
    if (!dev) {
        m.in.reserve(c.nsamps * in_stride);
        d_in = m.in.get<uint8_t>();
    }
    m.x.reserve(nchans * x_len * sizeof(float));
    m.X.reserve(nchans * nseg * bin_pitch * sizeof(float2));
    int nact_pad = 0, npad = 0, tc_dmax = -1;
    bool tc_direct = false, tc_hybrid = false;
    int tc_form = -1;
    const int seg_group = (int)std::min<size_t>(nseg, (size_t)kern::kTcMaxSeg);
    if (use_tc || nseg == 1) {
        // Largest delay index over all DMs and active channels (same float
        // operations as the kernels): the tensor-core MAC and the one-segment
        // FP32 MAC build a per-bin phasor table over 0..dmax when it fits
        // shared memory.
        const int rnd = opt.round_delays ? 1 : 0;
        if (m.dmax_version != v.version || m.dmax_round != rnd) {
            long dmax = 0;
            bool ok = true;
            for (size_t i = 0; i < ndm && ok; ++i) {
                const float d = v.dms[i];
                if (!(d >= 0.f)) { ok = false; break; }
                for (float dl : m.delays_active) {
                    const long x = rnd ? (long)hostmath::delay_rn(d, dl) : (long)hostmath::delay_trunc(d, dl);
                    dmax = std::max(dmax, x);
                }
            }
            m.dmax = (ok && dmax < (1l << 30)) ? (int)dmax : -1;
            m.dmax_version = v.version;
            m.dmax_round = rnd;
        }
    }
    if (use_tc) {
        nact_pad = kern::tc_pad_channels(m.nact);
        npad = kern::tc_pad_n(seg_group);
        m.B.reserve(kern::tc_b_bytes(nbins, nact_pad, seg_group));
        if (m.pad_version != v.version || m.delay_pad_n != nact_pad) {
            std::vector<float> dp(m.delays_active);
            dp.resize(nact_pad, 0.f);
            m.delay_pad.reserve(dp.size() * 4);
            RT_CHECK(cudaMemcpy(m.delay_pad.get(), dp.data(), dp.size() * 4, cudaMemcpyHostToDevice));
            m.pad_version = v.version;
            m.delay_pad_n = nact_pad;
        }
        // Phasor source: the per-bin delay table when it holds every delay,
        // else the cheapest of the quarter-wave table (power-of-two lengths),
        // the table over the small delays with the rest computed (hybrid),
        // or each phasor from the two-level twiddle tables.
        const int cap = std::min(kern::tc_table_capacity(npad, g.nfft / 256, nact_pad), kern::tc_table_cap_limit());
        const kern::TcSource src = kern::tc_choose_source(
            m.dmax, (unsigned)g.nfft, cap, kern::tc_quarter_mode_fits((unsigned)g.nfft, nact_pad, npad));
        if (src.dmax == -2)
            DD_THROW_MSG(DEDISP_UNKNOWN_ERROR,
                         "tensor-core MAC: transform length too large for its twiddle tables in shared "
                         "memory; use precision 0");
        tc_dmax = src.dmax;
        tc_direct = src.direct != 0;
        tc_hybrid = src.hybrid != 0;
        if (m.qtable_n != g.nfft) {
            const std::vector<uint2> t = kern::tc_quarter_table((unsigned)g.nfft);
            m.qtable.reserve(t.size() * sizeof(uint2));
            RT_CHECK(cudaMemcpy(m.qtable.get(), t.data(), t.size() * sizeof(uint2),
                                cudaMemcpyHostToDevice));
            m.qtable_n = (unsigned)g.nfft;
        }
        m.err.reserve(sizeof(unsigned));
    } else {
        m.Xt.reserve(nbins * nseg * std::max(1, m.nact) * sizeof(float2));
    }
    const bool inverse = g.timeseries;
    // Bin-major products, then one transpose to DM-major rows for the inverse
    // FFT: writing DM-major rows from the tensor-core epilogue directly (one
    // 8-byte store per row and bin) measured 1.8x slower for the MAC.
    const bool direct_y = false;
    m.Yt.reserve(nbins * nseg * ndm * sizeof(float2));
    if (inverse) m.Y.reserve(ndm * nseg * bin_pitch * sizeof(float2));
    float* d_out = reinterpret_cast<float*>(c.out);
    if (!dev) {
        m.out.reserve(ndm * g.row_len * sizeof(float));
        d_out = m.out.get<float>();
    }

    // stage boundaries: ev[0] start, ev[1] unpacked, ev[2] forward FFT,
    // ev[3] operand layout (= e1), ev[4] MAC (= e2), ev[5] transpose / spectrum
    // output, ev[6] inverse FFT (= e3)
    std::unique_ptr<rt::Event> ev[7];
    if (record_timing)
        for (auto& e : ev) e.reset(new rt::Event(true));
    auto mark = [&](int i) {
        if (ev[i]) ev[i]->record(st);
    };
    if (!dev)
        RT_CHECK(cudaMemcpyAsync(m.in.get(), c.in, c.nsamps * in_stride, cudaMemcpyHostToDevice, st));
    mark(0);

    const float scale = (float)(1.0 / (double)nchans);
    kern::launch_fdd_unpack(d_in, in_stride, c.in_nbits, c.nsamps, nchans, scale, m.x.get<float>(),
                            x_len, x_len, st);
    mark(1);
    const size_t tmp_elems = qpath ? std::max(nchans, ndm) * nseg * (g.nfft / 2)
                                   : kern::fft_scratch_elems((int)g.nfft, std::max(nchans, ndm) * nseg);
    if (tmp_elems) m.fft_tmp.reserve(tmp_elems * sizeof(float2));
    if (qpath)
        kern::launch_fft_r2c_q(m.x.get<float>(), x_len, nchans, nseg, seg_stride, g.nfft, m.X.get<float2>(),
                               bin_pitch, tw, twp, m.wq.get<float2>(), m.fft_tmp.get<float2>(), st);
    else
        kern::launch_fft_r2c(m.x.get<float>(), x_len, nchans, nseg, seg_stride, (int)g.nfft,
                             m.X.get<float2>(), bin_pitch, tw, m.fft_tmp.get<float2>(), st);
    mark(2);
    if (!use_tc && m.nact > 0)
        kern::launch_fdd_to_binmajor(m.X.get<float2>(), bin_pitch, nseg, nbins, m.chan.get<int32_t>(),
                                     m.km.get<float>(), m.nact, m.Xt.get<float2>(), bmap, st);
    // one segment group: its B operand is built here (operand stage); with
    // several, each group's B is built right before its MAC launch
    const bool one_group = nseg <= (size_t)seg_group;
    if (use_tc && one_group)
        kern::launch_fdd_prep_b(m.X.get<float2>(), bin_pitch, (int)nseg, nbins, m.chan.get<int32_t>(),
                                m.km.get<float>(), m.nact, nact_pad, npad, m.B.get(), bmap, 0, (int)nseg, st);
    mark(3);

    if (use_tc) {
        RT_CHECK(cudaMemsetAsync(m.err.get(), 0, sizeof(unsigned), st));
        kern::TcMacArgs ta;
        ta.Yt = direct_y ? nullptr : m.Yt.get<float2>();
        ta.Y = direct_y ? m.Y.get<float2>() : nullptr;
        ta.y_pitch = bin_pitch;
        ta.dms = m.dms.get<float>();
        ta.delay_act = m.delay_pad.get<float>();
        ta.table = m.qtable.get<uint2>();
        ta.tw_lo = m.tw_lo.get<float2>();
        ta.tw_hi = m.tw_hi.get<float2>();
        ta.err = m.err.get<unsigned>();
        ta.nact_pad = nact_pad;
        ta.ndm = (int)ndm;
        ta.nseg_total = (int)nseg;
        ta.npad = npad;
        ta.nbins = nbins;
        ta.nfft = (unsigned)g.nfft;
        ta.round_delays = opt.round_delays ? 1 : 0;
        ta.dmax = tc_dmax;
        ta.direct = tc_direct ? 1 : 0;
        ta.hybrid = tc_hybrid ? 1 : 0;
        const size_t wb = kern::tc_work_bytes((size_t)kern::tc_sm_count() + 64);
        m.tcwork.reserve(wb);
        // Segment groups of at most kTcMaxSeg (the accumulator's 128
        // columns): B operand and one MAC launch per group.
        stats.launches = 0;
        for (size_t s0 = 0; s0 < nseg; s0 += (size_t)seg_group) {
            const int ns = (int)std::min(nseg - s0, (size_t)seg_group);
            if (!one_group)
                kern::launch_fdd_prep_b(m.X.get<float2>(), bin_pitch, ns, nbins, m.chan.get<int32_t>(),
                                        m.km.get<float>(), m.nact, nact_pad, npad, m.B.get(), bmap, (int)s0,
                                        (int)nseg, st);
            ta.nseg = ns;
            ta.seg0 = (int)s0;
            tc_form = kern::launch_fdd_mac_tc(ta, m.B.get(), m.tcwork.get(), wb, st);
            ++stats.launches;
        }
    } else if (m.nact > 0) {
        kern::MacArgs a;
        a.Xt = m.Xt.get<float2>();
        a.Yt = m.Yt.get<float2>();
        a.dms = m.dms.get<float>();
        a.delay_act = m.delay_act.get<float>();
        a.nact = m.nact;
        a.ndm = (int)ndm;
        a.nseg = (int)nseg;
        a.nbins = nbins;
        a.nfft = (unsigned)g.nfft;
        a.round_delays = opt.round_delays ? 1 : 0;
        a.tw = tw;
        // one segment: the per-bin phasor table (each phasor feeds one
        // product); several: the tiled kernel, which reuses each phasor
        // across the segments
        if (nseg == 1 && kern::fdd_mac_series_fits(m.dmax, (unsigned)g.nfft, m.nact))
            kern::launch_fdd_mac_series(a, m.dmax, st);
        else
            kern::launch_fdd_mac_plain(a, st);
        stats.launches = 1;
    } else {
        RT_CHECK(cudaMemsetAsync(m.Yt.get(), 0, nbins * nseg * ndm * sizeof(float2), st));
    }
    mark(4);

    if (!inverse) {
        // spectrum: first nfft/2 bins of each DM row, interleaved re/im
        kern::launch_fdd_spectrum_out(m.Yt.get<float2>(), ndm, g.nfft / 2, d_out, g.row_len, st);
    } else {
        if (!direct_y)
            kern::launch_fdd_to_dmmajor(m.Yt.get<float2>(), nseg, ndm, nbins, m.Y.get<float2>(),
                                        bin_pitch, bmap, st);
        mark(5);
        const size_t keep = g.segmented ? g.nsamp_good : g.nfft;
        if (qpath)
            kern::launch_fft_c2r_q(m.Y.get<float2>(), bin_pitch, ndm, nseg, g.nfft, d_out, g.row_len, keep,
                                   g.row_len, tw, twp, m.wq.get<float2>(), m.fft_tmp.get<float2>(), st);
        else
            kern::launch_fft_c2r(m.Y.get<float2>(), bin_pitch, ndm, nseg, (int)g.nfft, d_out, g.row_len,
                                 keep, g.row_len, tw, m.fft_tmp.get<float2>(), st);
    }
    if (!inverse) mark(5);
    mark(6);
    if (!dev)
        RT_CHECK(cudaMemcpyAsync(c.out, d_out, ndm * g.row_len * sizeof(float),
                                 cudaMemcpyDeviceToHost, st));
    const bool async = dev && (c.flags & DEDISP_ASYNC) && !use_tc;
    if (!async) RT_CHECK(cudaStreamSynchronize(st));
    if (use_tc) {
        unsigned err = 0;
        RT_CHECK(cudaMemcpy(&err, m.err.get(), sizeof(err), cudaMemcpyDeviceToHost));
        if (err) DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "tensor-core MAC pipeline wait expired");
    }
    if (record_timing) {
        RT_CHECK(cudaEventSynchronize(*ev[6]));
        for (int i = 0; i < 6; ++i) RT_CHECK(cudaEventElapsedTime(&stats.stage_ms[i], *ev[i], *ev[i + 1]));
        // prep: unpack, forward FFT, operand layout; post: transpose, inverse FFT
        stats.prep_ms = stats.stage_ms[0] + stats.stage_ms[1] + stats.stage_ms[2] + stats.stage_ms[4] +
                        stats.stage_ms[5];
        stats.kernel_ms = stats.stage_ms[3];
        stats.variant = use_tc ? 1 : 0;
    }
    stats.phasor = !use_tc ? -1 : tc_hybrid ? 2 : tc_dmax >= 0 ? 0 : tc_direct ? 3 : 1;
    stats.tc_form = use_tc ? tc_form : -1;
}

}  // namespace detail
}  // namespace dedisp
