// FDDGPUPlan: validation (src/fdd/FDDGPUPlan.cpp:39-67) and geometry.
#include "fdd/FDDGPUPlan.hpp"

#include <cmath>
#include <cstdlib>

#include "fdd_engine.hpp"

namespace dedisp {

namespace detail {

size_t fdd_auto_segment(size_t nsamps, size_t max_delay, size_t ndm, size_t nchans)
{
    // Modelled device time (ps) of one execute with segments of n points,
    // from stage times measured on B200 (1536- and 1024-channel beams):
    // - tensor-core MAC: per (bin, DM row, channel) about 1.08 ps while the
    //   phasor generation bounds it, growing as the MMA's columns (2 x
    //   segments, padded to 16) pass about 70; segment groups of at most 64
    //   build their phasors again;
    // - transforms and layout changes: about 10 ps per channel point and 8
    //   ps per DM point of the segmented series.
    // The FP32 MAC's work is per (bin, segment), nearly the same for every
    // length, and its 40-segment tiles favour many segments: it keeps the
    // reference rule.
    const double ndm_pad = (double)((ndm + 127) / 128 * 128);
    double best = 0;
    size_t best_n = 0;
    for (size_t n = 2048; n <= (1u << 20); n *= 2) {
        if (n <= max_delay) continue;
        const double nbins = (double)(n / 2 + 1);
        const size_t nseg = (nsamps + (n - max_delay) - 1) / (n - max_delay);
        double mac = 0;
        for (size_t s0 = 0; s0 < nseg; s0 += 64) {
            const double npad = (double)((2 * std::min<size_t>(64, nseg - s0) + 15) / 16 * 16);
            mac += nbins * ndm_pad * (double)nchans * 1.08 * std::max(1.0, npad / 70.0);
        }
        const double xf = (10.0 * (double)nchans + 8.0 * (double)ndm) * (double)nseg * (double)n;
        const double t = mac + xf;
        if (best_n == 0 || t < best) {
            best = t;
            best_n = n;
        }
    }
    return best_n;  // 0: no power of two up to 2^20 exceeds the max delay
}

FddGeometry fdd_geometry(const FddOptions& opt, size_t nsamps, size_t max_delay, size_t ndm, size_t nchans)
{
    FddGeometry g;
    bool seg = opt.segmented > 0;
    if (opt.segmented < 0) {
        const char* s = std::getenv("USE_SEGMENTED");
        seg = s && std::atoi(s) != 0;
    }
    g.segmented = seg;
    if (seg) {
        // nfft doubles from 16384 while nfft*(1 - 0.8f) < max_delay
        // (FDDGPUPlan.cpp:742,762-768); nsamp_good = nfft - max_delay.
        const bool autoseg = opt.segment_nfft == FddOptions::kSegmentAuto;
        size_t n = (opt.segment_nfft && !autoseg) ? opt.segment_nfft : 16384;
        const size_t na = (autoseg && ndm && nchans && opt.precision == FddPrecision::BF16x3)
                              ? fdd_auto_segment(nsamps, max_delay, ndm, nchans)
                              : 0;
        if (na) {
            n = na;
        } else if (!opt.segment_nfft || autoseg) {
            const float min_eff = 0.8f;
            while ((double)n * (1.0 - (double)min_eff) < (double)max_delay) n *= 2;
        }
        if (n <= max_delay) DD_THROW_MSG(DEDISP_TOO_FEW_NSAMPS, "segment shorter than max delay");
        g.nfft = n;
        g.nsamp_good = n - max_delay;
        g.nchunk = (size_t)std::ceil((float)nsamps / (float)g.nsamp_good);
        g.timeseries = true;
        g.row_len = nsamps - max_delay;
    } else {
        g.timeseries = opt.output == FddOutput::TimeSeries;
        // Spectrum: round_up(nsamp + max_delay, 16384) (FDDGPUPlan.cpp:89);
        // time series: round_up(nsamp + 1, 16384) (FDDGPUPlan.cpp:86-87).
        const size_t n = g.timeseries ? nsamps + 1 : nsamps + max_delay;
        g.nfft = (n + 16383) / 16384 * 16384;
        g.nsamp_good = nsamps;
        g.nchunk = 1;
        g.row_len = g.timeseries ? nsamps - max_delay : g.nfft;
    }
    g.nbins = g.nfft / 2 + 1;
    return g;
}

}  // namespace detail

FDDGPUPlan::FDDGPUPlan(size_type nchans, float_type dt, float_type f0, float_type df, int device_idx)
    : GPUPlan(nchans, dt, f0, df, device_idx), m_engine(new detail::FddEngine(*m_gpu))
{
}

FDDGPUPlan::~FDDGPUPlan() {}

void FDDGPUPlan::set_options(const FddOptions& opt) { m_opt = opt; }
void FDDGPUPlan::set_timing(bool enable) { m_engine->record_timing = enable; }
ExecTiming FDDGPUPlan::last_timing() const { return m_engine->stats; }
const FddOptions& FDDGPUPlan::get_options() const { return m_opt; }

FDDGPUPlan::size_type FDDGPUPlan::output_row_length(size_type nsamps) const
{
    if (nsamps < m_max_delay) return 0;
    return detail::fdd_geometry(m_opt, nsamps, m_max_delay).row_len;
}

void FDDGPUPlan::execute(size_type nsamps, const byte_type* in, size_type in_nbits,
                         byte_type* out, size_type out_nbits, unsigned flags)
{
    // The reference asserts 8-bit input and float output (FDDGPUPlan.cpp:
    // 66-67); in_nbits 32 (IEEE float samples) and 1/2/4/16-bit packed
    // samples (centred at (2^nbits - 1) / 2 like the 8-bit 127.5) are
    // extensions.
    if (in == nullptr || out == nullptr) DD_THROW(DEDISP_INVALID_POINTER);
    if (m_dm_count == 0) DD_THROW(DEDISP_NO_DM_LIST_SET);
    if (nsamps < m_max_delay) DD_THROW(DEDISP_TOO_FEW_NSAMPS);
    if (in_nbits != 1 && in_nbits != 2 && in_nbits != 4 && in_nbits != 8 && in_nbits != 16 &&
        in_nbits != 32)
        DD_THROW(DEDISP_UNSUPPORTED_IN_NBITS);
    if ((m_nchans * in_nbits) % 8 != 0) DD_THROW(DEDISP_INVALID_STRIDE);
    if (out_nbits != 32) DD_THROW(DEDISP_UNSUPPORTED_OUT_NBITS);
    detail::FddView v{m_nchans, m_dt, h_delay_table.data(), h_killmask.data(),
                      h_dm_list.data(), m_dm_count, m_max_delay, m_state_version};
    detail::FddCall c{nsamps, in, (int)in_nbits, out, flags};
    m_engine->execute(m_opt, v, c);
}

}  // namespace dedisp
