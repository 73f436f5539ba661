// Execution engine behind TDDPlan and DedispPlan.
//
// One call = validate-free execution of a (sub-)range of the DM list over a
// time series, in gulps of output samples:
//   host rows --(H2D, pinned or pageable)--> gulp input buffer --K1d-->
//   quad-strided rows (quad variants; K1: channel-major packed rows for the
//   others) --K2--> output --(D2H)--> host rows. With several gulps, input and
//   output buffers are doubled so that the copies of neighbouring gulps
//   overlap a gulp's kernels; the last gulp's K2 and D2H run per DM group.
// With DEDISP_DEVICE_POINTERS the copies disappear and K1d/K1/K2 read/write
// the caller's buffers. Derived per-plan state (active channels, sorted DMs,
// window sizes) is cached until the DM list or killmask changes.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "gpu_state.hpp"
#include "tdd/TDDPlan.hpp"

namespace dedisp {
namespace detail {

struct TddView {
    size_t nchans;
    const float* delays;
    const int32_t* killmask;
    const float* dms;
    size_t ndm_total;
    size_t max_delay;
    unsigned long version;
};

struct TddCall {
    size_t nsamps;
    const uint8_t* in;
    int in_nbits;
    size_t in_stride;   // bytes
    uint8_t* out;
    int out_nbits;
    size_t out_stride;  // bytes
    size_t first_dm;
    size_t dm_count;
    unsigned flags;
};

// Timing of the last execute() (device time of the dedispersion kernels,
// measured with events on the execution stream; 0 when not recorded).
struct TddStats {
    float kernel_ms = 0.f;
    float transpose_ms = 0.f;
    int launches = 0;
    bool tiled = false;
};

class TddEngine {
public:
    // Gulp (output samples per pass) unless set: device-resident calls take
    // the largest; calls with host buffers take smaller gulps so that the
    // host copies of neighbouring gulps overlap the kernels.
    static constexpr size_t kDefaultGulp = (size_t)1 << 21;
    static constexpr size_t kHostDefaultGulp = (size_t)1 << 18;

    explicit TddEngine(GpuState& gpu);
    ~TddEngine();

    void execute(const TddView& v, const TddCall& c);

    size_t gulp_size = kDefaultGulp;
    bool gulp_set = false;  // gulp_size was set by the caller
    TddKernel kernel = TddKernel::Auto;
    int variant = -1;  // tile-shape variant of the tiled kernel (8-bit input; -1: default)
    bool record_timing = false;
    TddStats stats;

private:
    struct Setup;
    void prepare(const TddView& v, const TddCall& c);

    GpuState& m_gpu;
    std::unique_ptr<Setup> m_setup;
    rt::DeviceBuffer m_chan, m_cdl, m_km, m_dms, m_perm, m_tr, m_q, m_out[2], m_stage[2];
    rt::DeviceBuffer m_err;  // set by a quad-strided kernel whose bounded wait expired
    std::vector<std::unique_ptr<rt::Event>> m_events;
    rt::Event& event(size_t i);
};

}  // namespace detail
}  // namespace dedisp
