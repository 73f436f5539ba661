// Execution engine behind FDDGPUPlan.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "fdd/FDDGPUPlan.hpp"
#include "gpu_state.hpp"

namespace dedisp {
namespace detail {

struct FddView {
    size_t nchans;
    float dt;
    const float* delays;
    const int32_t* killmask;
    const float* dms;
    size_t ndm;
    size_t max_delay;
    unsigned long version;
};

struct FddCall {
    size_t nsamps;
    const uint8_t* in;
    int in_nbits;      // 8 or 32 (float)
    uint8_t* out;      // float rows of output_row_length() each
    unsigned flags;
};

// Geometry of one FDD execution, restating src/fdd/FDDGPUPlan.cpp:85-93
// (whole series) and :742-777 with src/fdd/chunk.cpp:26-63 (segmented).
struct FddGeometry {
    bool segmented = false;
    bool timeseries = false;
    size_t nfft = 0;        // transform length
    size_t nsamp_good = 0;  // segmented: output samples per segment
    size_t nchunk = 1;      // segments
    size_t nbins = 0;       // bins computed per segment (nfft/2 + 1)
    size_t row_len = 0;     // floats per output row
};
// ndm, nchans (active channels): used by the automatic segment length only.
FddGeometry fdd_geometry(const FddOptions& opt, size_t nsamps, size_t max_delay, size_t ndm = 0,
                         size_t nchans = 0);
// Segmented FDD, tensor-core MAC: the power-of-two segment length (2^11..2^20,
// above the max delay) with the least modelled device time for the DM count
// and the active channels; 0 if none exceeds the max delay (the reference
// rule then applies).
size_t fdd_auto_segment(size_t nsamps, size_t max_delay, size_t ndm, size_t nchans);

class FddEngine {
public:
    explicit FddEngine(GpuState& gpu);
    ~FddEngine();
    void execute(const FddOptions& opt, const FddView& v, const FddCall& c);
    bool record_timing = false;
    ExecTiming stats;

private:
    struct Impl;
    GpuState& m_gpu;
    std::unique_ptr<Impl> m_impl;
};

}  // namespace detail
}  // namespace dedisp
