// Batched multi-beam Fourier-domain dedispersion (no counterpart in the
// reference, whose FDDGPUPlan dedisperses one series per execute call,
// src/fdd/FDDGPUPlan.cpp:429-546 and :725-1271).
//
// Beams share the channel setup (nchans, dt, f0, df, killmask, input width)
// and each has its own device input, sample count, DM list and device output
// (dm_count rows of nsamps - max_delay floats: the segmented overlap-save
// time series, segment length from the reference doubling rule). One
// execute() enqueues, per beam, the unpack, the forward real FFTs and the
// split B operand of each segment group, then one persistent tensor-core
// (3xBF16) MAC launch over a work list of (beam segment group, DM tiles, bin
// range) items of all beams per MMA-form class (segment groups of at most 32
// MMA columns take the wide fused form, wider ones the three-MMA form: at
// most two launches), then per beam the DM-major transpose and the
// inverse FFTs straight into the caller's rows. The sequence is captured once
// into a CUDA graph and replayed. Results equal those of an FDDGPUPlan per
// beam (segmented, tensor-core precision), which is what the tests check.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <vector>

#include "fdd_engine.hpp"
#include "fdd_kernels.hpp"
#include "fdd_tc.hpp"
#include "runtime.hpp"
#include "tdd_kernels.hpp"

namespace dedisp {
namespace detail {

struct FddBeamSpec {
    const uint8_t* in;    // device, time-major rows
    size_t in_stride;     // bytes per input row
    size_t nsamps;
    std::vector<float> dms;
    uint8_t* out;         // device, dm_count rows of nsamps - max_delay floats
    size_t out_stride;    // bytes per output row
};

class FddBatch {
public:
    FddBatch(size_t nchans, float dt, float f0, float df, int in_nbits, int device);
    ~FddBatch();

    void set_killmask(const int32_t* killmask);  // nullptr: all channels
    // Segment length of every beam: 0 the reference doubling rule (default),
    // FddOptions::kSegmentAuto the least modelled time per beam, else that
    // power of two. Takes effect at the next set_beams.
    void set_segment_nfft(size_t n) { m_segment_nfft = n; }
    void set_beams(std::vector<FddBeamSpec> beams);
    size_t beam_count() const { return m_beams.size(); }
    size_t max_delay(size_t beam) const;
    // Phasor source of a beam's tensor-core MAC as planned by set_beams (the
    // codes of dedisp_b200_get_phasor_source); -1 when it has no MAC work.
    int phasor_source(size_t beam) const;
    size_t nsamp_out(size_t beam) const;

    // Device bytes of scratch and per-beam operands the batch needs.
    size_t workspace_bytes() const;
    // Caller-owned scratch (device, >= workspace_bytes()); nullptr: own.
    void set_workspace(void* ptr, size_t bytes);

    // Enqueues the whole batch on `stream` (graph: captured once, replayed).
    void execute(cudaStream_t stream, bool use_graph);
    // Waits for `stream`; DEDISP_INTERNAL_GPU_ERROR if a bounded wait of the
    // last execute's MAC expired.
    void sync(cudaStream_t stream);

    // With timing on, execute waits for its work and reports the device time
    // of the preparation (unpack, FFT, B operand), of the MAC launch and of the
    // inverse side (in graph mode: the whole graph as mac_ms, the others -1).
    bool record_timing = false;
    float last_prep_ms = 0.f, last_mac_ms = 0.f, last_post_ms = 0.f;
    int last_launches = 0;
    // Direct (non-graph) executes with timing on: the MAC's CTAs' busy times,
    // largest and mean (ms), to show how evenly the work list spreads.
    float last_cta_max_ms = 0.f, last_cta_mean_ms = 0.f;

private:
    struct Beam;
    void plan();                       // geometry, modes, workspace offsets
    void upload();                     // per-beam tables, work list
    void enqueue(cudaStream_t s, bool timing);
    void drop_graph();
    uint8_t* workspace_base();

    size_t m_nchans;
    int m_nbits, m_device;
    float m_dt;
    std::vector<float> m_delays;       // nchans
    std::vector<int32_t> m_km;
    std::vector<std::unique_ptr<Beam>> m_beams;
    bool m_dirty = true;
    size_t m_segment_nfft = 0;
    int m_nact = 0, m_nact_pad = 0;
    size_t m_ws_bytes = 0, m_shared_bytes = 0, m_scratch_off = 0, m_scratch_bytes = 0;

    rt::DeviceBuffer m_chan, m_kmv, m_delay_pad, m_err, m_twp_lo, m_twp_hi;
    // MAC launches: one per MMA-form class of the beams' segment groups
    // (at most 32 columns: the wide fused form; more: the three-MMA form)
    rt::DeviceBuffer m_items[2], m_cta_ns[2];
    rt::DeviceBuffer m_own_ws;
    void* m_ext_ws = nullptr;
    size_t m_ext_ws_bytes = 0;
    std::unique_ptr<kern::TcParams> m_params[2];
    cudaGraph_t m_graph = nullptr;
    cudaGraphExec_t m_exec = nullptr;
    int m_graph_launches = 0;
    std::unique_ptr<rt::Event> m_ev[4];
};

}  // namespace detail
}  // namespace dedisp
