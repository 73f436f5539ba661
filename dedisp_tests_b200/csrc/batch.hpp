// Batched multi-beam time-domain dedispersion (no counterpart in the
// reference, whose plans dedisperse one series per execute call).
//
// Many beams share one channel setup (nchans, dt, f0, df, killmask, input and
// output widths) but each has its own device input, sample count, DM list and
// device output. One execute() enqueues, per beam, the padding-row reset and
// the K1 transpose into a shared workspace, then ONE persistent K2 launch
// whose blocks walk a work list of (beam, DM block, time tile) items across
// all beams (8-bit input with a 0/1 killmask; other cases launch K2 per beam).
// The whole sequence is captured once into a CUDA graph and replayed.
//
// Tile shape (DMs per block, samples per thread, channels per stage) is set
// explicitly or chosen by autotune(), which times every candidate on the
// leading tiles of the beams with CUDA events.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <vector>

#include "runtime.hpp"
#include "tdd_kernels.hpp"

namespace dedisp {
namespace detail {

struct BatchBeamSpec {
    const uint8_t* in;    // device, time-major packed rows
    size_t in_stride;     // bytes per input row
    size_t nsamps;
    std::vector<float> dms;
    uint8_t* out;         // device, dm_count rows
    size_t out_stride;    // bytes per output row
};

struct BatchShape {
    int variant = 0;         // tiled-kernel tile-shape variant (a batch starts at its width's default)
    int chan_per_stage = 0;  // 0: the largest that fits shared memory
};

class TddBatch {
public:
    TddBatch(size_t nchans, float dt, float f0, float df, int in_nbits, int out_nbits, int device);
    ~TddBatch();

    void set_killmask(const int32_t* killmask);  // nullptr: all channels
    void set_beams(std::vector<BatchBeamSpec> beams);
    void set_shape(const BatchShape& shape);
    BatchShape shape() const { return m_shape; }

    // Device bytes of transposed-input scratch needed by any tile shape.
    size_t workspace_bytes() const;
    // Caller-owned scratch (device, >= workspace_bytes()); nullptr: own.
    void set_workspace(void* ptr, size_t bytes);

    // Times every candidate shape on the leading time tiles of all beams
    // and keeps the fastest. Runs work on `stream` and waits for it.
    BatchShape autotune(cudaStream_t stream);

    // Enqueues the whole batch on `stream` (graph: captured once, replayed).
    void execute(cudaStream_t stream, bool use_graph);
    // Waits for `stream` and throws DEDISP_INTERNAL_GPU_ERROR if a bounded
    // wait of the last execute's dedispersion expired.
    void sync(cudaStream_t stream);

    size_t beam_count() const { return m_beams.size(); }
    size_t max_delay(size_t beam) const;
    size_t nsamp_out(size_t beam) const;

    // With timing on, execute waits for its work and reports the device time
    // of the transposes (k1; -1 in graph mode, where they are inside the
    // graph) and of the dedispersion (k2; in graph mode the whole graph).
    bool record_timing = false;
    float last_k2_ms = 0.f;
    float last_k1_ms = 0.f;
    int last_launches = 0;

private:
    struct BeamState;
    struct Layout;
    Layout make_layout(const BatchShape& shape, size_t tile_limit_samples) const;
    void upload(Layout& L);
    void enqueue(cudaStream_t s, const Layout& L, bool timing);
    void drop_graph();
    uint8_t* workspace_base();

    size_t m_nchans;
    int m_nbits, m_out_nbits, m_device;
    std::vector<float> m_delays;     // nchans + 1 (last 0)
    std::vector<int32_t> m_km;
    bool m_general_mask = false;
    std::vector<int32_t> m_chan;     // active channels
    std::vector<uint32_t> m_kmv;
    std::vector<BeamState> m_beams;
    BatchShape m_shape;
    std::unique_ptr<Layout> m_layout;  // uploaded layout for m_shape
    bool m_dirty = true;

    rt::DeviceBuffer m_d_delay, m_d_chan, m_d_cdl, m_d_kmv, m_d_dms, m_d_perm, m_d_args, m_d_start, m_d_nbx;
    rt::DeviceBuffer m_d_err;  // set by a quad-strided kernel whose bounded wait expired
    rt::DeviceBuffer m_own_ws;
    void* m_ext_ws = nullptr;
    size_t m_ext_ws_bytes = 0;
    cudaGraph_t m_graph = nullptr;
    cudaGraphExec_t m_exec = nullptr;
    int m_graph_launches = 0;     // kernel launches inside the captured graph
    std::unique_ptr<rt::Event> m_ev[3];
};

}  // namespace detail
}  // namespace dedisp
