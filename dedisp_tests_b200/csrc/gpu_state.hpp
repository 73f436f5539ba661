// Device state owned by every GPU plan (the CUDA side of dedisp::GPUPlan).
#pragma once

#include <memory>

#include "runtime.hpp"

namespace dedisp {
namespace detail {

struct GpuState {
    bool has_device = false;
    int device = 0;
    std::unique_ptr<rt::Stream> exec;  // kernels
    std::unique_ptr<rt::Stream> h2d;   // host -> device copies
    std::unique_ptr<rt::Stream> d2h;   // device -> host copies
    cudaStream_t user_stream = nullptr;
    // Delay table, nchans + 1 floats; the extra entry (0) belongs to the
    // all-zero padding channel used by the kernels.
    rt::DeviceBuffer delay_table;

    cudaStream_t stream() const { return user_stream ? user_stream : exec->get(); }
    void require_device() const
    {
        if (!has_device)
            DD_THROW_MSG(DEDISP_INTERNAL_GPU_ERROR, "no CUDA device available for this plan");
    }
};

}  // namespace detail
}  // namespace dedisp
