// dedisp::GPUPlan -- binds a plan to a device (src/GPUPlan.cpp:12-82).
//
// Unlike the reference, a process without any CUDA device can still build a
// plan and use its host-side setters and getters; execute() then fails.
#include "GPUPlan.hpp"

#include <vector>

#include "gpu_state.hpp"

namespace dedisp {

GPUPlan::GPUPlan(size_type nchans, float_type dt, float_type f0, float_type df,
                 int device_idx)
    : Plan(nchans, dt, f0, df), m_device_idx(device_idx),
      m_gpu(new detail::GpuState())
{
    const int ndev = rt::device_count();
    if (ndev == 0) return;  // host-only plan
    if (device_idx < 0 || device_idx >= ndev) DD_THROW(DEDISP_INVALID_DEVICE_INDEX);
    rt::DeviceGuard guard(device_idx);
    m_gpu->has_device = true;
    m_gpu->device = device_idx;
    m_gpu->exec.reset(new rt::Stream());
    m_gpu->h2d.reset(new rt::Stream());
    m_gpu->d2h.reset(new rt::Stream());
    std::vector<float> table(h_delay_table);
    table.push_back(0.f);
    m_gpu->delay_table.reserve(table.size() * sizeof(float));
    RT_CHECK(cudaMemcpy(m_gpu->delay_table.get(), table.data(), table.size() * sizeof(float),
                        cudaMemcpyHostToDevice));
}

GPUPlan::~GPUPlan()
{
    if (m_gpu && m_gpu->has_device) {
        rt::DeviceGuard guard(m_gpu->device);
        cudaStreamSynchronize(m_gpu->stream());
    }
}

// The DM list and killmask are uploaded by the engines when they next run
// (they track Plan::m_state_version), so the setters stay host-only.
void GPUPlan::generate_dm_list(float_type dm_start, float_type dm_end, float_type ti,
                               float_type tol)
{
    Plan::generate_dm_list(dm_start, dm_end, ti, tol);
}

void GPUPlan::set_dm_list(const float_type* dm_list, size_type count)
{
    Plan::set_dm_list(dm_list, count);
}

void GPUPlan::set_killmask(const bool_type* killmask) { Plan::set_killmask(killmask); }

void GPUPlan::set_stream(void* cuda_stream)
{
    m_gpu->user_stream = static_cast<cudaStream_t>(cuda_stream);
}

}  // namespace dedisp
