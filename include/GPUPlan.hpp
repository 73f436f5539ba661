/*
 * GPUPlan.hpp -- device side shared by the GPU plans (namespace dedisp).
 *
 * Replaces the reference class dedisp::GPUPlan (src/GPUPlan.hpp:15-57): it
 * binds the plan to a CUDA device and keeps device copies of the DM list,
 * delay table and killmask. The CUDA objects live behind an opaque state
 * pointer so this header needs no CUDA include.
 */
#ifndef DEDISP_B200_GPUPLAN_HPP
#define DEDISP_B200_GPUPLAN_HPP

#include "Plan.hpp"

namespace dedisp {

namespace detail {
struct GpuState;
}

/* Device time of the last execute() when timing is enabled (extension). */
struct ExecTiming {
    float kernel_ms = 0.f;   /* dedispersion kernels */
    float prep_ms = 0.f;     /* transpose / unpack + forward FFT */
    int launches = 0;        /* dedispersion kernel launches */
    int variant = 0;         /* kernel form actually used (plan specific) */
    /* FDD plans: device time of each stage (ms), in pipeline order: unpack,
     * forward FFT, operand layout (B split or bin-major), MAC, DM-major
     * transpose or spectrum output, inverse FFT (0 when a stage did not run) */
    float stage_ms[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    /* FDD plans, tensor-core MAC: phasor source of the last execute (0 the
     * per-bin delay table, 1 the quarter-wave table, 2 the table for small
     * delays with the rest computed, 3 computed from twiddle tables); -1 none */
    int phasor = -1;
    /* FDD plans: MMA form of the last tensor-core MAC launch (0 three MMAs per
     * K step, 1 fused, 2 three MMAs with 3 A buffers, 3 CTA pairs (M = 256),
     * 4 CTA pairs with 3 A buffers, 5 fused at 64-channel chunks); -1 none */
    int tc_form = -1;
};

class GPUPlan : public Plan {
protected:
    GPUPlan(size_type nchans, float_type dt, float_type f0, float_type df,
            int device_idx = 0);

public:
    GPUPlan(const GPUPlan&) = delete;
    GPUPlan& operator=(const GPUPlan&) = delete;
    virtual ~GPUPlan();

    void generate_dm_list(float_type dm_start, float_type dm_end,
                          float_type ti, float_type tol) override;
    void set_dm_list(const float_type* dm_list, size_type count) override;
    void set_killmask(const bool_type* killmask) override;

    /* Extension: run this plan's device work on the given cudaStream_t
     * (nullptr restores the plan's own stream). */
    void set_stream(void* cuda_stream);

    int get_device() const { return m_device_idx; }

    /* Extension: record CUDA events around the device stages of execute(). */
    virtual void set_timing(bool enable) { (void)enable; }
    virtual ExecTiming last_timing() const { return ExecTiming(); }

protected:
    int m_device_idx;
    std::unique_ptr<detail::GpuState> m_gpu;
};

}  // namespace dedisp

#endif  // DEDISP_B200_GPUPLAN_HPP
