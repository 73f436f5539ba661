/*
 * FDDGPUPlan.hpp -- Fourier-domain dedispersion on one B200.
 *
 * Same public surface as the reference dedisp::FDDGPUPlan
 * (src/fdd/FDDGPUPlan.hpp:18-35): construct, set the DM list, execute().
 * Defaults follow this fork of the reference: 8-bit input, the whole series
 * transformed at once with nfft = round_up(nsamps + max_delay, 16384), and
 * the output is the dedispersed Fourier spectrum, nfft floats per DM (the
 * first nfft/2 complex bins, interleaved re/im) -- src/fdd/FDDGPUPlan.cpp:
 * 85-93,394-400. USE_SEGMENTED=1 in the environment selects the segmented
 * (overlap-save) path whose output is a time series of nsamps - max_delay
 * floats per DM (src/fdd/FDDGPUPlan.cpp:42-48,725-1271).
 *
 * Extensions (FddOptions): float32 input (in_nbits = 32), time-series output
 * for the whole-series path, round-to-nearest delays (TDD-compatible), and
 * the precision of the phasor multiply-accumulate (FP32 CUDA cores or the
 * 3xBF16 tensor-core complex GEMM).
 */
#ifndef DEDISP_B200_FDDGPUPLAN_HPP
#define DEDISP_B200_FDDGPUPLAN_HPP

#include "GPUPlan.hpp"

namespace dedisp {

namespace detail {
class FddEngine;
}

enum class FddOutput { Spectrum = 0, TimeSeries = 1 };
enum class FddPrecision { FP32 = 0, BF16x3 = 1 };

struct FddOptions {
    /* -1: read USE_SEGMENTED from the environment at execute time. */
    int segmented = -1;
    FddOutput output = FddOutput::Spectrum;   /* whole-series path only */
    FddPrecision precision = FddPrecision::FP32;
    bool round_delays = false;                /* false: (int) truncation */
    /* 0: reference doubling rule; 1 (kSegmentAuto): with the tensor-core MAC
     * the power of two with the least modelled device time for the plan's
     * DMs and channels (FP32: the reference rule); else the segment length
     * (a power of two above the max delay) */
    size_t segment_nfft = 0;
    static constexpr size_t kSegmentAuto = 1;
};

class FDDGPUPlan : public GPUPlan {
public:
    FDDGPUPlan(size_type nchans, float_type dt, float_type f0, float_type df,
               int device_idx = 0);
    ~FDDGPUPlan();

    void execute(size_type nsamps, const byte_type* in, size_type in_nbits,
                 byte_type* out, size_type out_nbits,
                 unsigned flags = 0) override;

    void set_options(const FddOptions& opt);
    const FddOptions& get_options() const;

    /* Number of floats per DM row that execute() writes for nsamps samples
     * under the current options. */
    size_type output_row_length(size_type nsamps) const;

    void set_timing(bool enable) override;
    ExecTiming last_timing() const override;

private:
    FddOptions m_opt;
    std::unique_ptr<detail::FddEngine> m_engine;
};

}  // namespace dedisp

#endif  // DEDISP_B200_FDDGPUPLAN_HPP
