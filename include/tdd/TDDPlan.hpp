/*
 * TDDPlan.hpp -- time-domain (brute-force) dedispersion on one B200.
 *
 * Same public surface as the reference dedisp::TDDPlan (src/tdd/TDDPlan.hpp:
 * 17-57): gulp size, execute, execute_adv (byte strides) and execute_guru
 * (a range of the DM list). Results are bit-identical to the reference
 * (integer sums, src/tdd/dedisperse/dedisperse_kernel.cuh:98-198, and its
 * FP32 epilogue :45-87).
 */
#ifndef DEDISP_B200_TDDPLAN_HPP
#define DEDISP_B200_TDDPLAN_HPP

#include "GPUPlan.hpp"

namespace dedisp {

namespace detail {
class TddEngine;
}

/* Kernel choice (extension). Auto picks the tiled shared-memory kernel
 * whenever the killmask holds only 0/1 values; Plain is the one-thread-per-
 * sample-pair form kept as the comparison baseline. */
enum class TddKernel { Auto = 0, Plain = 1, Tiled = 2 };

class TDDPlan : public GPUPlan {
public:
    TDDPlan(size_type nchans, float_type dt, float_type f0, float_type df,
            int device_idx = 0);
    ~TDDPlan();

    /* Maximum number of output samples computed per device pass. */
    void set_gulp_size(size_type gulp_size);
    dedisp_size get_gulp_size() const;

    void execute(size_type nsamps, const byte_type* in, size_type in_nbits,
                 byte_type* out, size_type out_nbits,
                 unsigned flags = 0) override;

    void execute_adv(size_type nsamps, const byte_type* in,
                     size_type in_nbits, size_type in_stride, byte_type* out,
                     size_type out_nbits, size_type out_stride);

    void execute_guru(size_type nsamps, const byte_type* in,
                      size_type in_nbits, size_type in_stride,
                      byte_type* out, size_type out_nbits,
                      size_type out_stride, dedisp_size first_dm_idx,
                      dedisp_size dm_count);

    /* Extensions: flags-aware guru call (DEDISP_DEVICE_POINTERS,
     * DEDISP_ASYNC) and kernel selection. */
    void execute_guru_flags(size_type nsamps, const byte_type* in,
                            size_type in_nbits, size_type in_stride,
                            byte_type* out, size_type out_nbits,
                            size_type out_stride, dedisp_size first_dm_idx,
                            dedisp_size dm_count, unsigned flags);
    void set_kernel(TddKernel k);
    void set_tile_variant(int variant);
    void set_timing(bool enable) override;
    ExecTiming last_timing() const override;

protected:
    std::unique_ptr<detail::TddEngine> m_engine;
};

}  // namespace dedisp

#endif  // DEDISP_B200_TDDPLAN_HPP
