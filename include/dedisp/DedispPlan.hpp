/*
 * DedispPlan.hpp -- the original dedisp plan interface.
 *
 * Same public surface as the reference dedisp::DedispPlan
 * (src/dedisp/DedispPlan.hpp:21-66), including the flags argument of
 * execute_adv / execute_guru. The reference legacy path computes exactly the
 * TDD sums and epilogue (src/dedisp/dedisperse/dedisperse_kernel.cuh:66-81,
 * 151-205), so this class runs on the same B200 engine as TDDPlan.
 */
#ifndef DEDISP_B200_DEDISPPLAN_HPP
#define DEDISP_B200_DEDISPPLAN_HPP

#include "tdd/TDDPlan.hpp"

namespace dedisp {

class DedispPlan : public GPUPlan {
public:
    DedispPlan(size_type nchans, float_type dt, float_type f0, float_type df,
               int device_idx = 0);
    ~DedispPlan();

    void set_gulp_size(size_type gulp_size);
    size_type get_gulp_size() const;

    void execute(size_type nsamps, const byte_type* in, size_type in_nbits,
                 byte_type* out, size_type out_nbits,
                 unsigned flags = 0) override;

    void execute_adv(size_type nsamps, const byte_type* in,
                     size_type in_nbits, size_type in_stride, byte_type* out,
                     size_type out_nbits, size_type out_stride,
                     unsigned flags);

    void execute_guru(size_type nsamps, const byte_type* in,
                      size_type in_nbits, size_type in_stride,
                      byte_type* out, size_type out_nbits,
                      size_type out_stride, dedisp_size first_dm_idx,
                      dedisp_size dm_count, unsigned flags);

    void set_kernel(TddKernel k);
    void set_tile_variant(int variant);
    void set_timing(bool enable) override;
    ExecTiming last_timing() const override;

private:
    std::unique_ptr<detail::TddEngine> m_engine;
};

}  // namespace dedisp

#endif  // DEDISP_B200_DEDISPPLAN_HPP
