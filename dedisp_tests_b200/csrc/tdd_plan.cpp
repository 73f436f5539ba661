// TDDPlan and DedispPlan: argument validation in the reference order, then
// the shared TDD engine.
//   TDDPlan::execute*     src/tdd/TDDPlan.cpp:102-195
//   DedispPlan::execute*  src/dedisp/DedispPlan.cpp:53-154
#include "dedisp/DedispPlan.hpp"
#include "tdd/TDDPlan.hpp"

#include "gpu_state.hpp"
#include "tdd_engine.hpp"

namespace dedisp {

namespace {

// Maximum channel count of the reference TDD/dedisp plans: its kernels keep
// the delay table and killmask in 64 KB of constant memory
// (src/tdd/TDDPlan.cpp:52-54,76-82, src/dedisp/DedispPlan.cpp:32-34).
constexpr size_t kMaxChans = 8192;

bool valid_in_nbits(size_t n)
{
    return n == 1 || n == 2 || n == 4 || n == 8 || n == 16 || n == 32;
}

// Checks of TDDPlan.cpp:167-195 / DedispPlan.cpp:121-154, same order and
// the same unsigned arithmetic (nsamps < max_delay wraps, so it is reported
// as DEDISP_INVALID_STRIDE exactly like the reference).
void validate(size_t nchans, size_t dm_count_total, size_t max_delay, size_t nsamps,
              const void* in, size_t in_nbits, size_t in_stride, const void* out,
              size_t out_nbits, size_t out_stride, bool check_flags, unsigned flags)
{
    const size_t out_bytes = out_nbits / 8;
    if (in == nullptr || out == nullptr) DD_THROW(DEDISP_INVALID_POINTER);
    if (in_stride < nchans * in_nbits / 8 || out_stride < (nsamps - max_delay) * out_bytes)
        DD_THROW(DEDISP_INVALID_STRIDE);
    if (dm_count_total == 0) DD_THROW(DEDISP_NO_DM_LIST_SET);
    if (nsamps < max_delay) DD_THROW(DEDISP_TOO_FEW_NSAMPS);
    if (check_flags && (flags & DEDISP_ASYNC) && (flags & DEDISP_WAIT))
        DD_THROW(DEDISP_INVALID_FLAG_COMBINATION);
    if (!valid_in_nbits(in_nbits)) DD_THROW(DEDISP_UNSUPPORTED_IN_NBITS);
    if (out_nbits != 8 && out_nbits != 16 && out_nbits != 32) DD_THROW(DEDISP_UNSUPPORTED_OUT_NBITS);
    // Beyond the reference: it silently drops a partial last channel word.
    if ((nchans * in_nbits) % 32 != 0)
        DD_THROW_MSG(DEDISP_UNSUPPORTED_IN_NBITS, "nchans * in_nbits must be a multiple of 32");
}

}  // namespace

// ---------------------------------------------------------------------------
// TDDPlan
// ---------------------------------------------------------------------------
TDDPlan::TDDPlan(size_type nchans, float_type dt, float_type f0, float_type df, int device_idx)
    : GPUPlan(nchans, dt, f0, df, device_idx)
{
    if (nchans > kMaxChans) DD_THROW(DEDISP_NCHANS_EXCEEDS_LIMIT);
    m_engine.reset(new detail::TddEngine(*m_gpu));
}

TDDPlan::~TDDPlan() {}

void TDDPlan::set_gulp_size(size_type gulp_size)
{
    m_engine->gulp_size = gulp_size;
    m_engine->gulp_set = true;
}
dedisp_size TDDPlan::get_gulp_size() const { return m_engine->gulp_size; }
void TDDPlan::set_kernel(TddKernel k) { m_engine->kernel = k; }
void TDDPlan::set_tile_variant(int variant) { m_engine->variant = variant; }
void TDDPlan::set_timing(bool enable) { m_engine->record_timing = enable; }
ExecTiming TDDPlan::last_timing() const
{
    ExecTiming t;
    t.kernel_ms = m_engine->stats.kernel_ms;
    t.prep_ms = m_engine->stats.transpose_ms;
    t.launches = m_engine->stats.launches;
    t.variant = m_engine->stats.tiled ? 1 : 0;
    return t;
}

void TDDPlan::execute(size_type nsamps, const byte_type* in, size_type in_nbits,
                      byte_type* out, size_type out_nbits, unsigned flags)
{
    const size_type ob = out_nbits / 8;
    const size_type in_stride = m_nchans * in_nbits / 8;
    const size_type out_stride = (nsamps - m_max_delay) * ob;
    execute_guru_flags(nsamps, in, in_nbits, in_stride, out, out_nbits, out_stride, 0,
                       m_dm_count, flags);
}

void TDDPlan::execute_adv(size_type nsamps, const byte_type* in, size_type in_nbits,
                          size_type in_stride, byte_type* out, size_type out_nbits,
                          size_type out_stride)
{
    execute_guru_flags(nsamps, in, in_nbits, in_stride, out, out_nbits, out_stride, 0,
                       m_dm_count, 0);
}

void TDDPlan::execute_guru(size_type nsamps, const byte_type* in, size_type in_nbits,
                           size_type in_stride, byte_type* out, size_type out_nbits,
                           size_type out_stride, dedisp_size first_dm_idx, dedisp_size dm_count)
{
    execute_guru_flags(nsamps, in, in_nbits, in_stride, out, out_nbits, out_stride,
                       first_dm_idx, dm_count, 0);
}

void TDDPlan::execute_guru_flags(size_type nsamps, const byte_type* in, size_type in_nbits,
                                 size_type in_stride, byte_type* out, size_type out_nbits,
                                 size_type out_stride, dedisp_size first_dm_idx,
                                 dedisp_size dm_count, unsigned flags)
{
    validate(m_nchans, m_dm_count, m_max_delay, nsamps, in, in_nbits, in_stride, out, out_nbits,
             out_stride, false, flags);
    if (first_dm_idx > m_dm_count || dm_count > m_dm_count - first_dm_idx)
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "DM range outside the DM list");
    detail::TddView v{m_nchans, h_delay_table.data(), h_killmask.data(), h_dm_list.data(),
                      m_dm_count, m_max_delay, m_state_version};
    detail::TddCall c{nsamps, in, (int)in_nbits, in_stride, out, (int)out_nbits, out_stride,
                      first_dm_idx, dm_count, flags};
    m_engine->execute(v, c);
}

// ---------------------------------------------------------------------------
// DedispPlan
// ---------------------------------------------------------------------------
DedispPlan::DedispPlan(size_type nchans, float_type dt, float_type f0, float_type df,
                       int device_idx)
    : GPUPlan(nchans, dt, f0, df, device_idx)
{
    if (nchans > kMaxChans) DD_THROW(DEDISP_NCHANS_EXCEEDS_LIMIT);
    m_engine.reset(new detail::TddEngine(*m_gpu));
}

DedispPlan::~DedispPlan() {}

void DedispPlan::set_gulp_size(size_type gulp_size)
{
    m_engine->gulp_size = gulp_size;
    m_engine->gulp_set = true;
}
DedispPlan::size_type DedispPlan::get_gulp_size() const { return m_engine->gulp_size; }
void DedispPlan::set_kernel(TddKernel k) { m_engine->kernel = k; }
void DedispPlan::set_tile_variant(int variant) { m_engine->variant = variant; }
void DedispPlan::set_timing(bool enable) { m_engine->record_timing = enable; }
ExecTiming DedispPlan::last_timing() const
{
    ExecTiming t;
    t.kernel_ms = m_engine->stats.kernel_ms;
    t.prep_ms = m_engine->stats.transpose_ms;
    t.launches = m_engine->stats.launches;
    t.variant = m_engine->stats.tiled ? 1 : 0;
    return t;
}

void DedispPlan::execute(size_type nsamps, const byte_type* in, size_type in_nbits,
                         byte_type* out, size_type out_nbits, unsigned flags)
{
    const size_type ob = out_nbits / 8;
    const size_type in_stride = m_nchans * in_nbits / 8;
    const size_type out_stride = (nsamps - m_max_delay) * ob;
    execute_guru(nsamps, in, in_nbits, in_stride, out, out_nbits, out_stride, 0, m_dm_count,
                 flags);
}

void DedispPlan::execute_adv(size_type nsamps, const byte_type* in, size_type in_nbits,
                             size_type in_stride, byte_type* out, size_type out_nbits,
                             size_type out_stride, unsigned flags)
{
    execute_guru(nsamps, in, in_nbits, in_stride, out, out_nbits, out_stride, 0, m_dm_count,
                 flags);
}

void DedispPlan::execute_guru(size_type nsamps, const byte_type* in, size_type in_nbits,
                              size_type in_stride, byte_type* out, size_type out_nbits,
                              size_type out_stride, dedisp_size first_dm_idx,
                              dedisp_size dm_count, unsigned flags)
{
    validate(m_nchans, m_dm_count, m_max_delay, nsamps, in, in_nbits, in_stride, out, out_nbits,
             out_stride, true, flags);
    if (first_dm_idx > m_dm_count || dm_count > m_dm_count - first_dm_idx)
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "DM range outside the DM list");
    detail::TddView v{m_nchans, h_delay_table.data(), h_killmask.data(), h_dm_list.data(),
                      m_dm_count, m_max_delay, m_state_version};
    detail::TddCall c{nsamps, in, (int)in_nbits, in_stride, out, (int)out_nbits, out_stride,
                      first_dm_idx, dm_count, flags};
    m_engine->execute(v, c);
}

}  // namespace dedisp
