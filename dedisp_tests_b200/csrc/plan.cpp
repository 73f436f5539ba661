// dedisp::Plan -- host-side plan state.
//
// Restates the reference arithmetic that defines every integer delay:
//   delay table   src/Plan.cpp:29-36,109-119
//   DM list       src/Plan.cpp:45-70,136-154
//   max delay     src/Plan.cpp:85-86,152-153
// Compiled with -ffp-contract=off so each float/double operation rounds once,
// in the reference's order and types.
#include "Plan.hpp"

#include <cuda_runtime.h>

#include <cmath>

#include "errors.hpp"
#include "host_math.hpp"
#include "runtime.hpp"

namespace dedisp {

Plan::Plan(size_type nchans, float_type dt, float_type f0, float_type df)
{
    m_dm_count = 0;
    m_nchans = nchans;
    m_max_delay = 0;
    m_dt = dt;
    m_f0 = f0;
    m_df = df;  // the getter reports the caller's sign (src/Plan.cpp:27)

    h_delay_table.resize(nchans);
    hostmath::delay_table(nchans, dt, f0, df, h_delay_table.data());
    h_killmask.assign(nchans, (dedisp_bool)1);
}

Plan::~Plan() {}

void Plan::generate_dm_list(float_type dm_start, float_type dm_end, float_type ti,
                            float_type tol)
{
    std::vector<float> list;
    if (!hostmath::generate_dm_list(list, dm_start, dm_end, (double)m_dt, (double)ti,
                                    (double)m_f0, (double)m_df, m_nchans, (double)tol))
        DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "DM list recurrence does not advance");
    h_dm_list.swap(list);
    m_dm_count = h_dm_list.size();
    m_max_delay = hostmath::max_delay(h_dm_list.back(), h_delay_table[m_nchans - 1]);
    ++m_state_version;
}

void Plan::set_dm_list(const float_type* dm_list, size_type count)
{
    if (!dm_list) DD_THROW(DEDISP_INVALID_POINTER);
    h_dm_list.assign(dm_list, dm_list + count);
    m_dm_count = count;
    // An empty list leaves no DM to compute (the reference reads element -1).
    m_max_delay = count ? hostmath::max_delay(h_dm_list[count - 1],
                                              h_delay_table[m_nchans - 1])
                        : 0;
    ++m_state_version;
}

void Plan::set_killmask(const bool_type* killmask)
{
    if (killmask) h_killmask.assign(killmask, killmask + m_nchans);
    else std::fill(h_killmask.begin(), h_killmask.end(), (dedisp_bool)1);
    ++m_state_version;
}

void Plan::sync()
{
    if (rt::device_count() > 0) RT_CHECK(cudaDeviceSynchronize());
}

}  // namespace dedisp
