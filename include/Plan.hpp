/*
 * Plan.hpp -- host side of a dedispersion plan (namespace dedisp).
 *
 * Same public surface as the reference class dedisp::Plan
 * (src/Plan.hpp:36-83): construction from (nchans, dt, f0, df), DM-list
 * generation or assignment, killmask, getters, sync, and a pure virtual
 * execute(). The delay table, DM list and max delay are computed with the
 * reference's arithmetic (src/Plan.cpp:16-40,45-119,136-154) so that every
 * integer delay, and therefore every output sample, matches.
 */
#ifndef DEDISP_B200_PLAN_HPP
#define DEDISP_B200_PLAN_HPP

#include <memory>
#include <vector>

#include "common/dedisp_types.h"

namespace dedisp {

class Plan {
public:
    typedef dedisp_size  size_type;
    typedef dedisp_byte  byte_type;
    typedef dedisp_float float_type;
    typedef dedisp_bool  bool_type;

    /* nchans channels, dt seconds per sample, f0 the highest channel
     * frequency in MHz, df the channel width in MHz (any sign). */
    Plan(size_type nchans, float_type dt, float_type f0, float_type df);

    Plan(const Plan&) = delete;
    Plan& operator=(const Plan&) = delete;
    virtual ~Plan();

    /* Levin's DM-trial spacing (src/Plan.cpp:45-70,136-154); ti is the
     * intrinsic pulse width in microseconds, tol the smearing tolerance. */
    virtual void generate_dm_list(float_type dm_start, float_type dm_end,
                                  float_type ti, float_type tol);

    /* Copies count DMs from the host array (src/Plan.cpp:72-87). */
    virtual void set_dm_list(const float_type* dm_list, size_type count);

    /* One value per channel; nullptr selects every channel
     * (src/Plan.cpp:89-101). */
    virtual void set_killmask(const bool_type* killmask);

    float_type get_max_delay() const { return (float_type)m_max_delay; }
    size_type get_channel_count() const { return m_nchans; }
    size_type get_dm_count() const { return m_dm_count; }
    float_type get_dt() const { return m_dt; }
    float_type get_df() const { return m_df; }
    float_type get_f0() const { return m_f0; }

    const float_type* get_dm_list() const { return h_dm_list.data(); }
    const float_type* get_delay_table() const { return h_delay_table.data(); }
    const bool_type* get_killmask() const { return h_killmask.data(); }

    /* Waits for all device work (src/Plan.cpp:103-106). */
    void sync();

    virtual void execute(size_type nsamps, const byte_type* in,
                         size_type in_nbits, byte_type* out,
                         size_type out_nbits, unsigned flags = 0) = 0;

protected:
    /* Bumped whenever the DM list or killmask changes, so device-side
     * caches know when to refresh. */
    unsigned long m_state_version = 0;

    dedisp_size m_dm_count;
    dedisp_size m_nchans;
    dedisp_size m_max_delay;

    dedisp_float m_dt;
    dedisp_float m_f0;
    dedisp_float m_df;

    std::vector<dedisp_float> h_dm_list;      /* size dm_count */
    std::vector<dedisp_float> h_delay_table;  /* size nchans */
    std::vector<dedisp_bool>  h_killmask;     /* size nchans */
};

}  // namespace dedisp

#endif  // DEDISP_B200_PLAN_HPP
