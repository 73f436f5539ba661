// Test infrastructure only: a C entry point around the reference's own
// dedisp::Plan host code (src/Plan.cpp), compiled from the reference sources
// by oracle/ref/Makefile. Used to pin the oracle's delay table, DM list and
// max-delay arithmetic bit for bit. Never linked into the product.
#include <cstddef>
#include <cstring>
#include <vector>

#include "Plan.hpp"

namespace {
// Plan::execute is pure virtual; this probe only exercises the host setup.
class ProbePlan : public dedisp::Plan {
public:
    ProbePlan(size_type n, float_type dt, float_type f0, float_type df)
        : Plan(n, dt, f0, df) {}
    void execute(size_type, const byte_type*, size_type, byte_type*, size_type,
                 unsigned) override {}
};
}  // namespace

extern "C" {

// Delay table as built by Plan::Plan (src/Plan.cpp:16-40,109-119).
int ref_plan_delay_table(size_t nchans, float dt, float f0, float df, float* out)
{
    try {
        ProbePlan p(nchans, dt, f0, df);
        std::memcpy(out, p.get_delay_table(), nchans * sizeof(float));
        return 0;
    } catch (...) {
        return -1;
    }
}

// Plan::generate_dm_list (src/Plan.cpp:136-154): writes up to cap DMs and the
// resulting max delay; returns the DM count.
long ref_plan_generate_dm_list(size_t nchans, float dt, float f0, float df,
                               float dm_start, float dm_end, float ti, float tol,
                               float* out, size_t cap, size_t* max_delay)
{
    try {
        ProbePlan p(nchans, dt, f0, df);
        p.generate_dm_list(dm_start, dm_end, ti, tol);
        size_t n = p.get_dm_count();
        std::memcpy(out, p.get_dm_list(), (n < cap ? n : cap) * sizeof(float));
        *max_delay = (size_t)p.get_max_delay();
        return (long)n;
    } catch (...) {
        return -1;
    }
}

// Plan::set_dm_list (src/Plan.cpp:72-87): returns the max delay.
long ref_plan_set_dm_list(size_t nchans, float dt, float f0, float df,
                          const float* dms, size_t count)
{
    try {
        ProbePlan p(nchans, dt, f0, df);
        p.set_dm_list(dms, count);
        return (long)(size_t)p.get_max_delay();
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
