// Test infrastructure only: C entry points that run the reference's own GPU
// plan classes (compiled from the reference sources by oracle/ref/Makefile).
// One shared library is built per plan class (REF_PLAN_TDD / REF_PLAN_DEDISP /
// REF_PLAN_FDD) because the reference defines the same helper symbols in
// each of its libraries. Used on a GPU box to produce golden outputs and to
// pin the oracle against the reference's real kernels. Never linked into the
// product.
#include <cstdlib>
#include <cstdio>
#include <exception>

#if defined(REF_PLAN_TDD)
#include "tdd/TDDPlan.hpp"
using RefPlan = dedisp::TDDPlan;
#elif defined(REF_PLAN_DEDISP)
#include "dedisp/DedispPlan.hpp"
using RefPlan = dedisp::DedispPlan;
#elif defined(REF_PLAN_FDD)
#include "fdd/FDDGPUPlan.hpp"
using RefPlan = dedisp::FDDGPUPlan;
#else
#error "define one of REF_PLAN_TDD, REF_PLAN_DEDISP, REF_PLAN_FDD"
#endif

extern "C" {

// Runs RefPlan::execute. dm_list/killmask are host arrays (killmask may be
// NULL for all-ones). gulp_size==0 keeps the plan default (ignored for FDD).
// For FDD, segmented!=0 selects the reference's USE_SEGMENTED path.
// Returns 0 on success, -1 if the plan threw.
int ref_execute(int device_idx, size_t nchans, float dt, float f0, float df,
                const float* dm_list, size_t dm_count, const int* killmask,
                size_t nsamps, const unsigned char* in, size_t in_nbits,
                unsigned char* out, size_t out_nbits, size_t gulp_size,
                int segmented, size_t* max_delay)
{
    try {
        RefPlan plan(nchans, dt, f0, df, device_idx);
        plan.set_dm_list(dm_list, dm_count);
        plan.set_killmask(killmask);
#if !defined(REF_PLAN_FDD)
        if (gulp_size) plan.set_gulp_size(gulp_size);
        (void)segmented;
#else
        (void)gulp_size;
        setenv("USE_SEGMENTED", segmented ? "1" : "0", 1);
#endif
        if (max_delay) *max_delay = (size_t)plan.get_max_delay();
        plan.execute(nsamps, in, in_nbits, out, out_nbits, 0);
        plan.sync();
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "reference plan error: %s\n", e.what());
        return -1;
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
