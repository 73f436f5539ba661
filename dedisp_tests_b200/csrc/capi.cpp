// C interface (include/dedisp.h, include/dedisp_b200.h).
//
// Mirrors the reference C wrapper src/clib/dedisp.cpp: process-global device
// index and implementation choice, a prior-GPU-error check at entry, and
// every exception from the plan classes reported as DEDISP_UNKNOWN_ERROR.
// Getters return 0 on error. The specific code and message of the last
// failure stay available through dedisp_b200_last_error.
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <typeinfo>

#include "dedisp.h"
#include "dedisp/DedispPlan.hpp"
#include "dedisp_b200.h"
#include "errors.hpp"
#include "tdd_kernels.hpp"
#include "fdd/FDDGPUPlan.hpp"
#include "fdd_engine.hpp"
#include "gpu_state.hpp"
#include "host_math.hpp"
#include "runtime.hpp"
#include "tdd/TDDPlan.hpp"
#include "tdd_engine.hpp"

struct dedisp_plan_struct {
    std::shared_ptr<dedisp::Plan> ptr;
};

namespace {
int g_device_idx = 0;
dedisp_implementation g_implementation = DEDISP_DEDISP;

thread_local dedisp_error t_last_code = DEDISP_NO_ERROR;
thread_local std::string t_last_msg;

dedisp_error note(dedisp_error code, const char* msg)
{
    t_last_code = code;
    t_last_msg = msg ? msg : "";
    return code;
}

// Runs fn; exceptions become DEDISP_UNKNOWN_ERROR like the reference while
// the detailed code is remembered for dedisp_b200_last_error.
template <typename F>
dedisp_error guarded(F&& fn)
{
    try {
        fn();
        return DEDISP_NO_ERROR;
    } catch (const dedisp::Error& e) {
        note(e.code(), e.what());
    } catch (const std::exception& e) {
        note(DEDISP_UNKNOWN_ERROR, e.what());
    } catch (...) {
        note(DEDISP_UNKNOWN_ERROR, "unknown exception");
    }
    return DEDISP_UNKNOWN_ERROR;
}

dedisp::TDDPlan* as_tdd(dedisp_plan p) { return dynamic_cast<dedisp::TDDPlan*>(p->ptr.get()); }
dedisp::DedispPlan* as_dedisp(dedisp_plan p)
{
    return dynamic_cast<dedisp::DedispPlan*>(p->ptr.get());
}
dedisp::FDDGPUPlan* as_fdd(dedisp_plan p) { return dynamic_cast<dedisp::FDDGPUPlan*>(p->ptr.get()); }
}  // namespace

namespace dedisp {
// Used by the other C entry points of the library (not exported in a header).
void note_last_error(dedisp_error code, const char* msg) { note(code, msg); }
}  // namespace dedisp

extern "C" {

dedisp_error dedisp_create_plan(dedisp_plan* plan, dedisp_size nchans, dedisp_float dt,
                                dedisp_float f0, dedisp_float df)
{
    if (!plan) return note(DEDISP_INVALID_POINTER, "plan is NULL");
    *plan = 0;
    if (dedisp::rt::prior_gpu_error()) return DEDISP_PRIOR_GPU_ERROR;
    dedisp_plan p = new dedisp_plan_struct();
    dedisp_error e = guarded([&] {
        switch (g_implementation) {
        case DEDISP_DEDISP: p->ptr.reset(new dedisp::DedispPlan(nchans, dt, f0, df, g_device_idx)); break;
        case DEDISP_TDD: p->ptr.reset(new dedisp::TDDPlan(nchans, dt, f0, df, g_device_idx)); break;
        // USE_CPU selects the reference's FFTW plan; this library has no CPU
        // path, so the GPU plan is created either way.
        case DEDISP_FDD: p->ptr.reset(new dedisp::FDDGPUPlan(nchans, dt, f0, df, g_device_idx)); break;
        default: DD_THROW(DEDISP_UNKNOWN_ERROR);
        }
    });
    if (e != DEDISP_NO_ERROR) {
        delete p;
        return e;
    }
    *plan = p;
    return DEDISP_NO_ERROR;
}

void dedisp_destroy_plan(dedisp_plan plan) { delete plan; }

dedisp_error dedisp_set_device(int device_idx)
{
    g_device_idx = device_idx;
    return DEDISP_NO_ERROR;
}

dedisp_error dedisp_select_implementation(dedisp_implementation imp)
{
    g_implementation = imp;
    return DEDISP_NO_ERROR;
}

dedisp_error dedisp_set_gulp_size(dedisp_plan plan, dedisp_size gulp_size)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    if (dedisp::rt::prior_gpu_error()) return DEDISP_PRIOR_GPU_ERROR;
    if (auto* d = as_dedisp(plan)) return guarded([&] { d->set_gulp_size(gulp_size); });
    if (auto* t = as_tdd(plan)) return guarded([&] { t->set_gulp_size(gulp_size); });
    if (as_fdd(plan)) return DEDISP_INVALID_PLAN;
    return DEDISP_UNKNOWN_ERROR;
}

// Like the reference, errors come back as the error code cast to
// dedisp_size (src/clib/dedisp.cpp:194-222).
dedisp_size dedisp_get_gulp_size(dedisp_plan plan)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    if (dedisp::rt::prior_gpu_error()) return DEDISP_PRIOR_GPU_ERROR;
    if (auto* d = as_dedisp(plan)) return d->get_gulp_size();
    if (auto* t = as_tdd(plan)) return t->get_gulp_size();
    return 0;
}

dedisp_error dedisp_set_dm_list(dedisp_plan plan, const dedisp_float* dm_list, dedisp_size count)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    if (dedisp::rt::prior_gpu_error()) return DEDISP_PRIOR_GPU_ERROR;
    return guarded([&] { plan->ptr->set_dm_list(dm_list, count); });
}

dedisp_error dedisp_generate_dm_list(dedisp_plan plan, dedisp_float dm_start, dedisp_float dm_end,
                                     dedisp_float ti, dedisp_float tol)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    if (dedisp::rt::prior_gpu_error()) return DEDISP_PRIOR_GPU_ERROR;
    return guarded([&] { plan->ptr->generate_dm_list(dm_start, dm_end, ti, tol); });
}

dedisp_error dedisp_set_killmask(dedisp_plan plan, const dedisp_bool* killmask)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    if (dedisp::rt::prior_gpu_error()) return DEDISP_PRIOR_GPU_ERROR;
    return guarded([&] { plan->ptr->set_killmask(killmask); });
}

dedisp_size dedisp_get_max_delay(const dedisp_plan plan)
{
    if (!plan || plan->ptr->get_dm_count() == 0) return 0;
    return (dedisp_size)plan->ptr->get_max_delay();
}

dedisp_size dedisp_get_dm_delay(const dedisp_plan plan, int dm_trial)
{
    if (!plan || plan->ptr->get_dm_count() == 0) return 0;
    if (dm_trial < 0 || (dedisp_size)dm_trial >= plan->ptr->get_dm_count()) return 0;
    const dedisp::Plan& p = *plan->ptr;
    return dedisp::hostmath::max_delay(p.get_dm_list()[dm_trial],
                                       p.get_delay_table()[p.get_channel_count() - 1]);
}

dedisp_size dedisp_get_channel_count(const dedisp_plan plan)
{
    return plan ? plan->ptr->get_channel_count() : 0;
}

dedisp_size dedisp_get_dm_count(const dedisp_plan plan) { return plan ? plan->ptr->get_dm_count() : 0; }

const dedisp_float* dedisp_get_dm_list(const dedisp_plan plan)
{
    if (!plan || plan->ptr->get_dm_count() == 0) return 0;
    return plan->ptr->get_dm_list();
}

const dedisp_bool* dedisp_get_killmask(const dedisp_plan plan)
{
    return plan ? plan->ptr->get_killmask() : 0;
}

dedisp_float dedisp_get_dt(const dedisp_plan plan) { return plan ? plan->ptr->get_dt() : 0; }
dedisp_float dedisp_get_f0(const dedisp_plan plan) { return plan ? plan->ptr->get_f0() : 0; }
dedisp_float dedisp_get_df(const dedisp_plan plan) { return plan ? plan->ptr->get_df() : 0; }

dedisp_error dedisp_execute_guru(const dedisp_plan plan, dedisp_size nsamps, const dedisp_byte* in,
                                 dedisp_size in_nbits, dedisp_size in_stride, dedisp_byte* out,
                                 dedisp_size out_nbits, dedisp_size out_stride,
                                 dedisp_size first_dm_idx, dedisp_size dm_count, unsigned flags)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    if (dedisp::rt::prior_gpu_error()) return DEDISP_PRIOR_GPU_ERROR;
    if (auto* d = as_dedisp(plan))
        return guarded([&] {
            d->execute_guru(nsamps, in, in_nbits, in_stride, out, out_nbits, out_stride,
                            first_dm_idx, dm_count, flags);
        });
    if (auto* t = as_tdd(plan))
        return guarded([&] {
            t->execute_guru_flags(nsamps, in, in_nbits, in_stride, out, out_nbits, out_stride,
                                  first_dm_idx, dm_count, flags);
        });
    if (as_fdd(plan)) return DEDISP_INVALID_PLAN;
    return DEDISP_UNKNOWN_ERROR;
}

dedisp_error dedisp_execute_adv(const dedisp_plan plan, dedisp_size nsamps, const dedisp_byte* in,
                                dedisp_size in_nbits, dedisp_size in_stride, dedisp_byte* out,
                                dedisp_size out_nbits, dedisp_size out_stride, unsigned flags)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    if (dedisp::rt::prior_gpu_error()) return DEDISP_PRIOR_GPU_ERROR;
    if (auto* d = as_dedisp(plan))
        return guarded([&] {
            d->execute_adv(nsamps, in, in_nbits, in_stride, out, out_nbits, out_stride, flags);
        });
    if (auto* t = as_tdd(plan))
        return guarded([&] {
            t->execute_guru_flags(nsamps, in, in_nbits, in_stride, out, out_nbits, out_stride, 0,
                                  t->get_dm_count(), flags);
        });
    if (as_fdd(plan)) return DEDISP_INVALID_PLAN;
    return DEDISP_UNKNOWN_ERROR;
}

dedisp_error dedisp_execute(const dedisp_plan plan, dedisp_size nsamps, const dedisp_byte* in,
                            dedisp_size in_nbits, dedisp_byte* out, dedisp_size out_nbits,
                            unsigned flags)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    if (dedisp::rt::prior_gpu_error()) return DEDISP_PRIOR_GPU_ERROR;
    return guarded([&] { plan->ptr->execute(nsamps, in, in_nbits, out, out_nbits, flags); });
}

dedisp_error dedisp_sync(void)
{
    if (dedisp::rt::device_count() == 0) return DEDISP_NO_ERROR;
    return cudaDeviceSynchronize() == cudaSuccess ? DEDISP_NO_ERROR : DEDISP_PRIOR_GPU_ERROR;
}

const char* dedisp_get_error_string(dedisp_error error)
{
    switch (error) {
    case DEDISP_NO_ERROR: return "No error";
    case DEDISP_MEM_ALLOC_FAILED: return "Memory allocation failed";
    case DEDISP_MEM_COPY_FAILED: return "Memory copy failed";
    case DEDISP_INVALID_DEVICE_INDEX: return "Invalid device index";
    case DEDISP_DEVICE_ALREADY_SET: return "Device is already set and cannot be changed";
    case DEDISP_NCHANS_EXCEEDS_LIMIT: return "No. channels exceeds internal limit";
    case DEDISP_INVALID_PLAN: return "Invalid plan";
    case DEDISP_INVALID_POINTER: return "Invalid pointer";
    case DEDISP_INVALID_STRIDE: return "Invalid stride";
    case DEDISP_NO_DM_LIST_SET: return "No DM list has been set";
    case DEDISP_TOO_FEW_NSAMPS: return "No. samples < maximum delay";
    case DEDISP_INVALID_FLAG_COMBINATION: return "Invalid flag combination";
    case DEDISP_UNSUPPORTED_IN_NBITS: return "Unsupported in_nbits value";
    case DEDISP_UNSUPPORTED_OUT_NBITS: return "Unsupported out_nbits value";
    case DEDISP_PRIOR_GPU_ERROR: return "Prior GPU error.";
    case DEDISP_INTERNAL_GPU_ERROR: return "Internal GPU error. Please contact the author(s).";
    case DEDISP_UNKNOWN_ERROR: return "Unknown error. Please contact the author(s).";
    default: return "Invalid error code";
    }
}

// ---------------------------------------------------------------------------
// Extensions (include/dedisp_b200.h)
// ---------------------------------------------------------------------------
dedisp_error dedisp_b200_set_tdd_kernel(dedisp_plan plan, int kernel)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    if (kernel < 0 || kernel > 2) return DEDISP_UNKNOWN_ERROR;
    const auto k = (dedisp::TddKernel)kernel;
    if (auto* d = as_dedisp(plan)) { d->set_kernel(k); return DEDISP_NO_ERROR; }
    if (auto* t = as_tdd(plan)) { t->set_kernel(k); return DEDISP_NO_ERROR; }
    return DEDISP_INVALID_PLAN;
}

dedisp_error dedisp_b200_set_tdd_variant(dedisp_plan plan, int variant)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    if (variant < 0 || variant >= dedisp::kern::tiled_variant_count(8)) return DEDISP_UNKNOWN_ERROR;
    if (auto* d = as_dedisp(plan)) { d->set_tile_variant(variant); return DEDISP_NO_ERROR; }
    if (auto* t = as_tdd(plan)) { t->set_tile_variant(variant); return DEDISP_NO_ERROR; }
    return DEDISP_INVALID_PLAN;
}

int dedisp_b200_tdd_variant_count(dedisp_size in_nbits)
{
    return dedisp::kern::tiled_variant_count((int)in_nbits);
}

dedisp_error dedisp_b200_set_stream(dedisp_plan plan, void* cuda_stream)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    auto* g = dynamic_cast<dedisp::GPUPlan*>(plan->ptr.get());
    if (!g) return DEDISP_INVALID_PLAN;
    g->set_stream(cuda_stream);
    return DEDISP_NO_ERROR;
}

dedisp_error dedisp_b200_set_timing(dedisp_plan plan, int enable)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    auto* g = dynamic_cast<dedisp::GPUPlan*>(plan->ptr.get());
    if (!g) return DEDISP_INVALID_PLAN;
    g->set_timing(enable != 0);
    return DEDISP_NO_ERROR;
}

dedisp_error dedisp_b200_get_timing(dedisp_plan plan, float* kernel_ms, float* prep_ms,
                                    int* launches, int* variant)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    auto* g = dynamic_cast<dedisp::GPUPlan*>(plan->ptr.get());
    if (!g) return DEDISP_INVALID_PLAN;
    const dedisp::ExecTiming t = g->last_timing();
    if (kernel_ms) *kernel_ms = t.kernel_ms;
    if (prep_ms) *prep_ms = t.prep_ms;
    if (launches) *launches = t.launches;
    if (variant) *variant = t.variant;
    return DEDISP_NO_ERROR;
}

dedisp_error dedisp_b200_get_stage_times(dedisp_plan plan, float* stage_ms, int count)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    auto* g = dynamic_cast<dedisp::GPUPlan*>(plan->ptr.get());
    if (!g) return DEDISP_INVALID_PLAN;
    if (!stage_ms && count > 0) return DEDISP_INVALID_POINTER;
    const dedisp::ExecTiming t = g->last_timing();
    for (int i = 0; i < count; ++i) stage_ms[i] = i < 6 ? t.stage_ms[i] : 0.f;
    return DEDISP_NO_ERROR;
}

dedisp_error dedisp_b200_get_phasor_source(dedisp_plan plan, int* source)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    auto* g = dynamic_cast<dedisp::GPUPlan*>(plan->ptr.get());
    if (!g) return DEDISP_INVALID_PLAN;
    if (!source) return DEDISP_INVALID_POINTER;
    *source = g->last_timing().phasor;
    return DEDISP_NO_ERROR;
}

dedisp_error dedisp_b200_get_tc_form(dedisp_plan plan, int* form)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    auto* g = dynamic_cast<dedisp::GPUPlan*>(plan->ptr.get());
    if (!g) return DEDISP_INVALID_PLAN;
    if (!form) return DEDISP_INVALID_POINTER;
    *form = g->last_timing().tc_form;
    return DEDISP_NO_ERROR;
}

dedisp_error dedisp_b200_last_error(char* msg, dedisp_size len)
{
    if (msg && len) {
        std::strncpy(msg, t_last_msg.c_str(), len - 1);
        msg[len - 1] = 0;
    }
    return t_last_code;
}

dedisp_error dedisp_b200_set_fdd_options(dedisp_plan plan, int segmented, int timeseries,
                                         int precision, int round_delays,
                                         dedisp_size segment_nfft)
{
    if (!plan) return DEDISP_INVALID_PLAN;
    auto* f = as_fdd(plan);
    if (!f) return DEDISP_INVALID_PLAN;
    return guarded([&] {
        dedisp::FddOptions o;
        o.segmented = segmented < 0 ? -1 : (segmented ? 1 : 0);
        o.output = timeseries ? dedisp::FddOutput::TimeSeries : dedisp::FddOutput::Spectrum;
        o.precision = precision ? dedisp::FddPrecision::BF16x3 : dedisp::FddPrecision::FP32;
        o.round_delays = round_delays != 0;
        o.segment_nfft = segment_nfft;
        f->set_options(o);
    });
}

dedisp_size dedisp_b200_fdd_segment_length(dedisp_size nsamps, dedisp_size max_delay, dedisp_size dm_count,
                                           dedisp_size nchans, int precision, dedisp_size segment_nfft)
{
    dedisp_size n = 0;
    guarded([&] {
        dedisp::FddOptions o;
        o.segmented = 1;
        o.precision = precision ? dedisp::FddPrecision::BF16x3 : dedisp::FddPrecision::FP32;
        o.segment_nfft = segment_nfft;
        n = dedisp::detail::fdd_geometry(o, nsamps, max_delay, dm_count, nchans).nfft;
    });
    return n;
}

dedisp_error dedisp_b200_set_wait_limit_ns(unsigned long long ns)
{
    dedisp::rt::set_wait_limit_ns(ns);
    return DEDISP_NO_ERROR;
}

unsigned long long dedisp_b200_get_wait_limit_ns(void) { return dedisp::rt::wait_limit_ns(); }

dedisp_error dedisp_b200_set_wait_expiry_test(int enable)
{
    dedisp::rt::set_wait_expiry_test(enable != 0);
    return DEDISP_NO_ERROR;
}

dedisp_size dedisp_b200_output_row_length(dedisp_plan plan, dedisp_size nsamps)
{
    if (!plan || plan->ptr->get_dm_count() == 0) return 0;
    if (auto* f = as_fdd(plan)) return f->output_row_length(nsamps);
    const dedisp_size md = (dedisp_size)plan->ptr->get_max_delay();
    return nsamps >= md ? nsamps - md : 0;
}

}  // extern "C"
