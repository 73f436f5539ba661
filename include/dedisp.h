/*
 * dedisp.h -- C interface of the B200 dedispersion engine.
 *
 * Drop-in for the reference C API (piyushplcr7/dedisp_tests,
 * src/clib/dedisp.h): the same types, enumerations (values and order), entry
 * points and argument meanings. A program written against the reference
 * header compiles and links against libdedisp.so from this repository
 * unchanged. Each declaration cites the reference declaration it replaces.
 *
 * Data conventions (src/clib/dedisp.h:336-350):
 *   input   time-major [nsamps][nchans], channels packed LSB-first inside
 *           little-endian 32-bit words, in_nbits in {1,2,4,8,16,32};
 *   output  DM-major [dm_count][nsamps - max_delay], out_nbits in {8,16,32}
 *           (32 = float).
 */
#ifndef DEDISP_H_INCLUDE_GUARD
#define DEDISP_H_INCLUDE_GUARD

#ifdef __cplusplus
extern "C" {
#endif

/* Types and flags: src/clib/dedisp.h:39 includes the same header. */
#include "common/dedisp_types.h"

/* Opaque plan handle: src/clib/dedisp.h:45 */
typedef struct dedisp_plan_struct* dedisp_plan;

/* Error codes, same values and order: src/clib/dedisp.h:76-94 */
#ifndef DEDISP_ERROR_ENUM_DEFINED
#define DEDISP_ERROR_ENUM_DEFINED
typedef enum {
    DEDISP_NO_ERROR,
    DEDISP_MEM_ALLOC_FAILED,
    DEDISP_MEM_COPY_FAILED,
    DEDISP_NCHANS_EXCEEDS_LIMIT,
    DEDISP_INVALID_PLAN,
    DEDISP_INVALID_POINTER,
    DEDISP_INVALID_STRIDE,
    DEDISP_NO_DM_LIST_SET,
    DEDISP_TOO_FEW_NSAMPS,
    DEDISP_INVALID_FLAG_COMBINATION,
    DEDISP_UNSUPPORTED_IN_NBITS,
    DEDISP_UNSUPPORTED_OUT_NBITS,
    DEDISP_INVALID_DEVICE_INDEX,
    DEDISP_DEVICE_ALREADY_SET,
    DEDISP_PRIOR_GPU_ERROR,
    DEDISP_INTERNAL_GPU_ERROR,
    DEDISP_UNKNOWN_ERROR
} dedisp_error;
#endif

/* Implementation selector: src/clib/dedisp.h:116-120 */
typedef enum {
    DEDISP_DEDISP,
    DEDISP_TDD,
    DEDISP_FDD
} dedisp_implementation;

/* Plan management ---------------------------------------------------------*/

/* src/clib/dedisp.h:139. Process-global choice used by the next
 * dedisp_create_plan; default DEDISP_DEDISP. */
dedisp_error dedisp_select_implementation(dedisp_implementation imp);

/* src/clib/dedisp.h:155-159. *plan is set to 0 first. dt in seconds, f0 the
 * highest channel frequency in MHz, df the channel width in MHz. */
dedisp_error dedisp_create_plan(dedisp_plan* plan, dedisp_size nchans,
                                dedisp_float dt, dedisp_float f0,
                                dedisp_float df);

/* src/clib/dedisp.h:165 */
void dedisp_destroy_plan(dedisp_plan plan);

/* Setters ------------------------------------------------------------------*/

/* src/clib/dedisp.h:181. Stores the device index used by later plans. */
dedisp_error dedisp_set_device(int device_idx);

/* src/clib/dedisp.h:192-193. DEDISP_DEDISP and DEDISP_TDD plans only. */
dedisp_error dedisp_set_gulp_size(dedisp_plan plan, dedisp_size gulp_size);

/* src/clib/dedisp.h:199 */
dedisp_size dedisp_get_gulp_size(dedisp_plan plan);

/* src/clib/dedisp.h:214-215. killmask: one value per channel on the host;
 * NULL means every channel is used. */
dedisp_error dedisp_set_killmask(dedisp_plan plan, const dedisp_bool* killmask);

/* src/clib/dedisp.h:234-236. dm_list: host array of count DMs (pc cm^-3). */
dedisp_error dedisp_set_dm_list(dedisp_plan plan, const dedisp_float* dm_list,
                                dedisp_size count);

/* src/clib/dedisp.h:254-258. pulse_width in microseconds. */
dedisp_error dedisp_generate_dm_list(dedisp_plan plan, dedisp_float dm_start,
                                     dedisp_float dm_end,
                                     dedisp_float pulse_width,
                                     dedisp_float tol);

/* Getters (return 0 on error) ----------------------------------------------*/

dedisp_size dedisp_get_max_delay(const dedisp_plan plan);          /* :276 */
dedisp_size dedisp_get_dm_delay(const dedisp_plan plan, int dm_trial); /* :281 */
dedisp_size dedisp_get_channel_count(const dedisp_plan plan);      /* :286 */
dedisp_size dedisp_get_dm_count(const dedisp_plan plan);           /* :291 */
const dedisp_float* dedisp_get_dm_list(const dedisp_plan plan);    /* :297 */
const dedisp_bool* dedisp_get_killmask(const dedisp_plan plan);    /* :303 */
dedisp_float dedisp_get_dt(const dedisp_plan plan);                /* :309 */
dedisp_float dedisp_get_f0(const dedisp_plan plan);                /* :314 */
dedisp_float dedisp_get_df(const dedisp_plan plan);                /* :321 */

/* src/clib/dedisp.h:329 */
const char* dedisp_get_error_string(dedisp_error error);

/* Execution ----------------------------------------------------------------*/

/* src/clib/dedisp.h:375-381. Blocking unless DEDISP_ASYNC. With
 * DEDISP_DEVICE_POINTERS, in and out are device pointers (the reference
 * documents this flag but never implemented it). */
dedisp_error dedisp_execute(const dedisp_plan plan, dedisp_size nsamps,
                            const dedisp_byte* in, dedisp_size in_nbits,
                            dedisp_byte* out, dedisp_size out_nbits,
                            unsigned flags);

/* src/clib/dedisp.h:425-433. Strides in bytes. DEDISP_DEDISP/TDD only. */
dedisp_error dedisp_execute_adv(const dedisp_plan plan, dedisp_size nsamps,
                                const dedisp_byte* in, dedisp_size in_nbits,
                                dedisp_size in_stride, dedisp_byte* out,
                                dedisp_size out_nbits, dedisp_size out_stride,
                                unsigned flags);

/* src/clib/dedisp.h:480-490. Computes DMs [first_dm_idx, first_dm_idx +
 * dm_count) of the list. DEDISP_DEDISP/TDD only. */
dedisp_error dedisp_execute_guru(const dedisp_plan plan, dedisp_size nsamps,
                                 const dedisp_byte* in, dedisp_size in_nbits,
                                 dedisp_size in_stride, dedisp_byte* out,
                                 dedisp_size out_nbits, dedisp_size out_stride,
                                 dedisp_size first_dm_idx,
                                 dedisp_size dm_count, unsigned flags);

/* src/clib/dedisp.h:501. Waits for all device work. */
dedisp_error dedisp_sync(void);

#ifdef __cplusplus
}
#endif

#endif /* DEDISP_H_INCLUDE_GUARD */
