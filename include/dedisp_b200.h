/*
 * dedisp_b200.h -- extensions of the dedisp C interface (no counterpart in
 * the reference unless noted). All entry points take the ordinary
 * dedisp_plan handle from dedisp.h and use plain C types only.
 */
#ifndef DEDISP_B200_H_INCLUDE_GUARD
#define DEDISP_B200_H_INCLUDE_GUARD

#include "dedisp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* TDD kernel selection for DEDISP_DEDISP / DEDISP_TDD plans. AUTO uses the
 * tiled shared-memory kernel when the killmask holds only 0/1 values; PLAIN
 * is the one-thread-per-sample-pair baseline (the reference's decomposition,
 * src/tdd/dedisperse/TDDKernel.cu:133-151). */
typedef enum {
    DEDISP_B200_TDD_AUTO = 0,
    DEDISP_B200_TDD_PLAIN = 1,
    DEDISP_B200_TDD_TILED = 2
} dedisp_b200_tdd_kernel;

dedisp_error dedisp_b200_set_tdd_kernel(dedisp_plan plan, int kernel);

/* Tile shape of the tiled TDD kernel (DMs per block, samples per thread).
 * Variants are numbered per input width, [0, dedisp_b200_tdd_variant_count(
 * in_nbits)): 8-bit 0-4 on channel-major packed rows, 5-8 on quad-strided
 * rows; 1/2/4-bit 0 the packed-row kernel, 1-4 quad-strided rows (samples
 * widened to bytes); 16/32-bit 0 only. Quad-strided rows are built per gulp
 * (four bytes per sample and channel in device memory). A variant outside
 * the executed width's range selects that width's default (quad-strided
 * 20 words x 12 DMs for widths up to 8 bits). Every variant computes the same
 * bit-exact sums; they differ in speed. */
dedisp_error dedisp_b200_set_tdd_variant(dedisp_plan plan, int variant);
int dedisp_b200_tdd_variant_count(dedisp_size in_nbits);

/* Runs the plan's device work on a caller-provided cudaStream_t (NULL
 * restores the plan's own stream). */
dedisp_error dedisp_b200_set_stream(dedisp_plan plan, void* cuda_stream);

/* Device-time instrumentation of execute(): when enabled, the next calls
 * record CUDA events around the preprocessing (transpose / unpack + FFT) and
 * the dedispersion kernels on the plan's stream. */
dedisp_error dedisp_b200_set_timing(dedisp_plan plan, int enable);
dedisp_error dedisp_b200_get_timing(dedisp_plan plan, float* kernel_ms, float* prep_ms,
                                    int* launches, int* variant);

/* FDD plans, with timing enabled: device time (ms) of each stage of the last
 * execute, in order: unpack, forward FFT, operand layout (split B or
 * bin-major), MAC, DM-major transpose (or spectrum output), inverse FFT.
 * Writes `count` values (at most 6 meaningful; the rest 0). */
dedisp_error dedisp_b200_get_stage_times(dedisp_plan plan, float* stage_ms, int count);

/* FDD plans: phasor source of the tensor-core MAC in the last execute: 0 the
 * per-bin delay table (every delay), 1 the quarter-wave table, 2 the per-bin
 * table for the small delays and the rest computed from the twiddle tables,
 * 3 every phasor from the twiddle tables; -1 no tensor-core MAC ran. The
 * environment variable DEDISP_TC_TABLE_CAP caps the per-bin table's extent
 * (to compare the sources on one shape). */
dedisp_error dedisp_b200_get_phasor_source(dedisp_plan plan, int* source);

/* FDD plans: MMA form of the last tensor-core MAC launch: 0 three MMAs per K
 * step, 1 fused at 32-channel chunks (DEDISP_TC_FORM=1), 2 three MMAs with 3 A
 * buffers, 3 CTA pairs (cta_group::2, M = 256; DEDISP_TC_PAIR), 4 CTA pairs
 * with 3 A buffers, 5 fused at 64-channel chunks with 3 A buffers (the
 * default for at most 32 MMA columns); -1 none ran. */
dedisp_error dedisp_b200_get_tc_form(dedisp_plan plan, int* form);

/* The C functions of dedisp.h report every failure inside the plan classes
 * as DEDISP_UNKNOWN_ERROR, like the reference (src/clib/dedisp.cpp:520-523).
 * This returns the specific code of the most recent such failure in the
 * calling thread and copies its message (may be NULL). */
dedisp_error dedisp_b200_last_error(char* msg, dedisp_size len);

/* FDD options (DEDISP_FDD plans):
 *   segmented      -1 follow USE_SEGMENTED, 0 whole series, 1 segmented
 *   timeseries     whole-series output: 0 spectrum (default), 1 time series
 *   precision      0 FP32 CUDA cores, 1 3xBF16 tensor-core GEMM
 *   round_delays   0 truncate (reference FDD), 1 round half to even (TDD)
 *   segment_nfft   0 reference doubling rule, DEDISP_B200_FDD_SEGMENT_AUTO
 *                  the power of two with the least modelled device time (the
 *                  output is the same series; only rounding differs), else a
 *                  power of two above the max delay */
#define DEDISP_B200_FDD_SEGMENT_AUTO 1

/* Segmented FDD: the segment length (points) a plan with these sizes uses
 * under `segment_nfft` (0 reference rule, DEDISP_B200_FDD_SEGMENT_AUTO, or an
 * explicit length); 0 if none fits (the max delay reaches the segment). Host
 * only. */
dedisp_size dedisp_b200_fdd_segment_length(dedisp_size nsamps, dedisp_size max_delay, dedisp_size dm_count,
                                           dedisp_size nchans, int precision, dedisp_size segment_nfft);
dedisp_error dedisp_b200_set_fdd_options(dedisp_plan plan, int segmented, int timeseries,
                                         int precision, int round_delays,
                                         dedisp_size segment_nfft);

/* Bounded device waits. No counterpart in the reference (its kernels do not
 * wait on asynchronous copies). The quad-strided TDD kernels and the
 * tensor-core FDD MAC poll mbarriers for their own bulk copies and MMAs; a
 * poll that has not seen its phase complete after `ns` nanoseconds of GPU
 * global time gives up: the kernel waits (bounded again) for its own work
 * still in flight, frees its tensor memory and returns, and the plan's
 * execute fails with DEDISP_INTERNAL_GPU_ERROR (dedisp_b200_last_error); the
 * plan stays usable. Process-wide, read at each launch (a captured CUDA graph
 * keeps the values of its capture). ns = 0 restores the default, 2 s.
 * With the expiry test enabled, each of those kernels additionally waits, at
 * the first wait of its pipeline, on an mbarrier that nothing arrives on, so
 * that the limit expires and the error path runs; for tests only. */
dedisp_error dedisp_b200_set_wait_limit_ns(unsigned long long ns);
unsigned long long dedisp_b200_get_wait_limit_ns(void);
dedisp_error dedisp_b200_set_wait_expiry_test(int enable);

/* Allocation-free time-domain dedispersion. No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc -- real-time pipelines that forbid
 * allocation once started (an allocation can block on the driver for an
 * unbounded time), or processes whose device memory belongs to another
 * allocator.
 * Computes what a DEDISP_TDD plan with DEDISP_DEVICE_POINTERS computes (same
 * bit-exact output) for a plan described by (nchans, dt, f0, df), the host
 * DM list and killmask (NULL: all channels; values must be 0 or 1), reading
 * d_in (device, time-major, in_stride bytes per sample) and writing d_out
 * (device, dm_count rows of out_stride bytes), then waits for `stream`.
 *
 * It allocates no device memory: its scratch is a fixed 64 MiB array in the
 * library (plus small tables for up to 16384 DMs and 8192 channels), held by
 * every GPU that loads the library until the process exits. Requests whose
 * channel-major copy, (nchans + 1) x (nsamps rounded up + padding) samples,
 * does not fit are rejected with DEDISP_MEM_ALLOC_FAILED. The first call on
 * a device looks up the arrays' device addresses (cudaGetSymbolAddress) and
 * should therefore come before any stream capture on that device; `stream`
 * (NULL: the legacy default stream) must belong to the current device
 * (DEDISP_INVALID_DEVICE_INDEX otherwise). All calls share the scratch:
 * calls that overlap on the GPU race. On failure,
 * dedisp_b200_noalloc_last_message() describes the reason; after a
 * successful call it is empty. */
dedisp_error dedisp_b200_tdd_execute_noalloc(
    dedisp_size nchans, dedisp_float dt, dedisp_float f0, dedisp_float df,
    const dedisp_float* dm_list, dedisp_size dm_count, const dedisp_bool* killmask,
    dedisp_size nsamps, const dedisp_byte* d_in, dedisp_size in_nbits, dedisp_size in_stride,
    dedisp_byte* d_out, dedisp_size out_nbits, dedisp_size out_stride, void* stream);
const char* dedisp_b200_noalloc_last_message(void);

/* ------------------------------------------------------------------------
 * Batched multi-beam TDD. No counterpart in the reference (its plans take one
 * series per execute call). Beams share the channel setup and widths; each
 * has its own DEVICE input (time-major packed rows), sample count, DM list
 * and DEVICE output (dm_count rows of nsamps - max_delay samples, out_stride
 * bytes apart; max_delay follows the reference rule: last DM of the list x
 * delay of the last channel). One execute enqueues the transposes of all
 * beams and one persistent dedispersion launch over all of them (8-bit input,
 * 0/1 killmask; otherwise one launch per beam), captured once into a CUDA
 * graph when use_graph != 0 and replayed on later calls. Results are
 * bit-identical to a TDD plan run per beam.
 * ---------------------------------------------------------------------- */
typedef struct dedisp_b200_batch_struct* dedisp_b200_batch;

typedef struct {
    const dedisp_byte* in;      /* device */
    dedisp_size in_stride;      /* bytes per input row */
    dedisp_size nsamps;
    const dedisp_float* dm_list;  /* host, dm_count entries (copied) */
    dedisp_size dm_count;
    dedisp_byte* out;           /* device */
    dedisp_size out_stride;     /* bytes per output row */
} dedisp_b200_beam;

dedisp_error dedisp_b200_batch_create(dedisp_b200_batch* batch, dedisp_size nchans, dedisp_float dt,
                                      dedisp_float f0, dedisp_float df, dedisp_size in_nbits,
                                      dedisp_size out_nbits, int device);
void dedisp_b200_batch_destroy(dedisp_b200_batch batch);
dedisp_error dedisp_b200_batch_set_killmask(dedisp_b200_batch batch, const dedisp_bool* killmask);
dedisp_error dedisp_b200_batch_set_beams(dedisp_b200_batch batch, const dedisp_b200_beam* beams,
                                         dedisp_size nbeams);
/* Scratch for the transposed inputs (any tile shape); a caller may hand the
 * same buffer to several batches that it runs one after another on one
 * stream. Without one the batch allocates its own. */
dedisp_size dedisp_b200_batch_workspace_size(dedisp_b200_batch batch);
dedisp_error dedisp_b200_batch_set_workspace(dedisp_b200_batch batch, void* d_workspace,
                                             dedisp_size bytes);
/* Tile shape: variant < dedisp_b200_batch_variant_count(in_nbits), channels
 * per stage even and <= 32 (0: the largest that fits shared memory; the
 * quad-strided variants size their stages per block and ignore it). */
int dedisp_b200_batch_variant_count(dedisp_size in_nbits);
dedisp_error dedisp_b200_batch_set_shape(dedisp_b200_batch batch, int variant, int chan_per_stage);
/* Times every candidate shape on the leading 8192 output samples of each
 * beam (CUDA events, on `stream`, synchronous) and keeps the fastest. */
dedisp_error dedisp_b200_batch_autotune(dedisp_b200_batch batch, void* stream, int* variant,
                                        int* chan_per_stage);
dedisp_error dedisp_b200_batch_execute(dedisp_b200_batch batch, void* stream, int use_graph);
/* Waits for the batch's work on `stream`; DEDISP_INTERNAL_GPU_ERROR if a
 * bounded wait of the last execute expired (dedisp_b200_set_wait_limit_ns).
 * With timing enabled execute performs this check itself. */
dedisp_error dedisp_b200_batch_sync(dedisp_b200_batch batch, void* stream);
/* Device time of the last execute's transposes and dedispersion (with
 * timing enabled; execute then waits for its work). With use_graph the
 * transposes are inside the graph: transpose_ms is -1 and dedisperse_ms is
 * the whole graph. */
dedisp_error dedisp_b200_batch_set_timing(dedisp_b200_batch batch, int enable);
dedisp_error dedisp_b200_batch_get_timing(dedisp_b200_batch batch, float* transpose_ms,
                                          float* dedisperse_ms, int* launches);
dedisp_size dedisp_b200_batch_max_delay(dedisp_b200_batch batch, dedisp_size beam);
/* The batch functions return their specific error code; the message of the
 * last failure on the calling thread is available from dedisp_b200_last_error. */

/* ------------------------------------------------------------------------
 * Batched multi-beam FDD. No counterpart in the reference (its FDDGPUPlan
 * takes one series per execute call, src/fdd/FDDGPUPlan.cpp:429-546).
 * Beams share the channel setup and input width; each has its own DEVICE
 * input (time-major rows, in_stride bytes apart), sample count, DM list and
 * DEVICE output: dm_count rows of nsamps - max_delay floats, out_stride bytes
 * apart (max_delay: last DM of the list x delay of the last channel). Every
 * beam is dedispersed in the segmented (overlap-save) form with the
 * reference's segment-length rule and the 3xBF16 tensor-core MAC, as an
 * FDD plan with segmented = 1, precision = 1 computes it. One execute
 * enqueues each beam's unpack, forward FFTs and split operand, ONE
 * persistent MAC launch over all beams (at most 48 segment groups of 64
 * segments per batch), then each beam's inverse FFTs; captured once into a
 * CUDA graph when use_graph != 0 and replayed. Inputs, outputs and the
 * workspace must stay valid while a captured graph may run.
 * ---------------------------------------------------------------------- */
typedef struct dedisp_b200_fdd_batch_struct* dedisp_b200_fdd_batch;

dedisp_error dedisp_b200_fdd_batch_create(dedisp_b200_fdd_batch* batch, dedisp_size nchans,
                                          dedisp_float dt, dedisp_float f0, dedisp_float df,
                                          dedisp_size in_nbits, int device);
void dedisp_b200_fdd_batch_destroy(dedisp_b200_fdd_batch batch);
dedisp_error dedisp_b200_fdd_batch_set_killmask(dedisp_b200_fdd_batch batch, const dedisp_bool* killmask);
dedisp_error dedisp_b200_fdd_batch_set_beams(dedisp_b200_fdd_batch batch, const dedisp_b200_beam* beams,
                                             dedisp_size nbeams);
/* Device bytes of scratch and per-beam operands (spectra split into BF16
 * parts and dedispersed spectra of every beam); a caller may hand in its own
 * buffer, else the batch allocates it at the first execute. */
dedisp_size dedisp_b200_fdd_batch_workspace_size(dedisp_b200_fdd_batch batch);
dedisp_error dedisp_b200_fdd_batch_set_workspace(dedisp_b200_fdd_batch batch, void* d_workspace,
                                                 dedisp_size bytes);
dedisp_error dedisp_b200_fdd_batch_execute(dedisp_b200_fdd_batch batch, void* stream, int use_graph);
/* Waits for the batch's work on `stream`; DEDISP_INTERNAL_GPU_ERROR if a
 * bounded wait of the last execute's MAC expired. */
dedisp_error dedisp_b200_fdd_batch_sync(dedisp_b200_fdd_batch batch, void* stream);
/* With timing enabled execute waits for its work and reports the device time
 * of the preparation, of the MAC launch and of the inverse side (graph mode:
 * the whole graph as mac_ms, the others -1). */
dedisp_error dedisp_b200_fdd_batch_set_timing(dedisp_b200_fdd_batch batch, int enable);
dedisp_error dedisp_b200_fdd_batch_get_timing(dedisp_b200_fdd_batch batch, float* prep_ms, float* mac_ms,
                                              float* post_ms, int* launches);
dedisp_size dedisp_b200_fdd_batch_max_delay(dedisp_b200_fdd_batch batch, dedisp_size beam);
/* Segment length of every beam, as segment_nfft of dedisp_b200_set_fdd_options
 * (0 the reference rule, the default; DEDISP_B200_FDD_SEGMENT_AUTO the least
 * modelled time per beam); takes effect at the next set_beams. */
dedisp_error dedisp_b200_fdd_batch_set_segment_nfft(dedisp_b200_fdd_batch batch, dedisp_size segment_nfft);
/* After a direct (use_graph = 0) execute with timing on: the MAC launch's
 * largest and mean per-CTA busy time (ms); their ratio shows how evenly the
 * work list spread over the SMs. 0 when not measured. */
dedisp_error dedisp_b200_fdd_batch_get_mac_balance(dedisp_b200_fdd_batch batch, float* cta_max_ms,
                                                   float* cta_mean_ms);
/* Phasor source of a beam's tensor-core MAC as planned for the current beam
 * set (codes of dedisp_b200_get_phasor_source); -1 on error or no MAC work. */
int dedisp_b200_fdd_batch_phasor_source(dedisp_b200_fdd_batch batch, dedisp_size beam);

/* ------------------------------------------------------------------------
 * Streaming server. No counterpart in the reference. Beams deliver host
 * gulps of any length (<= max_gulp); the server keeps each beam's last
 * max_delay input rows on the device, so a gulp of n rows yields n output
 * samples per DM (the dedispersion of tail + gulp; tails start as zero
 * rows). kind 0 beams run on TDD workers, kind 1 on FDD workers (segmented
 * time-series output; fdd_precision 0 FP32, 1 3xBF16 tensor cores;
 * fdd_segment 0 = the plan's FFT-length rule; FDD gulps at most
 * fdd_max_gulp samples, 0 = max_gulp). Each worker is a host thread
 * with its own CUDA stream and plans; start() allocates everything and
 * fails with DEDISP_MEM_ALLOC_FAILED above hbm_budget bytes (0: no limit),
 * after which submit() does not allocate. Gulps of one beam run in order.
 * d_out: device buffer of dm_count x nsamps floats, or NULL (the worker's
 * own buffer, reused by its next gulp). Host rows must stay valid until the
 * gulp is done; pinned memory makes the copy asynchronous.
 * ---------------------------------------------------------------------- */
typedef struct dedisp_b200_server_struct* dedisp_b200_server;

typedef struct {
    int beam;
    int worker;
    dedisp_size nsamps;
    double t_submit;   /* seconds, monotonic host clock */
    double t_start;
    double t_done;
    float device_ms;   /* H2D + dedispersion + tail copy, CUDA events */
} dedisp_b200_gulp_record;

dedisp_error dedisp_b200_server_create(dedisp_b200_server* server, dedisp_size nchans, dedisp_float dt,
                                       dedisp_float f0, dedisp_float df, dedisp_size in_nbits, int device,
                                       dedisp_size hbm_budget, dedisp_size max_gulp, int tdd_workers,
                                       int fdd_workers, int fdd_precision, dedisp_size fdd_segment,
                                       dedisp_size fdd_max_gulp);
void dedisp_b200_server_destroy(dedisp_b200_server server);
/* Returns the beam index, or -1 (dedisp_b200_last_error has the reason). */
int dedisp_b200_server_add_beam(dedisp_b200_server server, const dedisp_float* dm_list,
                                dedisp_size dm_count, int kind);
dedisp_size dedisp_b200_server_max_delay(dedisp_b200_server server, int beam);
dedisp_error dedisp_b200_server_start(dedisp_b200_server server, dedisp_size* bytes_held);
/* Returns a ticket >= 0, or -1. */
long dedisp_b200_server_submit(dedisp_b200_server server, int beam, const dedisp_byte* rows,
                               dedisp_size nsamps, dedisp_float* d_out);
/* 1 done, 0 pending, -1 error. */
int dedisp_b200_server_done(dedisp_b200_server server, long ticket);
dedisp_error dedisp_b200_server_wait(dedisp_b200_server server, long ticket);
dedisp_error dedisp_b200_server_drain(dedisp_b200_server server);
dedisp_size dedisp_b200_server_record_count(dedisp_b200_server server);
dedisp_error dedisp_b200_server_records(dedisp_b200_server server, dedisp_b200_gulp_record* records,
                                        dedisp_size count);

/* ------------------------------------------------------------------------
 * SIGPROC filterbank input and per-DM output, the file I/O of the
 * reference's *_fil tools (bin/fil/fil.hpp) as library calls.
 * ---------------------------------------------------------------------- */
typedef struct {
    double tsamp, tstart, fch1, foff;
    double src_raj, src_dej, az_start, za_start;
    int nchans, nifs, nbits;
    int telescope_id, machine_id, nbeams, ibeam;
    dedisp_size nsamples;       /* from the size of the data section (fil.hpp:366-370) */
    dedisp_size header_bytes;
    char source_name[80];
} dedisp_b200_fil_header;

/* Parses the header (typed SIGPROC keywords; replaces read_header,
 * fil.hpp:306-378, which stores the keyword instead of the source name). */
dedisp_error dedisp_b200_fil_read_header(const char* path, dedisp_b200_fil_header* header);
/* Raw time-major rows [first, first + count) (fil.hpp:210-213). */
dedisp_error dedisp_b200_fil_read_samples(const char* path, const dedisp_b200_fil_header* header,
                                          dedisp_size first, dedisp_size count, dedisp_byte* out);
/* 8-bit rows averaged over `factor` samples in place, truncated to bytes
 * (decimate_timeseries, fil.hpp:31-52; full blocks only). Returns the new
 * sample count. */
dedisp_size dedisp_b200_fil_decimate(dedisp_byte* data, dedisp_size nchans, dedisp_size nsamps,
                                     dedisp_size factor);
/* <prefix>_DM<dm, %.3f>.dat (n float32 samples) and .inf (PRESTO text,
 * writeinf, fil.hpp:485-538). */
dedisp_error dedisp_b200_write_dat(const char* prefix, dedisp_float dm, const dedisp_float* series,
                                   dedisp_size n);
dedisp_error dedisp_b200_write_inf(const char* prefix, dedisp_float dm,
                                   const dedisp_b200_fil_header* header, dedisp_size numout);

/* Floats per DM row that execute() writes for nsamps input samples. */
dedisp_size dedisp_b200_output_row_length(dedisp_plan plan, dedisp_size nsamps);

#ifdef __cplusplus
}
#endif

#endif /* DEDISP_B200_H_INCLUDE_GUARD */
