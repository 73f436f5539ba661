// Launch interface of the tensor-core (tcgen05, 3xBF16) FDD phasor MAC.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "fdd_kernels.hpp"

namespace dedisp {
namespace kern {

struct TcMacArgs {
    float2* Yt;                // [nbins][nseg][ndm] (Y == nullptr)
    float2* Y;                 // DM-major [ndm * nseg][y_pitch] (time-series output), or nullptr
    size_t y_pitch;
    const float* dms;
    const float* delay_act;    // nact_pad entries (padding channels 0)
    const uint2* table;        // quarter-wave table, nfft/4 + 1 entries
    const float2* tw_lo;       // exp(-2 pi i t / nfft), t < 256
    const float2* tw_hi;       // exp(-2 pi i 256 h / nfft), h < nfft / 256
    unsigned* err;             // set to 1 if a bounded wait expired (single launches)
    int nact_pad;              // channels, multiple of 64
    int ndm;
    int nseg;                  // segments of this launch (2*nseg <= 128)
    int seg0 = 0;              // first segment of this launch in Yt / Y
    int nseg_total = 0;        // segments per bin in Yt / Y
    int npad;                  // 2*nseg rounded up to 16
    size_t nbins;
    unsigned nfft;             // transform length (multiple of 256; quarter-wave mode: a power of two)
    int round_delays;
    int dmax;                  // >= 0: delay-table mode, every delay in 0..dmax; -1: quarter-wave mode
    int direct = 0;            // dmax < 0: 1 phasors from the two-level twiddles, 0 quarter-wave table
    int hybrid = 0;            // dmax >= 0: 1 the table covers 0..dmax only, larger delays computed
    unsigned long long nmagic = 0;  // set by the launcher
};

// One item of a MAC launch: bins [k_begin, k_end) of DM tiles
// tile .. tile + ntile - 1 (128 DMs each) of descriptor `desc`; per bin the
// tiles run one after another.
struct TcWork {
    int desc;
    int tile;
    int ntile;
    unsigned k_begin;
    unsigned k_end;
};

// Shared-memory layout and wait settings of a launch (the largest over its
// descriptors, which share the channel set).
struct TcLayout {
    int stages;                // B pipeline depth
    int fused;                 // 1: fused MMA form (largest npad <= 80)
    int deep;                  // 1: three-MMA form with 3 A buffers (largest npad <= 64)
    int pair;                  // 1: CTA pairs (cta_group::2, M = 256, npad a multiple of 32)
    uint32_t stage_bytes;      // per stage (largest npad)
    uint32_t table_entries;    // phasor table (largest)
    uint32_t tw_hi_entries;    // two-level twiddle table, hi part (largest nfft / 256)
    int nact_pad;
    size_t smem_bytes;
    unsigned long long wait_ns;  // bounded-wait limit (rt::wait_limit_ns)
    int wait_test;               // expiry test (rt::wait_expiry_test)
    unsigned* err;               // set to 1 if a bounded wait expired
};

// Parameters of a MAC launch: descriptors and their tensor maps (kernel
// parameter bank), work items (device memory).
constexpr int kTcMaxDesc = 48;
// Dynamic shared memory a MAC launch may use (the opt-in maximum per block).
constexpr size_t kTcMaxSmem = 227 * 1024;
struct alignas(64) TcParams {
    CUtensorMap maps[kTcMaxDesc];
    TcMacArgs descs[kTcMaxDesc];
    int ndesc;
    const TcWork* items;
    int nitems;
    TcLayout layout;
    // optional: each CTA's busy time (ns, from after its set-up to its end),
    // one entry per CTA of the launch
    unsigned long long* cta_ns = nullptr;
    // items claimed beyond the first one per CTA (device, zeroed before each
    // launch; it follows the items in their buffer)
    unsigned* next_item = nullptr;
};

// One launch covers at most kTcMaxSeg segments (2 x segments <= 128
// accumulator columns); the engine runs segment groups.
constexpr int kTcMaxSeg = 64;
// Quarter-wave mode (the phasor table of exp(2 pi i r / N), r <= N/4) fits
// shared memory and N is a power of two (tc_choose_source weighs it against
// the per-bin delay table and the computed phasors).
bool tc_quarter_mode_fits(unsigned nfft, int nact_pad, int npad);
int tc_pad_channels(int nact);
int tc_pad_n(int nseg);
// Bytes of the split B operand of one segment group (2 nseg stored rows per
// bin and split; the MMA's padding rows are not stored).
size_t tc_b_bytes(size_t nbins, int nact_pad, int nseg);
size_t tc_smem_bytes(unsigned nfft, int nact_pad, int npad, int dmax, int stages, bool direct);
// Deepest B pipeline (2..6 stages) that fits shared memory.
int tc_stages(unsigned nfft, int nact_pad, int npad, int dmax, bool direct);
// Direct mode (every phasor from the two-level twiddle tables, any length
// that is a multiple of 256) fits shared memory.
bool tc_direct_mode_fits(unsigned nfft, int nact_pad, int npad);
// Shared-memory bytes of a launch whose layout holds `table_entries` phasors
// and `hi_entries` coarse twiddles (tc_layout's formula).
size_t tc_layout_bytes(int npad, size_t table_entries, size_t hi_entries, int nact_pad, int stages);
// Largest per-bin table extent (delays 0..cap) a layout with `hi_entries`
// coarse twiddles leaves room for; -1 if none.
int tc_table_capacity(int npad, size_t hi_entries, int nact_pad);

// Phasor source of one descriptor: dmax >= 0 the per-bin table over 0..dmax
// (hybrid: larger delays computed directly); dmax == -1 the quarter-wave
// table (direct = 0) or the twiddle tables (direct = 1); dmax == -2 none fits.
struct TcSource {
    int dmax = -1;
    int direct = 0;
    int hybrid = 0;
};
// Upper limit on the table extent from the environment (DEDISP_TC_TABLE_CAP,
// to compare the phasor sources on one shape); INT_MAX when unset.
int tc_table_cap_limit();
// Cheapest source for a largest delay `dmax` (-1: unknown or too large) when
// the layout leaves room for a table over 0..table_cap (-1: none) and, with
// quarter_fits, for the quarter-wave table.
TcSource tc_choose_source(int dmax, unsigned nfft, int table_cap, bool quarter_fits);
std::vector<uint2> tc_quarter_table(unsigned nfft);

// X [nchans*nseg][bin_pitch] complex spectra -> B operand
// Bsplit[bin][hi|lo][n < 2 nseg][kk < 2*nact_pad] (bf16).
// X rows in the order `map` (fdd_kernels.hpp).
// Segments seg0 .. seg0 + nseg - 1 of X rows c * nseg_total + s.
void launch_fdd_prep_b(const float2* X, size_t bin_pitch, int nseg, size_t nbins,
                       const int32_t* chan, const float* km, int nact, int nact_pad, int npad,
                       void* B, const BinMap& map, int seg0, int nseg_total, cudaStream_t s);

// One plan's MAC (one descriptor). d_items: device scratch of at least
// tc_work_bytes(SMs) bytes for its work items.
// Returns the MMA form that ran (tc_form_code).
int launch_fdd_mac_tc(const TcMacArgs& a, const void* B, void* d_items, size_t items_bytes, cudaStream_t s);
// 0 three-MMA form, 1 fused, 2 three-MMA with 3 A buffers, 3 CTA pairs, 4 CTA
// pairs with 3 A buffers, 5 fused at 64-channel chunks.
int tc_form_code(const TcLayout& L);

// Up to kTcMaxDesc descriptors in one persistent launch: work items over all
// of them (tc_work_items: one descriptor, at most `ctas` equal bin ranges;
// several, about 32 per CTA listed longest first; CTA b of the launch runs
// item b, then claims the next unclaimed one each time it finishes one),
// tensor maps encoded (B operand per descriptor) into P, items copied to
// d_items; then launched (possibly later, or inside a graph: P is copied into
// the launch, the claim counter is reset by a memset before it).
size_t tc_work_bytes(size_t nitems);
std::vector<TcWork> tc_work_items(const std::vector<TcMacArgs>& descs, int ctas);
void tc_prepare_list(TcParams& P, const std::vector<TcMacArgs>& descs, const std::vector<const void*>& Bs,
                     const std::vector<TcWork>& items, unsigned* err, void* d_items, size_t items_bytes,
                     cudaStream_t s);
void launch_fdd_mac_tc_list(const TcParams& P, cudaStream_t s);
int tc_sm_count();

}  // namespace kern
}  // namespace dedisp
