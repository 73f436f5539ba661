// Launch interface of the time-domain (TDD) kernels.
//
// Device layout ("channel-major packed"): channel c of a gulp is a row of
// 32-bit words at tr + c * tr_pitch_words; word w holds samples
// w*spw .. w*spw+spw-1 (spw = 32/nbits), sample i of the word at bits
// i*nbits, LSB first. Row `nchans` is an all-zero row used to pad channel
// lists. The same little-endian packing as the input format, with time and
// channel swapped.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace dedisp {
namespace kern {

// K1: time-major packed rows -> channel-major packed rows.
struct TransposeArgs {
    const uint8_t* in;      // row r at in + r * in_pitch
    size_t in_pitch;        // bytes
    size_t rows_valid;      // rows present in `in`; later samples are zero
    size_t nchans;
    int nbits;
    uint32_t* tr;           // channel-major output
    size_t tr_pitch_words;  // words between channel rows
    size_t tr_word_offset;  // first word written in each row (= first row / spw)
    size_t tr_words;        // words written per row from there (zeros past rows_valid)
};
void launch_transpose(const TransposeArgs& a, cudaStream_t s);

// K2: dedispersion of one gulp.
struct DedisperseArgs {
    const uint32_t* tr;
    size_t tr_pitch_words;
    int nbits;
    size_t nchans;              // total channels (epilogue normalisation)
    const int32_t* chan_list;   // active channels, padded with `nchans`
    int nact;                   // active channels (plain kernel loop bound)
    int nstages;                // tiled: padded list length / chan_per_stage
    const uint32_t* km_vals;    // plain: multiplier per active channel
    const float* delay_table;   // nchans + 1 entries, last one 0
    const float* chan_delay;    // quad: delay_table[chan_list[j]] per list entry
    const float* dms;           // DM per slot (sorted ascending for tiled)
    const int32_t* perm;        // output row of slot i (nullptr: identity)
    int ndm;
    size_t nsamp_out;           // output samples in this gulp
    void* out;                  // row r at out + r * out_stride elements
    size_t out_stride;          // elements
    int out_nbits;              // 8, 16 or 32 (float)
    float den;                  // (float)(2^nbits-1) * (float)nchans
    float factor;               // (3.f*1024.f)/255.f/16.f
    int win_words;              // tiled: staged window per channel (words)
    int chan_per_stage;         // tiled: channels per pipeline stage (even)
    int variant;                // tiled: tile-shape variant (8-bit input)
    unsigned* err;              // quad-strided: device word set to 1 when a bounded
                                // wait on the staged copies expired (required)
};

// Tile geometry of the tiled kernel for a given input width and tile-shape
// variant (tiled_variant_count per width: 8-bit 9, 1/2/4-bit 5, 16/32-bit 1).
// Quad-strided variants (tiled_variant_quad: 8-bit 5-8, 1/2/4-bit 1-4) run
// on quad-strided rows: word n of a row holds samples n + i*P of the channel
// in byte i (i = 0..3, P = 32 * tiled_lane_words; narrower samples widened
// to bytes), built from the input rows by launch_quad_direct.
int tiled_variant_count(int nbits);
int tiled_batch_variant_count(int nbits);  // variants of the persistent batch kernel (all)
int tiled_default_variant(int nbits);      // the variant a plan uses unless told otherwise
bool tiled_variant_quad(int nbits, int variant);
int tiled_block_samples(int nbits, int variant);  // output samples per block
int tiled_block_dms(int nbits, int variant);      // DMs per block
int tiled_lane_words(int nbits, int variant);     // J: words per lane
size_t tiled_smem_bytes(int nbits, int win_words, int chan_per_stage, int variant);
size_t tiled_max_smem_bytes();
// Dynamic shared memory of the persistent batch launch for a beam's window.
size_t tiled_batch_smem_bytes(int nbits, int win_words, int chan_per_stage, int variant);
// Channels per pipeline stage for a window of win_words (0: does not fit).
int tiled_stage_channels(int nbits, int win_words, int variant);

// K1d: quad-strided rows straight from time-major packed 1/2/4/8-bit input:
// rows 0..nchans-1 of q, word n of channel c holding samples n + i*P
// (i = 0..3) of the channel as bytes, zero at or past rows_valid. The
// all-zero padding row is the caller's.
struct QuadDirectArgs {
    const uint8_t* in;    // input row t at in + t * in_pitch
    size_t in_pitch;      // bytes
    size_t rows_valid;    // rows present in `in`
    size_t nchans;
    int nbits;            // 1, 2, 4 or 8
    uint32_t* q;          // quad-strided rows, q_pitch_words apart
    size_t q_pitch_words; // words per row (a multiple of 4), all written
    int period_words;     // P, a multiple of 4
};
void launch_quad_direct(const QuadDirectArgs& a, cudaStream_t s);

// Value of a kernel error word (synchronises s first).
unsigned read_error_word(const unsigned* d_err, cudaStream_t s);

void launch_dedisperse_plain(const DedisperseArgs& a, cudaStream_t s);
void launch_dedisperse_tiled(const DedisperseArgs& a, cudaStream_t s);

// Persistent tiled kernel over many series (8-bit packed-row variants and
// the quad-strided variants of widths up to 8 bits): args[beam] describes beam
// `beam` (device array), its tiles are items item_start[beam] ..
// item_start[beam+1]-1 (nbeams+1 entries, device), nbx[beam] DM blocks per
// time tile (device). smem_bytes: the largest tiled_batch_smem_bytes of the
// beams. Quad-strided variants read quad-strided rows (args[beam].tr).
struct BatchLaunch {
    const DedisperseArgs* args;
    const unsigned long long* item_start;
    const int* nbx;
    int nbeams;
    unsigned long long total_items;
    size_t smem_bytes;
};
void launch_dedisperse_tiled_batch(const BatchLaunch& b, int nbits, int variant, cudaStream_t s);

}  // namespace kern
}  // namespace dedisp
