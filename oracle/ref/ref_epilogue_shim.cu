// Test infrastructure only: host-side C entry points around the reference's
// __host__ __device__ helpers scale_output / extract_subword, taken by include
// from src/tdd/dedisperse/dedisperse_kernel.cuh (REF_EPI_LEGACY=0) or the
// legacy src/dedisp/dedisperse/dedisperse_kernel.cuh (REF_EPI_LEGACY=1); each
// variant is its own translation unit because each header declares 64 KB of
// __constant__ tables. Compiled by oracle/ref/Makefile; pins the oracle's TDD
// epilogue bit for bit.
#include <cstdint>

// The reference headers include these at their top.
#include <cuda_runtime.h>
#include <device_launch_parameters.h>
#include <texture_fetch_functions.h>

#include "common/dedisp_types.h"

#if REF_EPI_LEGACY
#define DEDISP_MAX_NCHANS 8192
#include "dedisp/dedisperse/dedisperse_kernel.cuh"
#define REF_SCALE_FN ref_scale_output_legacy
#else
#include "tdd/dedisperse/dedisperse_kernel.cuh"
#define REF_SCALE_FN ref_scale_output_tdd
#endif

namespace {
template <int IN>
void scale(uint64_t sum, int out_nbits, dedisp_size nchans, void* out)
{
    using S = typename SumType<IN>::type;
    S s = (S)sum;
    switch (out_nbits) {
    case 8: *(unsigned char*)out = scale_output<IN, unsigned char>(s, nchans); break;
    case 16: *(unsigned short*)out = scale_output<IN, unsigned short>(s, nchans); break;
    default: *(float*)out = scale_output<IN, float>(s, nchans); break;
    }
}
}  // namespace

extern "C" {

// Returns 0 on success, -1 for an unsupported in_nbits.
int REF_SCALE_FN(uint64_t sum, int in_nbits, int out_nbits,
                 unsigned long nchans, void* out)
{
    switch (in_nbits) {
    case 1: scale<1>(sum, out_nbits, nchans, out); return 0;
    case 2: scale<2>(sum, out_nbits, nchans, out); return 0;
    case 4: scale<4>(sum, out_nbits, nchans, out); return 0;
    case 8: scale<8>(sum, out_nbits, nchans, out); return 0;
    case 16: scale<16>(sum, out_nbits, nchans, out); return 0;
    case 32: scale<32>(sum, out_nbits, nchans, out); return 0;
    default: return -1;
    }
}

#if !REF_EPI_LEGACY
unsigned int ref_extract_subword(unsigned int word, int in_nbits, int idx)
{
    switch (in_nbits) {
    case 1: return extract_subword<1>(word, idx);
    case 2: return extract_subword<2>(word, idx);
    case 4: return extract_subword<4>(word, idx);
    case 8: return extract_subword<8>(word, idx);
    case 16: return extract_subword<16>(word, idx);
    default: return extract_subword<32>(word, idx);
    }
}
#endif

}  // extern "C"
