// SIGPROC filterbank input and PRESTO-style per-DM output (.dat/.inf), the
// file I/O of the reference's *_fil tools (bin/fil/fil.hpp) as a library.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "dedisp_b200.h"

namespace dedisp {
namespace sigproc {

// Parses the header of a SIGPROC filterbank file (keyword strings, each a
// 32-bit length then the characters, followed by a value of the keyword's
// type, from HEADER_START to HEADER_END). The sample count is taken from
// the data size, as the reference does (fil.hpp:366-370).
void read_header(const std::string& path, dedisp_b200_fil_header* h);

// Raw time-major rows [first, first + count) of the data section.
void read_samples(const std::string& path, const dedisp_b200_fil_header& h, size_t first, size_t count,
                  uint8_t* out);

// 8-bit rows averaged over `factor` consecutive samples per channel, float
// mean truncated to a byte (fil.hpp:31-52); full blocks only. Returns the
// new sample count.
size_t decimate8(uint8_t* data, size_t nchans, size_t nsamps, size_t factor);

// <prefix>_DM<dm %.3f>.dat: n float32 samples (fil.hpp:267-296).
void write_dat(const std::string& prefix, float dm, const float* series, size_t n);

// <prefix>_DM<dm %.3f>.inf in the PRESTO text layout of fil.hpp:485-538.
void write_inf(const std::string& prefix, float dm, const dedisp_b200_fil_header& h, size_t numout);

std::string dm_stem(const std::string& prefix, float dm);

}  // namespace sigproc
}  // namespace dedisp
