// Host arithmetic shared by the plans: the reference's delay table, DM list
// and delay rounding, written so each operation rounds exactly once in the
// reference's type (compile with -ffp-contract=off).
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace dedisp {
namespace hostmath {

// src/Plan.cpp:31,109-119 (channel width forced negative for the table).
inline void delay_table(size_t nchans, float dt, float f0, float df, float* out)
{
    df = -std::fabs(df);
    for (size_t c = 0; c < nchans; ++c) {
        const float a = 1.f / (f0 + (float)c * df);
        const float b = 1.f / f0;
        const float diff = a * a - b * b;
        out[c] = (float)(4.15e3 / (double)dt * (double)diff);
    }
}

// src/Plan.cpp:45-70. Returns false if the recurrence cannot advance (the
// reference would loop forever).
inline bool generate_dm_list(std::vector<float>& out, float dm_start, float dm_end,
                             double dt, double ti, double f0, double df,
                             size_t nchans, double tol)
{
    dt *= 1e6;
    const double f = (f0 + ((double)(nchans / 2) - 0.5) * df) * 1e-3;
    const double tol2 = tol * tol;
    const double a = 8.3 * df / (f * f * f);
    const double a2 = a * a;
    const double b2 = a2 * ((double)(nchans * nchans) / 16.0);
    const double c = (dt * dt + ti * ti) * (tol2 - 1.0);
    out.clear();
    out.push_back(dm_start);
    while (out.back() < dm_end) {
        const double prev = (double)out.back();
        const double prev2 = prev * prev;
        const double k = c + tol2 * a2 * prev2;
        const double dm = ((b2 * prev + std::sqrt(-a2 * b2 * prev2 + (a2 + b2) * k)) / (a2 + b2));
        const float next = (float)dm;
        if (!(next > out.back()) || out.size() > ((size_t)1 << 26)) return false;
        out.push_back(next);
    }
    return true;
}

// src/Plan.cpp:85-86: size_t(float(dm*delay) + 0.5), negative -> 0.
inline size_t max_delay(float dm_last, float delay_last)
{
    const float p = dm_last * delay_last;
    const double v = (double)p + 0.5;
    return v > 0.0 ? (size_t)v : 0;
}

// __float2uint_rn(dm*delay): round half to even, saturating.
inline uint32_t delay_rn(float dm, float delay)
{
    const float x = dm * delay;
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967295.5f) return 0xFFFFFFFFu;
    return (uint32_t)std::nearbyint(x);
}

// (int)(dm*delay): FDD truncation (src/fdd/dedisperse/fdd_kernel.cuh:226-229).
inline int32_t delay_trunc(float dm, float delay)
{
    const float x = dm * delay;
    if (x != x) return 0;
    if (x >= 2147483647.0f) return 2147483647;
    if (x <= -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)x;
}

}  // namespace hostmath
}  // namespace dedisp
