// Integer-pipe throughput probe (extension, used by the benchmark to state
// the roofline of the TDD kernel, which is bound by 32-bit integer
// instruction issue rather than by HBM or tensor cores).
//
// Each thread runs 8 independent chains of 32-bit adds; the result is the
// measured rate of 32-bit integer add lane-operations per second on the
// device, with every SM fully occupied.
#include <cuda_runtime.h>

#include <cstdint>

#include "dedisp_b200.h"
#include "runtime.hpp"

namespace {

__global__ void __launch_bounds__(512) alu_probe_kernel(uint32_t* sink, int iters, uint32_t seed)
{
    uint32_t a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + threadIdx.x * 8 + k;
    const uint32_t inc = seed | 1u;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            // two dependent adds per step per chain; asm keeps them as adds
            asm volatile("add.u32 %0, %0, %1;" : "+r"(a[k]) : "r"(inc));
            asm volatile("add.u32 %0, %0, %1;" : "+r"(a[k]) : "r"(a[(k + 1) & 7]));
        }
    }
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s ^= a[k];
    if (s == 0x12345678u) sink[blockIdx.x] = s;  // keep the chains alive
}

}  // namespace

extern "C" dedisp_error dedisp_b200_alu_probe(int device, double* lane_adds_per_s)
{
    try {
        dedisp::rt::DeviceGuard guard(device);
        cudaDeviceProp prop;
        RT_CHECK(cudaGetDeviceProperties(&prop, device));
        const int blocks = prop.multiProcessorCount * 4;
        const int threads = 512;
        const int iters = 4096;
        uint32_t* sink = nullptr;
        RT_CHECK(cudaMalloc(&sink, blocks * sizeof(uint32_t)));
        cudaEvent_t e0, e1;
        RT_CHECK(cudaEventCreate(&e0));
        RT_CHECK(cudaEventCreate(&e1));
        alu_probe_kernel<<<blocks, threads>>>(sink, 64, 7u);  // warm-up
        RT_CHECK(cudaEventRecord(e0));
        for (int r = 0; r < 5; ++r) alu_probe_kernel<<<blocks, threads>>>(sink, iters, 7u + r);
        RT_CHECK(cudaEventRecord(e1));
        RT_CHECK(cudaEventSynchronize(e1));
        float ms = 0.f;
        RT_CHECK(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFree(sink);
        const double ops = 5.0 * blocks * threads * (double)iters * 16.0;
        *lane_adds_per_s = ops / (ms * 1e-3);
        return DEDISP_NO_ERROR;
    } catch (...) {
        return DEDISP_INTERNAL_GPU_ERROR;
    }
}
