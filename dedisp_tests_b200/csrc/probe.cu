// Integer-pipe throughput probe: a measurement tool of the benchmark, built
// into its own library (lib/libdedisp_probe.so), not into libdedisp.so. It
// states the roofline of the TDD kernel, which is bound by 32-bit integer
// instruction issue rather than by HBM or tensor cores.
//
// Each thread runs 8 independent chains of 32-bit adds; the result is the
// measured rate of 32-bit integer add lane-operations per second on the
// device, with every SM fully occupied.
#include <cuda_runtime.h>

#include <cstdint>

#include "dedisp.h"

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

// 32-bit integer add lane-operations per second on `device` (the caller's
// current device is restored).
extern "C" dedisp_error dedisp_probe_alu(int device, double* lane_adds_per_s)
{
    if (!lane_adds_per_s) return DEDISP_INVALID_POINTER;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return DEDISP_INVALID_DEVICE_INDEX;
    }
    cudaDeviceProp prop;
    uint32_t* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float ms = 0.f;
    const int threads = 512, iters = 4096;
    int blocks = 0;
    bool ok = cudaGetDeviceProperties(&prop, device) == cudaSuccess;
    if (ok) {
        blocks = prop.multiProcessorCount * 4;
        ok = cudaMalloc(&sink, blocks * sizeof(uint32_t)) == cudaSuccess &&
             cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
    }
    if (ok) {
        alu_probe_kernel<<<blocks, threads>>>(sink, 64, 7u);  // warm-up
        cudaEventRecord(e0);
        for (int r = 0; r < 5; ++r) alu_probe_kernel<<<blocks, threads>>>(sink, iters, 7u + r);
        cudaEventRecord(e1);
        ok = cudaGetLastError() == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
             cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms > 0.f;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (sink) cudaFree(sink);
    cudaSetDevice(prev);
    if (!ok) {
        cudaGetLastError();
        return DEDISP_INTERNAL_GPU_ERROR;
    }
    const double ops = 5.0 * blocks * threads * (double)iters * 16.0;
    *lane_adds_per_s = ops / (ms * 1e-3);
    return DEDISP_NO_ERROR;
}
