// Thin RAII layer over the CUDA runtime: device buffers that only grow,
// pinned host buffers, streams, events and a device guard. Plays the part of
// the reference's cu:: wrapper (src/common/cuda/CU.h), designed for reuse of
// large HBM buffers across execute() calls.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <utility>

#include "errors.hpp"

namespace dedisp {
namespace rt {

// Throws dedisp::Error(DEDISP_INTERNAL_GPU_ERROR, or MEM_ALLOC_FAILED for
// allocation failures) naming the failed call.
void check(cudaError_t e, const char* what, const char* file, int line);
#define RT_CHECK(call) ::dedisp::rt::check((call), #call, __FILE__, __LINE__)

// True when the CUDA runtime reports an error raised before this call by
// someone else (src/clib/dedisp.cpp:117-119). A process without a usable
// driver or device is not treated as a prior error.
bool prior_gpu_error();

// Number of usable devices (0 without a driver or device).
int device_count();

class DeviceGuard {
public:
    explicit DeviceGuard(int device);
    ~DeviceGuard();
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;

private:
    int m_prev = -1;
};

class DeviceBuffer {
public:
    DeviceBuffer() = default;
    ~DeviceBuffer() { release(); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;

    // Ensures capacity >= bytes; contents are not preserved on growth.
    void reserve(size_t bytes);
    void release();
    template <typename T = void>
    T* get() const { return static_cast<T*>(m_ptr); }
    size_t capacity() const { return m_cap; }

private:
    void* m_ptr = nullptr;
    size_t m_cap = 0;
};

class PinnedBuffer {
public:
    PinnedBuffer() = default;
    ~PinnedBuffer() { release(); }
    PinnedBuffer(const PinnedBuffer&) = delete;
    PinnedBuffer& operator=(const PinnedBuffer&) = delete;
    void reserve(size_t bytes);
    void release();
    template <typename T = void>
    T* get() const { return static_cast<T*>(m_ptr); }
    size_t capacity() const { return m_cap; }

private:
    void* m_ptr = nullptr;
    size_t m_cap = 0;
};

class Stream {
public:
    Stream();
    ~Stream();
    Stream(const Stream&) = delete;
    Stream& operator=(const Stream&) = delete;
    cudaStream_t get() const { return m_s; }
    operator cudaStream_t() const { return m_s; }

private:
    cudaStream_t m_s = nullptr;
};

class Event {
public:
    explicit Event(bool timing = false);
    ~Event();
    Event(const Event&) = delete;
    Event& operator=(const Event&) = delete;
    cudaEvent_t get() const { return m_e; }
    operator cudaEvent_t() const { return m_e; }
    void record(cudaStream_t s);

private:
    cudaEvent_t m_e = nullptr;
};

// True when p is host memory the GPU can DMA from directly (pinned or
// registered), so copies can be asynchronous without staging.
bool is_pinned_host(const void* p);

// Raise kernel `kfn`'s dynamic shared-memory limit on the current device to
// at least `bytes`. The limit only grows: each (kernel, device) keeps the
// largest value set so far, under one lock, so that a thread launching with
// a larger limit never has it lowered by another thread in between.
void raise_smem_limit(const void* kfn, size_t bytes);
template <typename K>
void raise_smem_limit(K* kfn, size_t bytes)
{
    raise_smem_limit(reinterpret_cast<const void*>(kfn), bytes);
}

// Kernels that poll an mbarrier for their own asynchronous copies or
// tensor-core work (the quad-strided TDD kernels, the tensor-core FDD MAC)
// give up after this many nanoseconds of global time, record an error that
// the plan reports as DEDISP_INTERNAL_GPU_ERROR, wait (again bounded) for
// their own work in flight and return. Process-wide; read at each launch.
constexpr unsigned long long kDefaultWaitLimitNs = 2000000000ull;
unsigned long long wait_limit_ns();
void set_wait_limit_ns(unsigned long long ns);  // 0 restores the default (2 s)
// Expiry test: each such kernel additionally waits (bounded by the limit)
// on an mbarrier that nothing arrives on, at the first wait of its
// pipeline, so the expiry path runs deterministically.
bool wait_expiry_test();
void set_wait_expiry_test(bool on);

}  // namespace rt
}  // namespace dedisp
