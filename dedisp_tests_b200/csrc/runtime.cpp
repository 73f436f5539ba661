// CUDA runtime RAII helpers (see runtime.hpp) and the error helpers.
#include "runtime.hpp"

#include <atomic>

#include <cstdio>
#include <map>
#include <mutex>
#include <sstream>

namespace dedisp {

void throw_error_at(dedisp_error code, const char* file, int line,
                    const char* detail)
{
    std::stringstream msg;
    msg << "An error occurred within dedisp on line " << line << " of " << file
        << ": " << dedisp_get_error_string(code);
    if (detail) msg << " (" << detail << ")";
    throw Error(code, msg.str());
}

namespace rt {

void check(cudaError_t e, const char* what, const char* file, int line)
{
    if (e == cudaSuccess) return;
    dedisp_error code = (e == cudaErrorMemoryAllocation)
                            ? DEDISP_MEM_ALLOC_FAILED
                            : DEDISP_INTERNAL_GPU_ERROR;
    std::string detail = std::string(what) + ": " + cudaGetErrorString(e);
    throw_error_at(code, file, line, detail.c_str());
}

bool prior_gpu_error()
{
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return false;
    // No driver / no device: nothing can have failed on a GPU before us.
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ||
        e == cudaErrorInitializationError || e == cudaErrorStubLibrary ||
        e == cudaErrorSystemDriverMismatch || e == cudaErrorCompatNotSupportedOnDevice)
        return false;
    return true;
}

int device_count()
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();  // clear the sticky-free error
        return 0;
    }
    return n;
}

DeviceGuard::DeviceGuard(int device)
{
    if (cudaGetDevice(&m_prev) != cudaSuccess) m_prev = -1;
    if (m_prev != device) RT_CHECK(cudaSetDevice(device));
}

DeviceGuard::~DeviceGuard()
{
    int cur = -1;
    if (m_prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != m_prev)
        cudaSetDevice(m_prev);
}

void DeviceBuffer::reserve(size_t bytes)
{
    if (bytes <= m_cap) return;
    release();
    if (bytes == 0) return;
    RT_CHECK(cudaMalloc(&m_ptr, bytes));
    m_cap = bytes;
}

void DeviceBuffer::release()
{
    if (m_ptr) cudaFree(m_ptr);
    m_ptr = nullptr;
    m_cap = 0;
}

void PinnedBuffer::reserve(size_t bytes)
{
    if (bytes <= m_cap) return;
    release();
    if (bytes == 0) return;
    RT_CHECK(cudaHostAlloc(&m_ptr, bytes, cudaHostAllocPortable));
    m_cap = bytes;
}

void PinnedBuffer::release()
{
    if (m_ptr) cudaFreeHost(m_ptr);
    m_ptr = nullptr;
    m_cap = 0;
}

Stream::Stream() { RT_CHECK(cudaStreamCreateWithFlags(&m_s, cudaStreamNonBlocking)); }
Stream::~Stream()
{
    if (m_s) cudaStreamDestroy(m_s);
}

Event::Event(bool timing)
{
    RT_CHECK(cudaEventCreateWithFlags(&m_e, timing ? cudaEventDefault
                                                   : cudaEventDisableTiming));
}
Event::~Event()
{
    if (m_e) cudaEventDestroy(m_e);
}
void Event::record(cudaStream_t s) { RT_CHECK(cudaEventRecord(m_e, s)); }

bool is_pinned_host(const void* p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

void raise_smem_limit(const void* kfn, size_t bytes)
{
    static std::mutex m;
    static std::map<std::pair<const void*, int>, size_t> set;
    int dev = 0;
    RT_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(m);
    size_t& have = set[{kfn, dev}];
    if (bytes <= have) return;
    RT_CHECK(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    have = bytes;
}

namespace {
std::atomic<unsigned long long> g_wait_limit_ns{kDefaultWaitLimitNs};
std::atomic<bool> g_wait_expiry_test{false};
}  // namespace

unsigned long long wait_limit_ns() { return g_wait_limit_ns.load(); }
void set_wait_limit_ns(unsigned long long ns) { g_wait_limit_ns.store(ns ? ns : kDefaultWaitLimitNs); }
bool wait_expiry_test() { return g_wait_expiry_test.load(); }
void set_wait_expiry_test(bool on) { g_wait_expiry_test.store(on); }

}  // namespace rt
}  // namespace dedisp
