// FDD execution engine (placeholder until the Fourier-domain kernels land).
#include "fdd_engine.hpp"

namespace dedisp {
namespace detail {

struct FddEngine::Impl {};

FddEngine::FddEngine(GpuState& gpu) : m_gpu(gpu), m_impl(new Impl()) {}
FddEngine::~FddEngine() {}

void FddEngine::execute(const FddOptions&, const FddView&, const FddCall&)
{
    m_gpu.require_device();
    DD_THROW_MSG(DEDISP_UNKNOWN_ERROR, "FDD execution not available in this build");
}

}  // namespace detail
}  // namespace dedisp
