#include "asg_common.hpp"

#include <atomic>
#include <cstdlib>

namespace asg {

namespace {
thread_local std::string g_last_error;
std::atomic<long long> g_alloc_count{0};
}  // namespace

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

void clear_error() { g_last_error.clear(); }

int cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
    const int code = (e == cudaErrorMemoryAllocation) ? ASG_ERR_OOM
                     : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
                         ? ASG_ERR_NO_DEVICE
                         : ASG_ERR_CUDA;
    return fail(code, "CUDA error %s (%s) in %s at %s:%d", cudaGetErrorName(e),
                cudaGetErrorString(e), what, file, line);
}

bool injected_alloc_failure() {
    static const long long limit = [] {
        const char* v = std::getenv("ASG_FAIL_ALLOC_AFTER");
        return v ? std::atoll(v) : -1LL;
    }();
    if (limit < 0) return false;
    return g_alloc_count.fetch_add(1) >= limit;
}

int DevBuf::alloc(std::size_t bytes, bool zero) {
    release();
    if (bytes == 0) return ASG_OK;
    if (injected_alloc_failure()) {
        return fail(ASG_ERR_OOM, "device allocation of %zu bytes refused (injected failure)",
                    bytes);
    }
    ASG_CUDA(cudaMalloc(&p_, bytes));
    n_ = bytes;
    if (zero) {
        // The engines work on non-blocking streams, which do not wait for the
        // legacy stream: finish the zeroing here, or a later copy on an
        // engine stream could land first and be overwritten.
        ASG_CUDA(cudaMemsetAsync(p_, 0, bytes, cudaStreamLegacy));
        ASG_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
    }
    return ASG_OK;
}

void DevBuf::release() {
    if (p_ != nullptr) cudaFree(p_);
    p_ = nullptr;
    n_ = 0;
}

}  // namespace asg

extern "C" const char* asg_last_error(void) { return asg::g_last_error.c_str(); }
extern "C" const char* asg_version(void) { return "astrosim-b200 0.1 (sm_100a, fp64)"; }
