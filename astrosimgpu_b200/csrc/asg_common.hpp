// Host-side helpers shared by the engine's translation units: thread-local
// error text behind asg_last_error(), status-returning CUDA checks, and a
// device-buffer owner.  Nothing here aborts: every failure becomes a status
// code that travels back through the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "asg_b200.h"

namespace asg {

// Records `fmt` as this thread's last error and returns `code`.
int fail(int code, const char* fmt, ...);
void clear_error();

// Maps a CUDA error to ASG_ERR_OOM / ASG_ERR_CUDA with the call site.
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define ASG_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t asg_e_ = (call);                                                     \
        if (asg_e_ != cudaSuccess) return ::asg::cuda_fail(asg_e_, #call, __FILE__, __LINE__); \
    } while (0)

#define ASG_TRY(expr)              \
    do {                           \
        int asg_s_ = (expr);       \
        if (asg_s_ != ASG_OK) return asg_s_; \
    } while (0)

// Test hook: when the environment variable ASG_FAIL_ALLOC_AFTER=n is set,
// the (n+1)-th device allocation of the process fails with out-of-memory.
// Lets the host error paths be exercised without exhausting a shared GPU.
bool injected_alloc_failure();

// Host-side NVTX range over a scope, named after the reference's phase
// table where one applies (Network::run's PhaseProfile, network.hpp:32-45:
// "update astrocytes", "SIC gather+deliver", ...).  Seen by Nsight Systems
// and by ncu's --nvtx filters; costs a call into the NVTX stub when no tool
// is attached.
class NvtxRange {
public:
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Owning device allocation (cudaMalloc / cudaFree), zero-filled on request.
class DevBuf {
public:
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
        return *this;
    }
    ~DevBuf() { release(); }

    int alloc(std::size_t bytes, bool zero = true);
    void release();
    void* get() const { return p_; }
    template <typename T> T* as() const { return static_cast<T*>(p_); }
    std::size_t bytes() const { return n_; }

private:
    void* p_ = nullptr;
    std::size_t n_ = 0;
};

}  // namespace asg
