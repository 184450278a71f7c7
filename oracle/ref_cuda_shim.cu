// Test/baseline infrastructure only: C-callable wrappers over the REFERENCE's
// native CUDA astrocyte backend (src/astrocyte_cuda.cu, astrocyte_cuda.hpp:
// cuda_astro_create / update / push_input / pull_calcium / destroy), compiled
// from the reference sources for sm_100a by oracle/Makefile into
// oracle/_ref/libastroref_cuda.so.  bench.py times it beside the B200 kernel
// as the GPU bar to beat; the product never loads it.

#include "astrosimgpu/astrocyte_cuda.hpp"

#include <cuda_runtime.h>

using namespace astrosimgpu;

extern "C" {

void* refcu_create(unsigned n, const double* Ca, const double* IP3, const double* h,
                   const double* Ca_tot, const double* IP3_0, const double* tau_IP3,
                   const double* delta_IP3) {
    return cuda_astro_create(n, Ca, IP3, h, Ca_tot, IP3_0, tau_IP3, delta_IP3);
}

void refcu_destroy(void* s, double* Ca, double* IP3, double* h) {
    cuda_astro_destroy(static_cast<CudaAstro*>(s), Ca, IP3, h);
}

void refcu_push_input(void* s, const double* ip3_input) {
    cuda_astro_push_input(static_cast<CudaAstro*>(s), ip3_input);
}

void refcu_pull_calcium(void* s, double* Ca) {
    cuda_astro_pull_calcium(static_cast<CudaAstro*>(s), Ca);
}

// consts as in AstroConstants (Kd_IP3_1 ... ratio_ER_cyt).
void refcu_update(void* s, const double* consts, double h_step, int substeps, double noise_std,
                  int independent, double shared_noise, unsigned long long noise_seed,
                  unsigned long long noise_index) {
    AstroConstants c{consts[0], consts[1], consts[2], consts[3], consts[4],
                     consts[5], consts[6], consts[7], consts[8], consts[9]};
    cuda_astro_update(static_cast<CudaAstro*>(s), c, h_step, substeps, noise_std,
                      independent != 0, shared_noise, noise_seed, noise_index);
}

// Device-side timing of `steps` back-to-back kernel launches with CUDA events
// on the default stream (no per-step copies).  Returns milliseconds.
float refcu_time_updates(void* s, const double* consts, double h_step, int substeps, int steps) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a, 0);
    for (int i = 0; i < steps; ++i) {
        refcu_update(s, consts, h_step, substeps, 0.0, 1, 0.0, 0, 0);
    }
    cudaEventRecord(b, 0);
    cudaEventSynchronize(b);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

}  // extern "C"
