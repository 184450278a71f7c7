// The reference's native CUDA astrocyte backend (include/astrosimgpu/
// astrocyte_cuda.hpp:15-27, src/astrocyte_cuda.cu) bound to the B200 engine:
// the five calls AstrocytePopulation makes under ASTROSIMGPU_CUDA
// (src/astrocyte.cpp:83-89, 126-132, 169-174, 195-200, 261-267), each one
// asg_astro_* call.  Linking this file in place of astrocyte_cuda.cu gives
// the reference's host step with the astrocyte update on the engine: the
// same movement points (create with resident state, push the step's input,
// update, pull calcium, destroy with the state copied back).
//
// The reference's backend aborts on a CUDA error; here a failing status is
// thrown with the engine's error text (the reference's main catches and
// reports exceptions).
#include <stdexcept>
#include <string>

#include "asg_b200.h"
#include "astrosimgpu/astrocyte_cuda.hpp"

namespace astrosimgpu {

struct CudaAstro {
    asg_astro* engine = nullptr;
};

namespace {

void check(int status, const char* what) {
    if (status != ASG_OK)
        throw std::runtime_error(std::string("B200 astrocyte backend: ") + what + ": " +
                                 asg_last_error());
}

}  // namespace

CudaAstro* cuda_astro_create(index_t n, const real* Ca, const real* IP3, const real* h,
                             const real* Ca_tot, const real* IP3_0, const real* tau_IP3,
                             const real* delta_IP3) {
    auto* s = new CudaAstro;
    const int st = asg_astro_create(n, Ca, IP3, h, Ca_tot, IP3_0, tau_IP3, delta_IP3, &s->engine);
    if (st != ASG_OK) delete s;
    check(st, "create");
    return s;
}

void cuda_astro_destroy(CudaAstro* s, real* Ca, real* IP3, real* h) {
    const int st = asg_astro_destroy(s->engine, Ca, IP3, h);
    delete s;
    check(st, "destroy");
}

void cuda_astro_push_input(CudaAstro* s, const real* ip3_input) {
    check(asg_astro_push_input(s->engine, ip3_input), "push_input");
}

void cuda_astro_pull_calcium(CudaAstro* s, real* Ca) {
    check(asg_astro_pull_calcium(s->engine, Ca), "pull_calcium");
}

void cuda_astro_update(CudaAstro* s, const AstroConstants& c, real h_step, int substeps,
                       real noise_std, bool independent_noise, real shared_noise,
                       std::uint64_t noise_seed, std::uint64_t noise_index) {
    const double k[10] = {c.Kd_IP3_1, c.Kd_IP3_2, c.Kd_act,    c.Kd_inh,     c.Km_SERCA,
                          c.k_IP3R,   c.rate_IP3R, c.rate_L, c.rate_SERCA, c.ratio_ER_cyt};
    check(asg_astro_update(s->engine, k, h_step, substeps, noise_std, independent_noise ? 1 : 0,
                           shared_noise, noise_seed, noise_index),
          "update");
}

}  // namespace astrosimgpu
