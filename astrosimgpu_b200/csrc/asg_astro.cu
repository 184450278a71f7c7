// Astrocyte-only engine: the drop-in for the reference's native CUDA
// astrocyte backend (astrocyte_cuda.hpp:15-27, astrocyte_cuda.cu:27-155) and
// the astrocyte kernel-scaling workload with its input generated on the
// device.
//
// Layout: SoA FP64 arrays Ca, IP3, h (+ Ca_tot, IP3_0, tau_IP3, delta_IP3
// when per-cell), 256-byte aligned.  Each thread owns two adjacent cells so
// every state array is read and written with one coalesced 128-bit access
// per thread, and the two independent RK4 chains interleave to cover FP64
// latency.  Grid-stride loop over cell pairs; grid sized in multiples of
// the SM count.
//
// Compiled with -fmad=false: results are bitwise equal to the host's
// astro_advance (no transcendental on this path when noise is off).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "asg_common.hpp"
#include "asg_device.cuh"

namespace asg {

namespace {

struct AstroArrays {
    double* Ca;
    double* IP3;
    double* h;
    double* input;  // per-step input (drop-in path) or nullptr
    const double* Ca_tot;
    const double* IP3_0;
    const double* tau;
    const double* inv_tau;  // correctly rounded 1/tau_IP3 per cell (host-formed)
    const double* delta;
};

struct UniformParams {
    double Ca_tot, IP3_0, tau, delta, inv_tau;
};

// Where a step's IP3 input comes from:
//   kInputArrayZero  the input array, zeroed after use (the reference kernel's
//                    contract; the allocation-free entry point, whose array
//                    belongs to the caller)
//   kInputBernoulli  generated on the device (the kernel-scaling workload)
//   kInputArray      the input array, left as it is: the resident engine
//                    knows the caller's next push overwrites all of it
//   kInputNone       zero input (no push since the last update), not read
enum InputMode { kInputArrayZero = 0, kInputBernoulli = 1, kInputArray = 2, kInputNone = 3 };

struct StepArgs {
    std::int64_t n;
    AstroK k;
    UniformParams u;
    // noise (drop-in path)
    double noise_std;
    int independent;
    double shared_noise;
    std::uint64_t noise_seed, noise_index;
    // Bernoulli input (scaling path): an event when the draw's 53-bit integer
    // k satisfies k < p_threshold = ceil(p * 2^53), which is exactly
    // k * 2^-53 < p (the reference's rng_uniform(...) < p) in integers.
    std::uint64_t seed;
    double p, weight;
    std::uint64_t p_threshold;
    const std::int64_t* step_base;  // device counter: step = *step_base + step_offset
    int step_offset;
    std::int64_t i0;  // global index of the first cell of this launch (RNG streams)
};

template <bool kUniform, int kInput, bool kNoise>
__device__ __forceinline__ void advance_cell(const StepArgs& a, const AstroArrays& s,
                                             std::int64_t i, std::int64_t step, double& ca,
                                             double& ip3, double& hh) {
    double in;
    if (kInput == kInputBernoulli) {
        in = (mix64(a.seed, static_cast<std::uint64_t>(a.i0 + i),
                    1000ULL + static_cast<std::uint64_t>(step)) >> 11) < a.p_threshold
                 ? a.weight
                 : 0.0;
    } else if (kInput == kInputNone) {
        in = 0.0;
    } else {
        in = s.input[i];
    }
    // kNoise: independent per-cell draws; otherwise the step's shared value
    // (0 with noise off, as the reference passes it).
    const double noise =
        kNoise ? a.noise_std * normal_clamped(a.noise_seed, a.noise_index * kStreamStride +
                                                                static_cast<std::uint64_t>(a.i0 + i))
               : a.shared_noise;
    if (kUniform) {
        astro_rk4(a.k, a.u.Ca_tot, a.u.IP3_0, a.u.tau, a.u.inv_tau, a.u.delta, in, noise, ca, ip3,
                  hh);
    } else {
        astro_rk4(a.k, s.Ca_tot[i], s.IP3_0[i], s.tau[i], s.inv_tau[i], s.delta[i], in, noise, ca,
                  ip3, hh);
    }
}

// kCells adjacent cells per thread (1: 64-bit accesses, 2: 128-bit accesses
// and two interleaved RK4 chains); kMinBlocks sets the register budget
// through __launch_bounds__ (65536 / (kBlock * kMinBlocks) per thread).
template <bool kUniform, int kInput, bool kNoise, int kCells, int kBlock, int kMinBlocks>
__global__ void __launch_bounds__(kBlock, kMinBlocks) astro_step_kernel(StepArgs a, AstroArrays s) {
    const std::int64_t step =
        (kInput == kInputBernoulli) ? (*a.step_base + a.step_offset) : 0;
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    if (kCells == 4) {
        // Four adjacent cells per thread (two 128-bit accesses per array):
        // four independent RK4 chains to interleave.
        const std::int64_t quads = a.n / 4;
        double2* Ca2 = reinterpret_cast<double2*>(s.Ca);
        double2* IP32 = reinterpret_cast<double2*>(s.IP3);
        double2* h2 = reinterpret_cast<double2*>(s.h);
        for (std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
             q < quads; q += stride) {
            double2 ca0 = Ca2[2 * q], ip30 = IP32[2 * q], hh0 = h2[2 * q];
            double2 ca1 = Ca2[2 * q + 1], ip31 = IP32[2 * q + 1], hh1 = h2[2 * q + 1];
            const std::int64_t i = 4 * q;
            advance_cell<kUniform, kInput, kNoise>(a, s, i, step, ca0.x, ip30.x, hh0.x);
            advance_cell<kUniform, kInput, kNoise>(a, s, i + 1, step, ca0.y, ip30.y, hh0.y);
            advance_cell<kUniform, kInput, kNoise>(a, s, i + 2, step, ca1.x, ip31.x, hh1.x);
            advance_cell<kUniform, kInput, kNoise>(a, s, i + 3, step, ca1.y, ip31.y, hh1.y);
            Ca2[2 * q] = ca0;
            IP32[2 * q] = ip30;
            h2[2 * q] = hh0;
            Ca2[2 * q + 1] = ca1;
            IP32[2 * q + 1] = ip31;
            h2[2 * q + 1] = hh1;
            if (kInput == kInputArrayZero) {
                reinterpret_cast<double2*>(s.input)[2 * q] = make_double2(0.0, 0.0);
                reinterpret_cast<double2*>(s.input)[2 * q + 1] = make_double2(0.0, 0.0);
            }
        }
        // Up to three tail cells.
        if (blockIdx.x == 0 && threadIdx.x < static_cast<unsigned>(a.n & 3)) {
            const std::int64_t i = 4 * quads + threadIdx.x;
            double ca = s.Ca[i], ip3 = s.IP3[i], hh = s.h[i];
            advance_cell<kUniform, kInput, kNoise>(a, s, i, step, ca, ip3, hh);
            s.Ca[i] = ca;
            s.IP3[i] = ip3;
            s.h[i] = hh;
            if (kInput == kInputArrayZero) s.input[i] = 0.0;
        }
    } else if (kCells == 2) {
        const std::int64_t pairs = a.n / 2;
        double2* Ca2 = reinterpret_cast<double2*>(s.Ca);
        double2* IP32 = reinterpret_cast<double2*>(s.IP3);
        double2* h2 = reinterpret_cast<double2*>(s.h);
        for (std::int64_t p = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
             p < pairs; p += stride) {
            double2 ca = Ca2[p], ip3 = IP32[p], hh = h2[p];
            const std::int64_t i = 2 * p;
            advance_cell<kUniform, kInput, kNoise>(a, s, i, step, ca.x, ip3.x, hh.x);
            advance_cell<kUniform, kInput, kNoise>(a, s, i + 1, step, ca.y, ip3.y, hh.y);
            Ca2[p] = ca;
            IP32[p] = ip3;
            h2[p] = hh;
            if (kInput == kInputArrayZero)
                reinterpret_cast<double2*>(s.input)[p] = make_double2(0.0, 0.0);
        }
        // Odd tail cell.
        if ((a.n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
            const std::int64_t i = a.n - 1;
            double ca = s.Ca[i], ip3 = s.IP3[i], hh = s.h[i];
            advance_cell<kUniform, kInput, kNoise>(a, s, i, step, ca, ip3, hh);
            s.Ca[i] = ca;
            s.IP3[i] = ip3;
            s.h[i] = hh;
            if (kInput == kInputArrayZero) s.input[i] = 0.0;
        }
    } else {
        for (std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
             i < a.n; i += stride) {
            double ca = s.Ca[i], ip3 = s.IP3[i], hh = s.h[i];
            advance_cell<kUniform, kInput, kNoise>(a, s, i, step, ca, ip3, hh);
            s.Ca[i] = ca;
            s.IP3[i] = ip3;
            s.h[i] = hh;
            if (kInput == kInputArrayZero) s.input[i] = 0.0;
        }
    }
}

// Launch shapes the autotuner chooses between (cells/thread, block, blocks/SM
// the register budget allows).
struct Shape {
    int cells, block, min_blocks;
};
constexpr Shape kShapes[] = {{2, 128, 4}, {1, 128, 8}, {1, 256, 4}, {2, 128, 6}, {1, 128, 6},
                             {1, 64, 12}, {4, 64, 8}, {4, 128, 4}, {2, 128, 5}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

template <bool kUniform, int kInput, bool kNoise>
cudaError_t launch_astro(int shape, int sms, StepArgs a, AstroArrays s, cudaStream_t st) {
    // Independent noise (log and cos per cell) is compiled for one shape: one
    // cell per thread, 128 threads, 6 blocks per SM (85 registers, no spills).
    if (kNoise) shape = 4;
    const Shape sh = kShapes[shape];
    const std::int64_t units = std::max<std::int64_t>(1, a.n / sh.cells);
    const std::int64_t want = (units + sh.block - 1) / sh.block;
    const std::int64_t cap = static_cast<std::int64_t>(sms) * sh.min_blocks * 4;
    const int grid = static_cast<int>(std::max<std::int64_t>(1, std::min(want, cap)));
    if constexpr (kNoise) {
        astro_step_kernel<kUniform, kInput, kNoise, 1, 128, 6><<<grid, 128, 0, st>>>(a, s);
    } else {
        switch (shape) {
            case 0: astro_step_kernel<kUniform, kInput, kNoise, 2, 128, 4><<<grid, 128, 0, st>>>(a, s); break;
            case 1: astro_step_kernel<kUniform, kInput, kNoise, 1, 128, 8><<<grid, 128, 0, st>>>(a, s); break;
            case 2: astro_step_kernel<kUniform, kInput, kNoise, 1, 256, 4><<<grid, 256, 0, st>>>(a, s); break;
            case 3: astro_step_kernel<kUniform, kInput, kNoise, 2, 128, 6><<<grid, 128, 0, st>>>(a, s); break;
            case 4: astro_step_kernel<kUniform, kInput, kNoise, 1, 128, 6><<<grid, 128, 0, st>>>(a, s); break;
            case 5: astro_step_kernel<kUniform, kInput, kNoise, 1, 64, 12><<<grid, 64, 0, st>>>(a, s); break;
            case 6: astro_step_kernel<kUniform, kInput, kNoise, 4, 64, 8><<<grid, 64, 0, st>>>(a, s); break;
            case 7: astro_step_kernel<kUniform, kInput, kNoise, 4, 128, 4><<<grid, 128, 0, st>>>(a, s); break;
            default: astro_step_kernel<kUniform, kInput, kNoise, 2, 128, 5><<<grid, 128, 0, st>>>(a, s); break;
        }
    }
    return cudaGetLastError();
}

// Precision study: the kernel-scaling workload in FP32 (astro_rk4_f32),
// four adjacent cells per thread with 128-bit float4 accesses; uniform
// parameters, Bernoulli input from the same counter RNG draws as the FP64
// kernel (the event test is exact, so both see the same events).
__global__ void __launch_bounds__(128, 8) astro_step_kernel_f32(StepArgs a, AstroKf kf, float* Ca,
                                                                float* IP3, float* h) {
    const std::int64_t step = *a.step_base + a.step_offset;
    const float ca_tot = static_cast<float>(a.u.Ca_tot), ip3_0 = static_cast<float>(a.u.IP3_0),
                tau = static_cast<float>(a.u.tau), delta = static_cast<float>(a.u.delta),
                weight = static_cast<float>(a.weight);
    const std::int64_t quads = (a.n + 3) / 4;
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t q = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
         q < quads; q += stride) {
        const std::int64_t i0 = 4 * q;
        const bool full = i0 + 4 <= a.n;
        float c[4], i3[4], hv[4];
        if (full) {
            const float4 C4 = reinterpret_cast<const float4*>(Ca)[q];
            const float4 I4 = reinterpret_cast<const float4*>(IP3)[q];
            const float4 H4 = reinterpret_cast<const float4*>(h)[q];
            c[0] = C4.x; c[1] = C4.y; c[2] = C4.z; c[3] = C4.w;
            i3[0] = I4.x; i3[1] = I4.y; i3[2] = I4.z; i3[3] = I4.w;
            hv[0] = H4.x; hv[1] = H4.y; hv[2] = H4.z; hv[3] = H4.w;
        } else {
            for (int j = 0; j < 4; ++j) {
                const bool in = i0 + j < a.n;
                c[j] = in ? Ca[i0 + j] : 0.0f;
                i3[j] = in ? IP3[i0 + j] : 0.0f;
                hv[j] = in ? h[i0 + j] : 0.0f;
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float in =
                (mix64(a.seed, static_cast<std::uint64_t>(i0 + j), 1000ULL +
                       static_cast<std::uint64_t>(step)) >> 11) < a.p_threshold ? weight : 0.0f;
            astro_rk4_f32(kf, ca_tot, ip3_0, tau, delta, in, 0.0f, c[j], i3[j], hv[j]);
        }
        if (full) {
            reinterpret_cast<float4*>(Ca)[q] = make_float4(c[0], c[1], c[2], c[3]);
            reinterpret_cast<float4*>(IP3)[q] = make_float4(i3[0], i3[1], i3[2], i3[3]);
            reinterpret_cast<float4*>(h)[q] = make_float4(hv[0], hv[1], hv[2], hv[3]);
        } else {
            for (int j = 0; j < 4 && i0 + j < a.n; ++j) {
                Ca[i0 + j] = c[j];
                IP3[i0 + j] = i3[j];
                h[i0 + j] = hv[j];
            }
        }
    }
}

// float <-> double copies of the study's state.
__global__ void narrow_kernel(std::int64_t n, const double* __restrict__ src,
                              float* __restrict__ dst) {
    for (std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::int64_t>(gridDim.x) * blockDim.x)
        dst[i] = static_cast<float>(src[i]);
}
__global__ void widen_kernel(std::int64_t n, const float* __restrict__ src,
                             double* __restrict__ dst) {
    for (std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<std::int64_t>(gridDim.x) * blockDim.x)
        dst[i] = src[i];
}

// The drop-in update's kernel for its parameter form, input and noise.
template <bool kUniform>
cudaError_t launch_update_p(bool pending, bool noisy, int shape, int sms, const StepArgs& a,
                            const AstroArrays& s, cudaStream_t st) {
    if (noisy)
        return pending ? launch_astro<kUniform, kInputArray, true>(shape, sms, a, s, st)
                       : launch_astro<kUniform, kInputNone, true>(shape, sms, a, s, st);
    return pending ? launch_astro<kUniform, kInputArray, false>(shape, sms, a, s, st)
                   : launch_astro<kUniform, kInputNone, false>(shape, sms, a, s, st);
}

cudaError_t launch_update(bool uniform, bool pending, bool noisy, int shape, int sms,
                          const StepArgs& a, const AstroArrays& s, cudaStream_t st) {
    return uniform ? launch_update_p<true>(pending, noisy, shape, sms, a, s, st)
                   : launch_update_p<false>(pending, noisy, shape, sms, a, s, st);
}

__global__ void advance_counter_kernel(std::int64_t* base, std::int64_t by) { *base += by; }

// ceil(p * 2^53): k * 2^-53 < p exactly when the integer k is below it
// (p * 2^53 is exact, and an integer is below a real number exactly when it
// is below its ceiling).  p <= 0 or NaN gives no events, p >= 1 every one.
std::uint64_t bernoulli_threshold(double p) {
    if (!(p > 0.0)) return 0;
    if (p >= 1.0) return 1ull << 53;
    return static_cast<std::uint64_t>(std::ceil(std::ldexp(p, 53)));
}

// Divisors taken through host-rounded reciprocals (div_by) must have a
// magnitude in [2^-46, 2^63], the range where that division is exact.
bool divisor_ok(double b) {
    const double m = std::fabs(b);
    return m >= 0x1p-46 && m <= 0x1p63;
}

AstroK make_astro_k(const double* c, double h_step, int substeps) {
    // c: Kd_IP3_1, Kd_IP3_2, Kd_act, Kd_inh, Km_SERCA, k_IP3R, rate_IP3R,
    //    rate_L, rate_SERCA, ratio_ER_cyt
    AstroK k{};
    k.Kd_IP3_1 = c[0];
    k.Kd_IP3_2 = c[1];
    k.Kd_act = c[2];
    k.ratio_ER_cyt = c[9];
    k.inv_ratio = 1.0 / c[9];
    k.chan = c[9] * c[6];
    k.serca = c[8];
    k.km2 = c[4] * c[4];
    k.leak = c[9] * c[7];
    k.ah = c[5] * c[3];
    k.k_IP3R = c[5];
    k.half_h = 0.5 * h_step;
    k.h = h_step;
    k.h6 = h_step / 6.0;
    k.substeps = substeps;
    return k;
}

}  // namespace

struct AstroEngine {
    std::int64_t n = 0;
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DevBuf Ca, IP3, h, input, Ca_tot, IP3_0, tau, inv_tau, delta, step_base;
    // Precision study: the state rounded to float, valid while no FP64 call
    // has advanced the FP64 state since (f32_valid).
    DevBuf Ca32, IP332, h32;
    bool f32_valid = false;
    double last_ms = 0.0;
    std::int64_t last_kernels = 0;
    int shape = 0;  // launch shape (see kShapes), set by asg_astro_autotune
    // Per-cell parameters given at create.  When every cell has the same four
    // values (bit for bit) they are kept as scalars and no array is read.
    bool has_params = false;
    bool params_uniform = false;
    UniformParams up{};
    // A push since the last update: the update reads the input array.  With
    // none, the input is zero (the reference kernel zeroes it after use) and
    // is not read; the engine never writes it, since each push overwrites
    // the whole array.
    bool input_pending = false;
    // Device time of consecutive asg_astro_update calls: ev0 is recorded by
    // the first update after the last timing read, ev1 by every update.
    bool upd_armed = false;
    std::int64_t upd_calls = 0;
    // Captured chunk of Bernoulli steps, rebuilt when its arguments change.
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    int graph_shape = -1;
    StepArgs graph_args{};
    bool graph_uniform = true;

    ~AstroEngine() {
        join_copies();
        if (graph) cudaGraphExecDestroy(graph);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (int c = 0; c < kMaxPieces; ++c) {
            if (ev_in[c]) cudaEventDestroy(ev_in[c]);
            if (ev_k[c]) cudaEventDestroy(ev_k[c]);
            if (ev_out[c]) cudaEventDestroy(ev_out[c]);
        }
        if (h2d) cudaStreamDestroy(h2d);
        if (d2h) cudaStreamDestroy(d2h);
        if (stream) cudaStreamDestroy(stream);
    }

    int grid_for(std::int64_t pairs, int block) const {
        const std::int64_t want = (pairs + block - 1) / block;
        const std::int64_t cap = static_cast<std::int64_t>(sms) * 16;
        return static_cast<int>(std::max<std::int64_t>(1, std::min(want, cap)));
    }

    AstroArrays arrays() {
        return AstroArrays{Ca.as<double>(),     IP3.as<double>(),    h.as<double>(),
                           input.as<double>(),  Ca_tot.as<double>(), IP3_0.as<double>(),
                           tau.as<double>(),    inv_tau.as<double>(), delta.as<double>()};
    }
    // The same arrays from cell `off` on (per-cell parameters when present).
    AstroArrays arrays_at(std::int64_t off) {
        auto at = [off](DevBuf& b) { return b.get() ? b.as<double>() + off : nullptr; };
        return AstroArrays{at(Ca), at(IP3), at(h), at(input), at(Ca_tot), at(IP3_0), at(tau),
                           at(inv_tau), at(delta)};
    }

    // Drop-in copies and updates run as a pipeline over `pieces()` cell
    // ranges: the input copy of range c+1 (host->device engine), the update
    // of range c and the Ca copy of range c-1 (device->host engine) overlap.
    // Events keep each range's order: input copy -> update -> Ca copy, and
    // the next step's input copy and update after this step's update and Ca
    // copy of the same range.
    static constexpr int kMaxPieces = 8;
    static constexpr std::int64_t kPieceCells = 1 << 18;
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t ev_in[kMaxPieces] = {}, ev_k[kMaxPieces] = {}, ev_out[kMaxPieces] = {};
    int pieces() const {
        return static_cast<int>(std::max<std::int64_t>(
            1, std::min<std::int64_t>(kMaxPieces, n / kPieceCells)));
    }
    // [begin, end) of range c: multiples of 64 cells (512-byte aligned).
    std::int64_t piece_begin(int c) const {
        return c == 0 ? 0 : ((n * c / pieces()) & ~static_cast<std::int64_t>(63));
    }
    std::int64_t piece_end(int c) const { return c + 1 == pieces() ? n : piece_begin(c + 1); }
    // Later work on `stream` (state pulls, other updates) after every copy.
    cudaError_t join_copies() {
        cudaError_t e = cudaSuccess;
        if (h2d) e = cudaStreamSynchronize(h2d);
        if (e == cudaSuccess && d2h) e = cudaStreamSynchronize(d2h);
        return e;
    }
};

}  // namespace asg

using asg::AstroEngine;

extern "C" {

int asg_astro_create(uint32_t n, const double* Ca, const double* IP3, const double* h,
                     const double* Ca_tot, const double* IP3_0, const double* tau_IP3,
                     const double* delta_IP3, asg_astro** out) {
    asg::clear_error();
    if (out == nullptr) return asg::fail(ASG_ERR_ARG, "asg_astro_create: out is NULL");
    *out = nullptr;
    if (n > 0 && (Ca == nullptr || IP3 == nullptr || h == nullptr))
        return asg::fail(ASG_ERR_ARG, "asg_astro_create: state arrays are required");
    // The per-cell parameters come as a set (the reference's cuda_astro_create
    // takes all four): a partial set would leave the update reading a missing
    // array.
    const int n_params = (Ca_tot != nullptr) + (IP3_0 != nullptr) + (tau_IP3 != nullptr) +
                         (delta_IP3 != nullptr);
    if (n_params != 0 && n_params != 4)
        return asg::fail(ASG_ERR_ARG,
                         "asg_astro_create: give all four per-cell parameter arrays (Ca_tot, "
                         "IP3_0, tau_IP3, delta_IP3) or none; %d of 4 given",
                         n_params);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return asg::fail(ASG_ERR_NO_DEVICE, "asg_astro_create: no CUDA device");
    auto* e = new AstroEngine;
    e->n = n;
    cudaGetDevice(&e->device);
    cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, e->device);
    const std::size_t bytes = static_cast<std::size_t>(n) * sizeof(double);
    int st = ASG_OK;
    // Parameter arrays are optional (the scaling run takes uniform scalars);
    // a NULL parameter array allocates nothing.
    auto upload = [&](asg::DevBuf& b, const double* src, bool required) {
        if (st != ASG_OK || (src == nullptr && !required)) return;
        st = b.alloc(bytes, src == nullptr);
        if (st == ASG_OK && src != nullptr && bytes > 0) {
            const cudaError_t ce = cudaMemcpy(b.get(), src, bytes, cudaMemcpyHostToDevice);
            if (ce != cudaSuccess) st = asg::cuda_fail(ce, "upload", __FILE__, __LINE__);
        }
    };
    upload(e->Ca, Ca, true);
    upload(e->IP3, IP3, true);
    upload(e->h, h, true);
    upload(e->input, nullptr, true);
    e->has_params = n_params == 4;
    if (e->has_params && n > 0) {
        auto same = [n](const double* v) {
            for (uint32_t i = 1; i < n; ++i)
                if (std::memcmp(&v[i], &v[0], sizeof(double)) != 0) return false;
            return true;
        };
        e->params_uniform = same(Ca_tot) && same(IP3_0) && same(tau_IP3) && same(delta_IP3);
        if (e->params_uniform) {
            if (!asg::divisor_ok(tau_IP3[0]) || !asg::diff_param_ok(Ca_tot[0]) ||
                !asg::diff_param_ok(IP3_0[0]))
                st = asg::fail(ASG_ERR_UNSUPPORTED,
                               "asg_astro_create: tau_IP3 outside [2^-46, 2^63] or Ca_tot / IP3_0 "
                               "outside [2^-906, 2^976] in magnitude");
            e->up = asg::UniformParams{Ca_tot[0], IP3_0[0], tau_IP3[0], delta_IP3[0],
                                       1.0 / tau_IP3[0]};
            Ca_tot = IP3_0 = tau_IP3 = delta_IP3 = nullptr;  // nothing per cell to upload
        }
    }
    upload(e->Ca_tot, Ca_tot, false);
    upload(e->IP3_0, IP3_0, false);
    upload(e->tau, tau_IP3, false);
    if (tau_IP3 != nullptr) {
        std::vector<double> inv(n);
        for (uint32_t i = 0; i < n && st == ASG_OK; ++i) {
            if (!asg::divisor_ok(tau_IP3[i]))
                st = asg::fail(ASG_ERR_UNSUPPORTED,
                               "asg_astro_create: tau_IP3[%u] = %g outside [2^-46, 2^63]", i,
                               tau_IP3[i]);
            else if (!asg::diff_param_ok(Ca_tot[i]) || !asg::diff_param_ok(IP3_0[i]))
                st = asg::fail(ASG_ERR_UNSUPPORTED,
                               "asg_astro_create: Ca_tot[%u] or IP3_0[%u] has a magnitude outside "
                               "[2^-906, 2^976]", i, i);
            inv[i] = 1.0 / tau_IP3[i];
        }
        upload(e->inv_tau, inv.data(), false);
    }
    upload(e->delta, delta_IP3, false);
    if (st == ASG_OK) st = e->step_base.alloc(sizeof(std::int64_t));
    if (st == ASG_OK) {
        cudaError_t ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
        if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->h2d, cudaStreamNonBlocking);
        if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->d2h, cudaStreamNonBlocking);
        if (ce == cudaSuccess) ce = cudaEventCreate(&e->ev0);
        if (ce == cudaSuccess) ce = cudaEventCreate(&e->ev1);
        for (int c = 0; c < AstroEngine::kMaxPieces && ce == cudaSuccess; ++c) {
            ce = cudaEventCreateWithFlags(&e->ev_in[c], cudaEventDisableTiming);
            if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->ev_k[c], cudaEventDisableTiming);
            if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->ev_out[c], cudaEventDisableTiming);
        }
        if (ce != cudaSuccess) st = asg::cuda_fail(ce, "stream/event", __FILE__, __LINE__);
    }
    if (st != ASG_OK) {
        delete e;
        return st;
    }
    *out = reinterpret_cast<asg_astro*>(e);
    return ASG_OK;
}

int asg_astro_destroy(asg_astro* s, double* Ca, double* IP3, double* h) {
    asg::clear_error();
    if (s == nullptr) return ASG_OK;
    auto* e = reinterpret_cast<AstroEngine*>(s);
    int st = ASG_OK;
    if (e->n > 0 && Ca != nullptr && IP3 != nullptr && h != nullptr) {
        st = asg_astro_pull_state(s, Ca, IP3, h);
    }
    delete e;
    return st;
}

int asg_astro_pull_state(asg_astro* s, double* Ca, double* IP3, double* h) {
    asg::clear_error();
    if (s == nullptr) return asg::fail(ASG_ERR_ARG, "asg_astro_pull_state: NULL handle");
    auto* e = reinterpret_cast<AstroEngine*>(s);
    const std::size_t bytes = static_cast<std::size_t>(e->n) * sizeof(double);
    if (bytes == 0) return ASG_OK;
    ASG_CUDA(e->join_copies());
    ASG_CUDA(cudaMemcpyAsync(Ca, e->Ca.get(), bytes, cudaMemcpyDeviceToHost, e->stream));
    ASG_CUDA(cudaMemcpyAsync(IP3, e->IP3.get(), bytes, cudaMemcpyDeviceToHost, e->stream));
    ASG_CUDA(cudaMemcpyAsync(h, e->h.get(), bytes, cudaMemcpyDeviceToHost, e->stream));
    ASG_CUDA(cudaStreamSynchronize(e->stream));
    return ASG_OK;
}

int asg_astro_push_input(asg_astro* s, const double* ip3_input) {
    asg::NvtxRange nvtx("astrocyte input push (host to device)");
    asg::clear_error();
    if (s == nullptr || ip3_input == nullptr)
        return asg::fail(ASG_ERR_ARG, "asg_astro_push_input: NULL argument");
    auto* e = reinterpret_cast<AstroEngine*>(s);
    if (e->n == 0) return ASG_OK;
    for (int c = 0; c < e->pieces(); ++c) {
        const std::int64_t b = e->piece_begin(c), n = e->piece_end(c) - b;
        // after the previous update consumed (zeroed) this range's input
        ASG_CUDA(cudaStreamWaitEvent(e->h2d, e->ev_k[c], 0));
        ASG_CUDA(cudaMemcpyAsync(e->input.as<double>() + b, ip3_input + b,
                                 static_cast<std::size_t>(n) * sizeof(double),
                                 cudaMemcpyHostToDevice, e->h2d));
        ASG_CUDA(cudaEventRecord(e->ev_in[c], e->h2d));
    }
    e->input_pending = true;
    return ASG_OK;
}

int asg_astro_pull_calcium(asg_astro* s, double* Ca) {
    asg::NvtxRange nvtx("astrocyte calcium pull (device to host)");
    asg::clear_error();
    if (s == nullptr || Ca == nullptr)
        return asg::fail(ASG_ERR_ARG, "asg_astro_pull_calcium: NULL argument");
    auto* e = reinterpret_cast<AstroEngine*>(s);
    if (e->n == 0) return ASG_OK;
    for (int c = 0; c < e->pieces(); ++c) {
        const std::int64_t b = e->piece_begin(c), n = e->piece_end(c) - b;
        ASG_CUDA(cudaStreamWaitEvent(e->d2h, e->ev_k[c], 0));  // after this range's update
        ASG_CUDA(cudaMemcpyAsync(Ca + b, e->Ca.as<double>() + b,
                                 static_cast<std::size_t>(n) * sizeof(double),
                                 cudaMemcpyDeviceToHost, e->d2h));
        ASG_CUDA(cudaEventRecord(e->ev_out[c], e->d2h));
    }
    ASG_CUDA(cudaStreamSynchronize(e->d2h));
    return ASG_OK;
}

int asg_astro_update(asg_astro* s, const double* consts, double h_step, int32_t substeps,
                     double noise_std, int32_t independent_noise, double shared_noise,
                     uint64_t noise_seed, uint64_t noise_index) {
    asg::NvtxRange nvtx("update astrocytes");
    asg::clear_error();
    if (s == nullptr || consts == nullptr)
        return asg::fail(ASG_ERR_ARG, "asg_astro_update: NULL argument");
    if (substeps < 0) return asg::fail(ASG_ERR_ARG, "asg_astro_update: substeps < 0");
    if (!asg::divisor_ok(consts[9]))
        return asg::fail(ASG_ERR_UNSUPPORTED, "asg_astro_update: ratio_ER_cyt = %g outside "
                         "[2^-46, 2^63]", consts[9]);
    auto* e = reinterpret_cast<AstroEngine*>(s);
    if (e->n == 0) return ASG_OK;
    if (!e->has_params) {
        return asg::fail(ASG_ERR_STATE,
                         "asg_astro_update: per-cell parameters were not given at create");
    }
    asg::StepArgs a{};
    a.n = e->n;
    a.k = asg::make_astro_k(consts, h_step, substeps);
    a.u = e->up;
    a.noise_std = noise_std;
    a.independent = independent_noise;
    a.shared_noise = shared_noise;
    a.noise_seed = noise_seed;
    a.noise_index = noise_index;
    a.step_base = e->step_base.as<std::int64_t>();
    if (!e->upd_armed) {
        ASG_CUDA(cudaEventRecord(e->ev0, e->stream));
        e->upd_armed = true;
        e->upd_calls = 0;
    }
    // The reference applies noise only when noise_std > 0 (astrocyte.cpp:
    // 313-322); otherwise the caller's shared value (0) enters the RHS.
    if (!(noise_std > 0.0)) a.independent = 0;
    const bool pending = e->input_pending;
    if (!pending) {
        // No input copy to overlap: one launch over every cell, after the
        // last calcium copies of every range have read the state.
        for (int c = 0; c < e->pieces(); ++c)
            ASG_CUDA(cudaStreamWaitEvent(e->stream, e->ev_out[c], 0));
        a.n = e->n;
        a.i0 = 0;
        ASG_CUDA(asg::launch_update(e->params_uniform, false, a.independent != 0, e->shape,
                                    e->sms, a, e->arrays(), e->stream));
        for (int c = 0; c < e->pieces(); ++c)
            ASG_CUDA(cudaEventRecord(e->ev_k[c], e->stream));
        e->upd_calls += 1;
    } else {
        for (int c = 0; c < e->pieces(); ++c) {
            const std::int64_t b = e->piece_begin(c);
            ASG_CUDA(cudaStreamWaitEvent(e->stream, e->ev_in[c], 0));   // this range's input
            ASG_CUDA(cudaStreamWaitEvent(e->stream, e->ev_out[c], 0));  // last Ca copy read it
            a.n = e->piece_end(c) - b;
            a.i0 = b;
            ASG_CUDA(asg::launch_update(e->params_uniform, true, a.independent != 0, e->shape,
                                        e->sms, a, e->arrays_at(b), e->stream));
            ASG_CUDA(cudaEventRecord(e->ev_k[c], e->stream));
        }
        e->upd_calls += e->pieces();
    }
    e->input_pending = false;
    e->f32_valid = false;
    ASG_CUDA(cudaEventRecord(e->ev1, e->stream));
    return ASG_OK;
}

int asg_astro_run_bernoulli(asg_astro* s, const double* consts, double h_step, int32_t substeps,
                            uint64_t seed, double p, double weight, int64_t first, int64_t count,
                            int32_t uniform, double Ca_tot, double IP3_0, double tau_IP3,
                            double delta_IP3) {
    asg::NvtxRange nvtx("update astrocytes (kernel-scaling workload)");
    asg::clear_error();
    if (s == nullptr || consts == nullptr)
        return asg::fail(ASG_ERR_ARG, "asg_astro_run_bernoulli: NULL argument");
    if (count < 0 || first < 0 || substeps < 0)
        return asg::fail(ASG_ERR_ARG, "asg_astro_run_bernoulli: negative step range");
    if (!asg::divisor_ok(consts[9]) ||
        (uniform && (!asg::divisor_ok(tau_IP3) || !asg::diff_param_ok(Ca_tot) ||
                     !asg::diff_param_ok(IP3_0))))
        return asg::fail(ASG_ERR_UNSUPPORTED, "asg_astro_run_bernoulli: ratio_ER_cyt or tau_IP3 "
                         "outside [2^-46, 2^63], or Ca_tot / IP3_0 outside [2^-906, 2^976]");
    auto* e = reinterpret_cast<AstroEngine*>(s);
    if (!uniform && !e->has_params)
        return asg::fail(ASG_ERR_STATE, "asg_astro_run_bernoulli: no per-cell parameters");
    e->upd_armed = false;
    e->f32_valid = false;
    // Per-cell parameters that are all equal run as the scalars they are.
    if (!uniform && e->params_uniform) {
        uniform = 1;
        Ca_tot = e->up.Ca_tot;
        IP3_0 = e->up.IP3_0;
        tau_IP3 = e->up.tau;
        delta_IP3 = e->up.delta;
    }
    if (e->n == 0 || count == 0) {
        e->last_ms = 0.0;
        e->last_kernels = 0;
        return ASG_OK;
    }
    ASG_CUDA(e->join_copies());
    asg::StepArgs a;
    std::memset(&a, 0, sizeof a);
    a.n = e->n;
    a.k = asg::make_astro_k(consts, h_step, substeps);
    a.u = asg::UniformParams{Ca_tot, IP3_0, tau_IP3, delta_IP3, 1.0 / tau_IP3};
    a.seed = seed;
    a.p = p;
    a.p_threshold = asg::bernoulli_threshold(p);
    a.weight = weight;
    a.step_base = e->step_base.as<std::int64_t>();

    // Steps run as captured chunks of up to 64 launches: kernel j of a chunk
    // reads step = *step_base + j, and a one-thread node advances the base.
    const int chunk = static_cast<int>(std::min<std::int64_t>(64, count));
    cudaError_t launch_err = cudaSuccess;
    auto launch_step = [&](int j) {
        asg::StepArgs aj = a;
        aj.step_offset = j;
        const cudaError_t le =
            uniform ? asg::launch_astro<true, asg::kInputBernoulli, false>(e->shape, e->sms, aj,
                                                                            e->arrays(), e->stream)
                    : asg::launch_astro<false, asg::kInputBernoulli, false>(e->shape, e->sms, aj,
                                                                             e->arrays(), e->stream);
        if (le != cudaSuccess) launch_err = le;
    };
    const bool same = e->graph != nullptr && e->graph_steps == chunk &&
                      e->graph_uniform == (uniform != 0) && e->graph_shape == e->shape &&
                      std::memcmp(&e->graph_args, &a, sizeof a) == 0;
    if (!same) {
        if (e->graph) cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
        cudaGraph_t g = nullptr;
        ASG_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        for (int j = 0; j < chunk; ++j) launch_step(j);
        ASG_CUDA(launch_err);
        asg::advance_counter_kernel<<<1, 1, 0, e->stream>>>(e->step_base.as<std::int64_t>(), chunk);
        ASG_CUDA(cudaStreamEndCapture(e->stream, &g));
        const cudaError_t ce = cudaGraphInstantiate(&e->graph, g, 0);
        cudaGraphDestroy(g);
        ASG_CUDA(ce);
        e->graph_steps = chunk;
        e->graph_args = a;
        e->graph_uniform = uniform != 0;
        e->graph_shape = e->shape;
    }
    std::int64_t base = first;
    ASG_CUDA(cudaMemcpyAsync(e->step_base.get(), &base, sizeof base, cudaMemcpyHostToDevice, e->stream));
    ASG_CUDA(cudaStreamSynchronize(e->stream));
    ASG_CUDA(cudaEventRecord(e->ev0, e->stream));
    std::int64_t done = 0;
    std::int64_t kernels = 0;
    while (count - done >= chunk) {
        ASG_CUDA(cudaGraphLaunch(e->graph, e->stream));
        done += chunk;
        kernels += chunk + 1;
    }
    if (done < count) {
        // Remainder: plain launches with the base already advanced.
        for (int j = 0; done + j < count; ++j) launch_step(j);
        ASG_CUDA(launch_err);
        kernels += count - done;
    }
    ASG_CUDA(cudaEventRecord(e->ev1, e->stream));
    ASG_CUDA(cudaEventSynchronize(e->ev1));
    float ms = 0.0f;
    ASG_CUDA(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
    e->last_ms = ms;
    e->last_kernels = kernels;
    return ASG_OK;
}

int asg_astro_last_timing(asg_astro* s, double* device_ms, int64_t* kernels) {
    asg::clear_error();
    if (s == nullptr) return asg::fail(ASG_ERR_ARG, "asg_astro_last_timing: NULL handle");
    auto* e = reinterpret_cast<AstroEngine*>(s);
    if (e->upd_armed) {
        // updates since the last read: ev0 of the first .. ev1 of the last
        ASG_CUDA(cudaEventSynchronize(e->ev1));
        float ms = 0.0f;
        ASG_CUDA(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
        e->last_ms = ms;
        e->last_kernels = e->upd_calls;
        e->upd_armed = false;
    }
    if (device_ms) *device_ms = e->last_ms;
    if (kernels) *kernels = e->last_kernels;
    return ASG_OK;
}

int asg_astro_run_bernoulli_f32(asg_astro* s, const double* consts, double h_step,
                                int32_t substeps, uint64_t seed, double p, double weight,
                                int64_t first, int64_t count, double Ca_tot, double IP3_0,
                                double tau_IP3, double delta_IP3) {
    asg::NvtxRange nvtx("update astrocytes in FP32 (precision study)");
    asg::clear_error();
    if (s == nullptr || consts == nullptr)
        return asg::fail(ASG_ERR_ARG, "asg_astro_run_bernoulli_f32: NULL argument");
    if (count < 0 || first < 0 || substeps < 0)
        return asg::fail(ASG_ERR_ARG, "asg_astro_run_bernoulli_f32: negative step range");
    auto* e = reinterpret_cast<AstroEngine*>(s);
    if (e->n == 0 || count == 0) {
        e->last_ms = 0.0;
        e->last_kernels = 0;
        return ASG_OK;
    }
    ASG_CUDA(e->join_copies());
    e->upd_armed = false;
    const std::size_t fbytes = static_cast<std::size_t>(e->n) * sizeof(float);
    const int cgrid = e->sms * 8;
    if (e->Ca32.get() == nullptr) {
        ASG_TRY(e->Ca32.alloc(fbytes, false));
        ASG_TRY(e->IP332.alloc(fbytes, false));
        ASG_TRY(e->h32.alloc(fbytes, false));
    }
    if (!e->f32_valid) {
        asg::narrow_kernel<<<cgrid, 256, 0, e->stream>>>(e->n, e->Ca.as<double>(), e->Ca32.as<float>());
        asg::narrow_kernel<<<cgrid, 256, 0, e->stream>>>(e->n, e->IP3.as<double>(), e->IP332.as<float>());
        asg::narrow_kernel<<<cgrid, 256, 0, e->stream>>>(e->n, e->h.as<double>(), e->h32.as<float>());
        ASG_CUDA(cudaGetLastError());
    }
    asg::StepArgs a;
    std::memset(&a, 0, sizeof a);
    a.n = e->n;
    a.k = asg::make_astro_k(consts, h_step, substeps);
    a.u = asg::UniformParams{Ca_tot, IP3_0, tau_IP3, delta_IP3, 1.0 / tau_IP3};
    a.seed = seed;
    a.p = p;
    a.p_threshold = asg::bernoulli_threshold(p);
    a.weight = weight;
    a.step_base = e->step_base.as<std::int64_t>();
    const asg::AstroKf kf = asg::astro_k_f32(a.k);
    const std::int64_t quads = (e->n + 3) / 4;
    const int grid = static_cast<int>(std::max<std::int64_t>(
        1, std::min<std::int64_t>((quads + 127) / 128, static_cast<std::int64_t>(e->sms) * 8 * 4)));
    std::int64_t base = first;
    ASG_CUDA(cudaMemcpyAsync(e->step_base.get(), &base, sizeof base, cudaMemcpyHostToDevice,
                             e->stream));
    // Plain launches of 64-step groups, the step read from the device
    // counter; the counter advances by a one-thread kernel after each group.
    ASG_CUDA(cudaEventRecord(e->ev0, e->stream));
    std::int64_t done = 0, kernels = 0;
    while (done < count) {
        const int chunk = static_cast<int>(std::min<std::int64_t>(64, count - done));
        for (int j = 0; j < chunk; ++j) {
            a.step_offset = j;
            asg::astro_step_kernel_f32<<<grid, 128, 0, e->stream>>>(
                a, kf, e->Ca32.as<float>(), e->IP332.as<float>(), e->h32.as<float>());
        }
        asg::advance_counter_kernel<<<1, 1, 0, e->stream>>>(e->step_base.as<std::int64_t>(), chunk);
        ASG_CUDA(cudaGetLastError());
        done += chunk;
        kernels += chunk + 1;
    }
    ASG_CUDA(cudaEventRecord(e->ev1, e->stream));
    // The FP64 state holds the widened result, for pulls and FP64 calls.
    asg::widen_kernel<<<cgrid, 256, 0, e->stream>>>(e->n, e->Ca32.as<float>(), e->Ca.as<double>());
    asg::widen_kernel<<<cgrid, 256, 0, e->stream>>>(e->n, e->IP332.as<float>(), e->IP3.as<double>());
    asg::widen_kernel<<<cgrid, 256, 0, e->stream>>>(e->n, e->h32.as<float>(), e->h.as<double>());
    ASG_CUDA(cudaGetLastError());
    ASG_CUDA(cudaStreamSynchronize(e->stream));
    e->f32_valid = true;
    float ms = 0.0f;
    ASG_CUDA(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
    e->last_ms = ms;
    e->last_kernels = kernels;
    return ASG_OK;
}

}  // extern "C"

extern "C" int asg_astro_set_shape(asg_astro* s, int32_t shape) {
    asg::clear_error();
    if (s == nullptr) return asg::fail(ASG_ERR_ARG, "asg_astro_set_shape: NULL handle");
    if (shape < 0 || shape >= asg::kNumShapes)
        return asg::fail(ASG_ERR_ARG, "asg_astro_set_shape: shape %d not in [0, %d)", shape,
                         asg::kNumShapes);
    reinterpret_cast<AstroEngine*>(s)->shape = shape;
    return ASG_OK;
}

extern "C" int asg_astro_autotune(asg_astro* s, const double* consts, double h_step,
                                  int32_t substeps, int32_t steps, int32_t* chosen,
                                  double* us_per_step) {
    asg::clear_error();
    if (s == nullptr || consts == nullptr || steps <= 0)
        return asg::fail(ASG_ERR_ARG, "asg_astro_autotune: bad arguments");
    auto* e = reinterpret_cast<AstroEngine*>(s);
    if (e->n == 0) return ASG_OK;
    const std::size_t bytes = static_cast<std::size_t>(e->n) * sizeof(double);
    ASG_CUDA(e->join_copies());
    // Scratch copies of the state: the trials advance these, not the handle's.
    asg::DevBuf ca, ip3, h;
    ASG_TRY(ca.alloc(bytes, false));
    ASG_TRY(ip3.alloc(bytes, false));
    ASG_TRY(h.alloc(bytes, false));
    ASG_CUDA(cudaMemcpyAsync(ca.get(), e->Ca.get(), bytes, cudaMemcpyDeviceToDevice, e->stream));
    ASG_CUDA(cudaMemcpyAsync(ip3.get(), e->IP3.get(), bytes, cudaMemcpyDeviceToDevice, e->stream));
    ASG_CUDA(cudaMemcpyAsync(h.get(), e->h.get(), bytes, cudaMemcpyDeviceToDevice, e->stream));
    asg::AstroArrays arr = e->arrays();
    arr.Ca = ca.as<double>();
    arr.IP3 = ip3.as<double>();
    arr.h = h.as<double>();
    asg::StepArgs a;
    std::memset(&a, 0, sizeof a);
    a.n = e->n;
    a.k = asg::make_astro_k(consts, h_step, substeps);
    a.u = asg::UniformParams{1.8958264782990153, 0.010925583871830699, 1058.7589568400845,
                             0.04911592657233997, 1.0 / 1058.7589568400845};
    a.seed = 1;
    a.p = 0.01;
    a.p_threshold = asg::bernoulli_threshold(a.p);
    a.weight = 0.2;
    a.step_base = e->step_base.as<std::int64_t>();
    int best = e->shape;
    float best_ms = 1e30f;
    for (int shape = 0; shape < asg::kNumShapes; ++shape) {
        for (int rep = 0; rep < 2; ++rep) {  // first pass warms up
            ASG_CUDA(cudaEventRecord(e->ev0, e->stream));
            for (int j = 0; j < steps; ++j) {
                a.step_offset = j;
                ASG_CUDA((asg::launch_astro<true, asg::kInputBernoulli, false>(shape, e->sms, a,
                                                                                arr, e->stream)));
            }
            ASG_CUDA(cudaEventRecord(e->ev1, e->stream));
            ASG_CUDA(cudaEventSynchronize(e->ev1));
        }
        float ms = 0.0f;
        ASG_CUDA(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
        if (ms < best_ms) {
            best_ms = ms;
            best = shape;
        }
    }
    e->shape = best;
    if (chosen) *chosen = best;
    if (us_per_step) *us_per_step = 1e3 * best_ms / steps;
    return ASG_OK;
}

// ------------------------------------------------- allocation-free variant
//
// Some callers cannot call cudaMalloc: for example the reference's OpenMP
// target-offload build, whose device copies of Ca, IP3, h and the per-cell
// parameters are owned by the OpenMP runtime (`omp target enter data`) and
// reach us only as device pointers, or a host framework whose memory pool
// owns all device memory and forbids allocations of its own during a run.
// asg_astro_update_noalloc serves them: it updates caller-owned device arrays
// in place and allocates nothing.  Its only scratch -- the correctly rounded
// reciprocal of each cell's tau_IP3 that the division in the IP3 rate uses --
// lives in the file-scope array below.  The array is reserved with this
// file's device code: when the module is loaded, i.e. at context creation
// under eager module loading, or at the first call that needs the module
// (the address lookup below) under CUDA's default lazy loading.  From then
// on every GPU that uses the library holds it until the process exits.

namespace asg {
namespace {

constexpr std::uint32_t kNoAllocMaxCells = 1u << 20;  // 8 MiB of FP64 reciprocals
__device__ __align__(256) double g_noalloc_inv_tau[kNoAllocMaxCells];

constexpr int kNoAllocMaxDevices = 64;
struct ScratchAddr {
    unsigned long long ctx_id = 0;  // driver id of the context the address belongs to
    double* ptr = nullptr;
};
ScratchAddr g_noalloc_scratch[kNoAllocMaxDevices];  // per device ordinal
std::mutex g_noalloc_mu;

// inv_tau[i] = 1 / tau[i] (IEEE division: the correctly rounded reciprocal).
__global__ void noalloc_reciprocals(std::uint32_t n, const double* __restrict__ tau,
                                    double* __restrict__ inv_tau) {
    const std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) inv_tau[i] = 1.0 / tau[i];
}

// Unique id of the context current on this thread (0 when none is current),
// from the driver's cuCtxGetCurrent and cuCtxGetId, reached through the
// runtime's entry-point query so the library need not link libcuda.  Ids are
// never reused within a process, unlike context handles.
int current_context_id(unsigned long long* id) {
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    if (get_current == nullptr || get_id == nullptr) {
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1{}, q2{};
        ASG_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1));
        ASG_CUDA(cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2));
        if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
            return fail(ASG_ERR_UNSUPPORTED, "driver lacks cuCtxGetCurrent/cuCtxGetId");
        get_current = reinterpret_cast<GetCurrent>(f1);
        get_id = reinterpret_cast<GetId>(f2);
    }
    void* ctx = nullptr;
    *id = 0;
    if (get_current(&ctx) != 0) return fail(ASG_ERR_CUDA, "cuCtxGetCurrent failed");
    if (ctx != nullptr && get_id(ctx, id) != 0) return fail(ASG_ERR_CUDA, "cuCtxGetId failed");
    return ASG_OK;
}

// Device address of the scratch array in the current device's context.  In
// host code the array's name is only a host-side stand-in, so the address is
// looked up with cudaGetSymbolAddress, with the device current, once per
// device -- and again whenever the device's context is a new one (after
// cudaDeviceReset, or after a host framework released and re-created the
// primary context), because the cached address belongs to the old context.
int noalloc_scratch(int dev, double** out) {
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return fail(ASG_ERR_UNSUPPORTED, "device ordinal %d beyond %d", dev, kNoAllocMaxDevices);
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    ScratchAddr& e = g_noalloc_scratch[dev];
    unsigned long long ctx = 0;
    ASG_TRY(current_context_id(&ctx));
    if (e.ptr == nullptr || ctx == 0 || ctx != e.ctx_id) {
        void* p = nullptr;
        const cudaError_t ce = cudaGetSymbolAddress(&p, g_noalloc_inv_tau);
        if (ce == cudaErrorMemoryAllocation)
            return fail(ASG_ERR_OOM,
                        "asg_astro_update_noalloc: loading the module that holds the %u-cell "
                        "(8 MiB) scratch array failed: device memory is exhausted",
                        kNoAllocMaxCells);
        ASG_CUDA(ce);
        ASG_TRY(current_context_id(&ctx));  // the lookup made the context current
        e.ctx_id = ctx;
        e.ptr = static_cast<double*>(p);
    }
    *out = e.ptr;
    return ASG_OK;
}

}  // namespace
}  // namespace asg

extern "C" int asg_astro_update_noalloc(uint32_t n, double* Ca, double* IP3, double* h,
                                        double* ip3_input, const double* Ca_tot,
                                        const double* IP3_0, const double* tau_IP3,
                                        const double* delta_IP3, const double* consts,
                                        double h_step, int32_t substeps, double noise_std,
                                        int32_t independent_noise, double shared_noise,
                                        uint64_t noise_seed, uint64_t noise_index, void* stream) {
    asg::clear_error();
    if (n == 0) return ASG_OK;
    if (n > asg::kNoAllocMaxCells)
        return asg::fail(ASG_ERR_ARG,
                         "asg_astro_update_noalloc: %u cells exceed the %u-cell scratch limit; "
                         "use asg_astro_create/asg_astro_update for larger populations",
                         n, asg::kNoAllocMaxCells);
    if (Ca == nullptr || IP3 == nullptr || h == nullptr || ip3_input == nullptr ||
        Ca_tot == nullptr || IP3_0 == nullptr || tau_IP3 == nullptr || delta_IP3 == nullptr ||
        consts == nullptr)
        return asg::fail(ASG_ERR_ARG, "asg_astro_update_noalloc: NULL argument");
    if (substeps < 0) return asg::fail(ASG_ERR_ARG, "asg_astro_update_noalloc: substeps < 0");
    if (!asg::divisor_ok(consts[9]))
        return asg::fail(ASG_ERR_UNSUPPORTED, "asg_astro_update_noalloc: ratio_ER_cyt = %g "
                         "outside [2^-46, 2^63]", consts[9]);
    for (const void* p : {static_cast<const void*>(Ca), static_cast<const void*>(IP3),
                          static_cast<const void*>(h), static_cast<const void*>(ip3_input),
                          static_cast<const void*>(Ca_tot), static_cast<const void*>(IP3_0),
                          static_cast<const void*>(tau_IP3), static_cast<const void*>(delta_IP3)})
        if (reinterpret_cast<std::uintptr_t>(p) % alignof(double) != 0)
            return asg::fail(ASG_ERR_ARG, "asg_astro_update_noalloc: array not 8-byte aligned");
    // A launch error is read back with cudaGetLastError, which would also
    // return an error some earlier work left pending on this thread: refuse
    // to run on top of one rather than report it as this call's failure.
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess)
        return asg::fail(ASG_ERR_CUDA,
                         "asg_astro_update_noalloc: a CUDA error from earlier work is pending "
                         "on this thread (%s: %s); nothing was launched",
                         cudaGetErrorName(pending), cudaGetErrorString(pending));
    int dev = 0, sms = 148;
    ASG_CUDA(cudaGetDevice(&dev));
    ASG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    double* inv_tau = nullptr;
    ASG_TRY(asg::noalloc_scratch(dev, &inv_tau));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // Every entry this call reads is written first, in stream order, so the
    // previous call's contents never leak in.
    asg::noalloc_reciprocals<<<(n + 255) / 256, 256, 0, st>>>(n, tau_IP3, inv_tau);
    ASG_CUDA(cudaGetLastError());
    asg::StepArgs a;
    std::memset(&a, 0, sizeof a);
    a.n = n;
    a.k = asg::make_astro_k(consts, h_step, substeps);
    a.noise_std = noise_std;
    a.independent = noise_std > 0.0 ? independent_noise : 0;
    a.shared_noise = shared_noise;
    a.noise_seed = noise_seed;
    a.noise_index = noise_index;
    const asg::AstroArrays arr{Ca, IP3, h, ip3_input, Ca_tot, IP3_0, tau_IP3, inv_tau, delta_IP3};
    // Shape 1: one cell per thread with 8-byte accesses, so caller arrays need
    // no more than double alignment.
    ASG_CUDA(a.independent
                 ? (asg::launch_astro<false, asg::kInputArrayZero, true>(1, sms, a, arr, st))
                 : (asg::launch_astro<false, asg::kInputArrayZero, false>(1, sms, a, arr, st)));
    return ASG_OK;
}
