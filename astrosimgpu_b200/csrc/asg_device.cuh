// Device-side building blocks shared by every kernel of the engine:
//   - the counter-based RNG of the model (splitmix64 finaliser over
//     seed + stream*phi + counter*c, reference rng.hpp:26-50 and the
//     CounterRng methods rng.hpp:64-124),
//   - the Li-Rinzel astrocyte right-hand side and its RK4 advance
//     (reference astrocyte_kernel.hpp:47-103),
//   - the AdEx right-hand side (reference neuron.cpp:85-99).
//
// Bitwise parity with the host build is a design requirement, so every
// floating-point expression below evaluates the same IEEE operations in the
// same order as the reference's C++ (left to right, no contraction).  The
// translation units that include this header are compiled with
// -fmad=false so nvcc cannot fuse a multiply and an add.  Products of
// constants that the reference evaluates at run time (for example
// ratio_ER_cyt * rate_IP3R) are formed once on the host with the same
// rounding and passed in, which changes no bit of any result.
#pragma once

#include <cstdint>

namespace asg {

// ------------------------------------------------------------------ RNG

// Golden-ratio increment and the two splitmix64 multipliers (Steele, Lea &
// Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014).
constexpr std::uint64_t kPhi = 0x9E3779B97F4A7C15ULL;
constexpr std::uint64_t kMixA = 0xBF58476D1CE4E5B9ULL;
constexpr std::uint64_t kMixB = 0x94D049BB133111EBULL;

// Seed salts of the model's independent streams (reference: noise of the
// astrocytes astrocyte.cpp:318, Poisson drive of neurons neuron.cpp:230,
// independent neuron noise neuron.cpp:243, shared neuron noise
// neuron.cpp:204/208, astrocyte Poisson drive network.cpp:461, builder
// stream network.cpp:57).
constexpr std::uint64_t kSaltAstroNoise = 0x9E3779B97F4A7C15ULL;
constexpr std::uint64_t kSaltNeuronPoisson = 0x2545F4914F6CDD1DULL;
constexpr std::uint64_t kSaltNeuronNoise = 0x9E3779B185EBCA87ULL;
constexpr std::uint64_t kSaltSharedExc = 0xD1B54A32D192ED03ULL;
constexpr std::uint64_t kSaltSharedInh = 0xA24BAED4963EE407ULL;
constexpr std::uint64_t kSaltAstroPoisson = 0xC2B2AE3D27D4EB4FULL;
// Stream strides: step*1000003+cell (Poisson, astro noise), idx*1000033+cell
// (neuron noise).
constexpr std::uint64_t kStreamStride = 1000003ULL;
constexpr std::uint64_t kNoiseStride = 1000033ULL;

__host__ __device__ __forceinline__ std::uint64_t mix64(std::uint64_t seed, std::uint64_t stream,
                                                        std::uint64_t counter) {
    std::uint64_t z = seed + stream * kPhi + counter * kMixA;
    z = (z ^ (z >> 30)) * kMixA;
    z = (z ^ (z >> 27)) * kMixB;
    return z ^ (z >> 31);
}

// 53 random bits scaled into [0, 1).
__host__ __device__ __forceinline__ double unit53(std::uint64_t bits) {
    return static_cast<double>(bits >> 11) * (1.0 / 9007199254740992.0);
}

__host__ __device__ __forceinline__ double uniform_at(std::uint64_t seed, std::uint64_t stream,
                                                      std::uint64_t counter) {
    return unit53(mix64(seed, stream, counter));
}

constexpr double kTwoPi = 6.283185307179586476925286766559;

// Box-Muller cosine branch over counters 0 and 1 with u1 clamped at 1e-300
// (the free-function form, reference rng.hpp:42-50).
__device__ __forceinline__ double normal_clamped(std::uint64_t seed, std::uint64_t stream) {
    double u1 = uniform_at(seed, stream, 0);
    if (u1 <= 1e-300) u1 = 1e-300;
    const double u2 = uniform_at(seed, stream, 1);
    return sqrt(-2.0 * log(u1)) * cos(kTwoPi * u2);
}

static __device__ __noinline__ int poisson_large(std::uint64_t seed, std::uint64_t stream,
                                                 std::uint64_t counter, double lambda);

// Sequential draws of one (seed, stream), the CounterRng object form.
struct Draws {
    std::uint64_t seed, stream, counter;
    __device__ __forceinline__ Draws(std::uint64_t s, std::uint64_t st)
        : seed(s), stream(st), counter(0) {}
    __device__ __forceinline__ double uniform() { return uniform_at(seed, stream, counter++); }
    // First variate of a fresh object: Box-Muller cosine branch, u1 redrawn
    // while <= 1e-300 (rng.hpp:74-89).  The sine spare is never consumed on
    // the step path (each object serves one draw), so it is not formed.
    __device__ __forceinline__ double normal_first() {
        double u1;
        do {
            u1 = uniform();
        } while (u1 <= 1e-300);
        const double u2 = uniform();
        return sqrt(-2.0 * log(u1)) * cos(kTwoPi * u2);
    }
    // Knuth's product method for lambda <= 30 with exp(-lambda) supplied by
    // the caller (a per-population constant); normal approximation above,
    // out of line (rare, and it carries log/cos code the common path does
    // not need in the instruction cache).  The object is not used after.
    __device__ __forceinline__ int poisson(double lambda, double limit) {
        if (lambda <= 0.0) return 0;
        if (lambda > 30.0) return poisson_large(seed, stream, counter, lambda);
        double product = uniform();
        int count = 0;
        while (product > limit) {
            ++count;
            product *= uniform();
        }
        return count;
    }
};

// Normal approximation of Poisson(lambda) for lambda > 30 (rng.hpp:111-114):
// round(lambda + sqrt(lambda) * N(0,1)), clamped at zero.
static __device__ __noinline__ int poisson_large(std::uint64_t seed, std::uint64_t stream,
                                                 std::uint64_t counter, double lambda) {
    Draws r(seed, stream);
    r.counter = counter;
    const double v = lambda + sqrt(lambda) * r.normal_first();
    return v < 0.0 ? 0 : static_cast<int>(v + 0.5);
}

// ------------------------------------------------------------- division

// a / b for a divisor known in advance, from y = RN(1/b) formed once on the
// host (IEEE division, correctly rounded): q = RN(a*y), r = a - q*b exactly
// (one FMA), result RN(q + r*y).  Markstein's theorem (P. Markstein, "Computation
// of elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990; Muller et al., Handbook of Floating-Point Arithmetic, on
// division with a fused multiply-add) guarantees the result equals the
// correctly rounded a / b whenever y is the correctly rounded reciprocal and
// no underflow or overflow occurs, i.e. it is bitwise the IEEE quotient the
// reference computes, in three dependent operations instead of a full divide.
//
// The theorem's exclusions are kept off the fast path by the exponent of a
// (an integer test): with 2^-959 <= |a| < 2^978 and a divisor of magnitude
// in [2^-46, 2^63] (every divisor of the model is a time constant, a
// capacitance, a slope factor or a volume ratio well inside it), the
// quotient and the remainder are normal and the quotient is finite.  Every
// other a -- tiny, huge, +-0 (whose quotient keeps a's sign), inf, NaN --
// takes the IEEE division itself.  tests/div_by_check.cu checks the result
// against IEEE division over random and edge-case operands of every class.
__host__ __device__ __noinline__ inline double ieee_div(double a, double b) { return a / b; }

// Numerator outside the range where the reciprocal division is exact
// without a test (div_by's exponent test, as an integer flag).
__host__ __device__ __forceinline__ unsigned div_out_of_range(double a) {
#ifdef __CUDA_ARCH__
    const unsigned biased = (static_cast<unsigned>(__double2hiint(a)) >> 20) & 0x7FFu;
#else
    std::uint64_t u;
    __builtin_memcpy(&u, &a, sizeof u);
    const unsigned biased = static_cast<unsigned>(u >> 52) & 0x7FFu;
#endif
    return (biased - 64u > 1936u) ? 1u : 0u;
}

// div_by without its exponent test, for callers that test the numerator
// themselves (div_out_of_range) and redo the case it flags.
__host__ __device__ __forceinline__ double div_by_untested(double a, double b, double y) {
    const double q = a * y;
    const double r = fma(-q, b, a);
    return fma(r, y, q);
}

__host__ __device__ __forceinline__ double div_by(double a, double b, double y) {
    // biased exponent outside [64, 2000]: the IEEE division itself
    if (div_out_of_range(a)) return ieee_div(a, b);
    return div_by_untested(a, b, y);
}


// (x - y) / b through the reciprocal y_b = RN(1/b), without div_by's
// exponent test, for a numerator formed from a model parameter: one of x, y
// is a parameter of magnitude in [2^-906, 2^976] (checked on the host when
// the parameters are set).  A non-zero x - y then has a magnitude of at least
// 2^-959 -- if the other operand is below half the parameter the difference
// exceeds 2^-907, else both exponents are >= -907 and the difference is a
// multiple of 2^-959 -- so the remainder stays normal; x - y is never -0 (a
// difference is -0 only for -0 - +0, and the parameter is non-zero) and +0
// gives the IEEE +0; and the quotient is finite while |x - y| < 2^977, far
// beyond any concentration or potential of the model.  Under those
// conditions Markstein's theorem makes the result the IEEE (x - y) / b.
// tests/div_by_check.cu checks it over every operand class it covers.
__host__ __device__ __forceinline__ double div_diff_by(double x, double y, double b,
                                                       double yb) {
    const double a = x - y;
    const double q = a * yb;
    const double r = fma(-q, b, a);
    return fma(r, yb, q);
}

// Magnitude range a parameter needs for div_diff_by (see there).
__host__ __device__ __forceinline__ bool diff_param_ok(double p) {
    const double m = p < 0.0 ? -p : p;
    return m >= 0x1p-906 && m <= 0x1p976;
}

// ------------------------------------------------------ Li-Rinzel astrocyte

// Population constants, with the run-time constant products of the
// reference's right-hand side pre-formed (same rounding).
struct AstroK {
    double Kd_IP3_1, Kd_IP3_2, Kd_act, ratio_ER_cyt, inv_ratio;  // inv_ratio = 1/ratio_ER_cyt
    double chan;    // ratio_ER_cyt * rate_IP3R
    double serca;   // rate_SERCA
    double km2;     // Km_SERCA * Km_SERCA
    double leak;    // ratio_ER_cyt * rate_L
    double ah;      // k_IP3R * Kd_inh
    double k_IP3R;
    double half_h;  // 0.5 * h_step
    double h;       // h_step
    double h6;      // h_step / 6.0
    int substeps;
};

struct AstroRates {
    double Ca, IP3, h;
};

// d/dt of (Ca, IP3, h) for one cell.
// `tau` and `inv_tau` (its correctly rounded reciprocal) give dIP3 with
// div_diff_by; the result is the IEEE quotient (IP3_0 - IP3) / tau, as the ER
// calcium is (Ca_tot - Ca) / ratio_ER_cyt, for Ca_tot and IP3_0 within
// diff_param_ok (checked where the parameters enter the engine).
__device__ __forceinline__ AstroRates li_rinzel(const AstroK& k, double ca_tot, double ip3_0,
                                                double tau, double inv_tau, double ca, double ip3,
                                                double hh, double noise) {
    const double er = div_diff_by(ca_tot, ca, k.ratio_ER_cyt, k.inv_ratio);  // ER calcium
    const double ip3_k1 = ip3 + k.Kd_IP3_1;
    const double m = ip3 / ip3_k1;                      // IP3 activation
    const double n = ca / (ca + k.Kd_act);              // Ca activation
    const double m3 = m * m * m;
    const double n3 = n * n * n;
    const double h3 = hh * hh * hh;
    const double gradient = er - ca;
    const double release = k.chan * m3 * n3 * h3 * gradient;
    const double ca2 = ca * ca;
    const double uptake = k.serca * ca * ca / (k.km2 + ca2);
    const double leak = k.leak * gradient;
    const double open_rate = k.ah * ip3_k1 / (ip3 + k.Kd_IP3_2);
    const double close_rate = k.k_IP3R * ca;
    AstroRates r;
    r.Ca = release - uptake + leak + noise;
    r.IP3 = div_diff_by(ip3_0, ip3, tau, inv_tau);
    r.h = open_rate * (1.0 - hh) - close_rate * hh;
    return r;
}

// Input jump, then `substeps` classical RK4 steps with the physical clamps.
// kUnroll = false runs the four stages as a loop (one copy of the right-hand
// side in the instruction stream, for kernels that also hold other roles'
// code); the weighted stage sum is accumulated left to right either way, so
// both forms perform the same IEEE operations in the same order.
template <bool kUnroll = true>
__device__ __forceinline__ void astro_rk4(const AstroK& k, double ca_tot, double ip3_0, double tau,
                                          double inv_tau, double delta, double input, double noise,
                                          double& ca, double& ip3, double& hh) {
    if (input != 0.0) ip3 += delta * input;
    for (int s = 0; s < k.substeps; ++s) {
        double sCa = 0.0, sIP3 = 0.0, sh = 0.0;  // k1 + 2 k2 + 2 k3 + k4, in that order
        double xCa = ca, xIP3 = ip3, xh = hh;     // stage inputs
#pragma unroll(kUnroll ? 4 : 1)
        for (int st = 0; st < 4; ++st) {
            const AstroRates r = li_rinzel(k, ca_tot, ip3_0, tau, inv_tau, xCa, xIP3, xh, noise);
            if (st == 0) {
                sCa = r.Ca;
                sIP3 = r.IP3;
                sh = r.h;
            } else if (st < 3) {
                // s + 2r in one rounding: 2r is exact, so fma(2, r, s) is
                // the same IEEE result as s + (2.0 * r) (while 2r is finite)
                sCa = fma(2.0, r.Ca, sCa);
                sIP3 = fma(2.0, r.IP3, sIP3);
                sh = fma(2.0, r.h, sh);
            } else {
                sCa = sCa + r.Ca;
                sIP3 = sIP3 + r.IP3;
                sh = sh + r.h;
            }
            const double step = st < 2 ? k.half_h : k.h;
            xCa = ca + step * r.Ca;
            xIP3 = ip3 + step * r.IP3;
            xh = hh + step * r.h;
        }
        ca += k.h6 * sCa;
        ip3 += k.h6 * sIP3;
        hh += k.h6 * sh;
        ca = ca < 0.0 ? 0.0 : (ca > ca_tot ? ca_tot : ca);
        hh = hh < 0.0 ? 0.0 : (hh > 1.0 ? 1.0 : hh);
        ip3 = ip3 < 0.0 ? 0.0 : ip3;
    }
}

// ------------------------------------- Li-Rinzel in FP32 (precision study)
//
// The reference's precision question (docs/experiments.md, "Single or double
// precision"): is FP32 enough for the Li-Rinzel calcium dynamics, whose ER
// calcium (Ca_tot - Ca) / ratio_ER_cyt subtracts quantities of similar size?
// Its method is `real = float` throughout.  This is that form for the
// astrocyte: state rounded to float, every operation of the right-hand side
// and of the RK4 stages in float, IEEE float division, the same operation
// order.  It is an opt-in study form, never the default and never compared
// bitwise: the FP64 path above is the product.
struct AstroKf {
    float Kd_IP3_1, Kd_IP3_2, Kd_act, ratio_ER_cyt, chan, serca, km2, leak, ah, k_IP3R;
    float half_h, h, h6;
    int substeps;
};

__host__ __device__ inline AstroKf astro_k_f32(const AstroK& k) {
    AstroKf f;
    f.Kd_IP3_1 = static_cast<float>(k.Kd_IP3_1);
    f.Kd_IP3_2 = static_cast<float>(k.Kd_IP3_2);
    f.Kd_act = static_cast<float>(k.Kd_act);
    f.ratio_ER_cyt = static_cast<float>(k.ratio_ER_cyt);
    f.chan = static_cast<float>(k.chan);
    f.serca = static_cast<float>(k.serca);
    f.km2 = static_cast<float>(k.km2);
    f.leak = static_cast<float>(k.leak);
    f.ah = static_cast<float>(k.ah);
    f.k_IP3R = static_cast<float>(k.k_IP3R);
    f.half_h = static_cast<float>(k.half_h);
    f.h = static_cast<float>(k.h);
    f.h6 = static_cast<float>(k.h6);
    f.substeps = k.substeps;
    return f;
}

__device__ __forceinline__ void astro_rk4_f32(const AstroKf& k, float ca_tot, float ip3_0,
                                              float tau, float delta, float input, float noise,
                                              float& ca, float& ip3, float& hh) {
    auto rhs = [&](float c, float i3, float hv, float& dCa, float& dIP3, float& dh) {
        const float er = (ca_tot - c) / k.ratio_ER_cyt;
        const float ip3_k1 = i3 + k.Kd_IP3_1;
        const float m = i3 / ip3_k1;
        const float n = c / (c + k.Kd_act);
        const float m3 = m * m * m;
        const float n3 = n * n * n;
        const float h3 = hv * hv * hv;
        const float gradient = er - c;
        const float release = k.chan * m3 * n3 * h3 * gradient;
        const float ca2 = c * c;
        const float uptake = k.serca * c * c / (k.km2 + ca2);
        const float leak = k.leak * gradient;
        const float open_rate = k.ah * ip3_k1 / (i3 + k.Kd_IP3_2);
        const float close_rate = k.k_IP3R * c;
        dCa = release - uptake + leak + noise;
        dIP3 = (ip3_0 - i3) / tau;
        dh = open_rate * (1.0f - hv) - close_rate * hv;
    };
    if (input != 0.0f) ip3 += delta * input;
    for (int s = 0; s < k.substeps; ++s) {
        float sCa = 0.0f, sIP3 = 0.0f, sh = 0.0f;
        float xCa = ca, xIP3 = ip3, xh = hh;
#pragma unroll
        for (int st = 0; st < 4; ++st) {
            float rCa, rIP3, rh;
            rhs(xCa, xIP3, xh, rCa, rIP3, rh);
            if (st == 0) {
                sCa = rCa;
                sIP3 = rIP3;
                sh = rh;
            } else if (st < 3) {
                sCa = sCa + 2.0f * rCa;
                sIP3 = sIP3 + 2.0f * rIP3;
                sh = sh + 2.0f * rh;
            } else {
                sCa = sCa + rCa;
                sIP3 = sIP3 + rIP3;
                sh = sh + rh;
            }
            const float step = st < 2 ? k.half_h : k.h;
            xCa = ca + step * rCa;
            xIP3 = ip3 + step * rIP3;
            xh = hh + step * rh;
        }
        ca += k.h6 * sCa;
        ip3 += k.h6 * sIP3;
        hh += k.h6 * sh;
        ca = ca < 0.0f ? 0.0f : (ca > ca_tot ? ca_tot : ca);
        hh = hh < 0.0f ? 0.0f : (hh > 1.0f ? 1.0f : hh);
        ip3 = ip3 < 0.0f ? 0.0f : ip3;
    }
}

// ---------------------------------------------------------------- AdEx

// Population constants of one neuron population.
struct NeuronK {
    double C_m, g_L, E_L, V_th, Delta_T, a, tau_w, V_peak, E_ex, E_in, I_e;
    double inv_C_m, inv_Delta_T, inv_tau_w;  // correctly rounded reciprocals (div_by)
    double neg_g_L;      // -g_L
    double gl_dt;        // g_L * Delta_T
    double psc_ex, psc_in;           // e / tau_syn (neuron.cpp:157-158)
    double decay_ex, decay_in;       // exp(-h / tau_syn), host libm
    int ref_steps;                   // (int)(t_ref / h + 0.5)
    double poiss_rate, poiss_weight, lambda, knuth_limit;  // lambda = rate*dt*1e-3
    double noise_std;
    int independent_noise;
    int steps_per_noise;
};

struct AdexRates {
    double V, w;
};

// AdEx membrane and adaptation rates.  The spike current is skipped when
// `with_spike` is false: the refractory branch of the reference evaluates it
// but only uses dw, which does not depend on it.
template <bool with_spike>
__device__ __noinline__ AdexRates adex_ieee(const NeuronK& p, double V, double w, double g_ex,
                                            double g_in, double I_ext);

template <bool with_spike>
__device__ __forceinline__ AdexRates adex(const NeuronK& p, double V, double w, double g_ex,
                                          double g_in, double I_ext) {
    const double v = (p.V_peak < V) ? p.V_peak : V;  // std::min(V, V_peak)
    const double rel = v - p.E_L;
    AdexRates r;
    // The three divisions go through the reciprocals untested; their
    // numerators' exponent tests are or-ed into one flag (integer work off
    // the FP64 chain), and the rare evaluation they flag is redone with IEEE
    // divisions: one branch per right-hand side instead of one per division.
    unsigned bad = 0u;
    if (with_spike) {
        const double n_spike = v - p.V_th;
        bad |= div_out_of_range(n_spike);
        const double spike = p.gl_dt * exp(div_by_untested(n_spike, p.Delta_T, p.inv_Delta_T));
        const double syn_ex = g_ex * (v - p.E_ex);
        const double syn_in = g_in * (v - p.E_in);
        const double n_V = p.neg_g_L * rel + spike - syn_ex - syn_in - w + p.I_e + I_ext;
        bad |= div_out_of_range(n_V);
        r.V = div_by_untested(n_V, p.C_m, p.inv_C_m);
    } else {
        r.V = 0.0;
    }
    const double n_w = p.a * rel - w;
    bad |= div_out_of_range(n_w);
    r.w = div_by_untested(n_w, p.tau_w, p.inv_tau_w);
    if (bad != 0u) r = adex_ieee<with_spike>(p, V, w, g_ex, g_in, I_ext);
    return r;
}

// The same right-hand side with IEEE divisions (out of line: the rare case).
template <bool with_spike>
__device__ __noinline__ AdexRates adex_ieee(const NeuronK& p, double V, double w, double g_ex,
                                            double g_in, double I_ext) {
    const double v = (p.V_peak < V) ? p.V_peak : V;
    const double rel = v - p.E_L;
    AdexRates r;
    if (with_spike) {
        const double spike = p.gl_dt * exp((v - p.V_th) / p.Delta_T);
        const double syn_ex = g_ex * (v - p.E_ex);
        const double syn_in = g_in * (v - p.E_in);
        r.V = (p.neg_g_L * rel + spike - syn_ex - syn_in - w + p.I_e + I_ext) / p.C_m;
    } else {
        r.V = 0.0;
    }
    r.w = (p.a * rel - w) / p.tau_w;
    return r;
}

}  // namespace asg
