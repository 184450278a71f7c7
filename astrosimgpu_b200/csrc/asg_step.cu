// The fused per-timestep kernel of the network engine (layout and design in
// asg_engine.cuh).  Compiled with -fmad=false: every floating-point
// expression is evaluated as separate IEEE operations in the reference's
// order (neuron.cpp:101-250, astrocyte.cpp:233-329, network.cpp:230-355).

#include <cuda_runtime.h>

#include "asg_engine.cuh"

namespace asg {

namespace {

constexpr int kMaxBlock = 512;

// Routes one arrival the way NeuronPopulation::add_synaptic_input does
// (neuron.cpp:77-83): positive weights to the excitatory input, negative
// ones (as magnitudes) to the inhibitory input.
__device__ __forceinline__ void add_syn(double v, double& exc_in, double& inh_in) {
    if (v > 0.0) {
        exc_in += v;
    } else if (v < 0.0) {
        inh_in -= v;
    }
}

// Ordered sum of one target's arrivals in `slot` (see asg_engine.cuh), given
// the summary word already read (and cleared) by the caller.  Loads are
// issued in batches of independent requests -- up to 8 bitmap words, then up
// to 8 values -- so a target with several arrivals pays a few memory round
// trips, not one per arrival; the additions stay in ascending bit order.
// kSubtract selects ring_inh's `-=` accumulation (network.cpp:271-275).
template <bool kSubtract>
__device__ __forceinline__ double ring_gather(const InRing& R, int slot, std::uint32_t t,
                                              unsigned long long groups) {
    std::uint32_t* bits = R.bits + static_cast<std::size_t>(slot) * R.words;
    const double* vals = R.vals + static_cast<std::size_t>(slot) * R.words * 32;
    const std::uint32_t w0 = R.wbase[t], nw = R.wbase[t + 1] - w0;
    const std::uint32_t G = (nw + 63) >> 6;  // words per summary bit
    double acc = 0.0;
    std::uint32_t idx[8];
    int n = 0;
    auto flush = [&]() {
        double v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = k < n ? __ldcg(vals + idx[k]) : 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k < n) {
                if (kSubtract) {
                    acc -= v[k];
                } else {
                    acc += v[k];
                }
            }
        }
        n = 0;
    };
    auto take_word = [&](std::uint32_t q, std::uint32_t word) {
        while (word != 0) {
            const int b = __ffs(word) - 1;
            word &= word - 1;
            idx[n++] = q * 32 + b;
            if (n == 8) flush();
        }
    };
    // Word groups in ascending order, up to 8 words loaded at once.
    std::uint32_t q[8], wv[8];
    std::uint32_t cur = 0, cur_end = 0;  // words [cur, cur_end) of the open group
    bool open = false;
    for (;;) {
        int nq = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (!open && groups != 0) {
                const std::uint32_t g = __ffsll(groups) - 1;
                groups &= groups - 1;
                cur = w0 + g * G;
                cur_end = min(cur + G, w0 + nw);
                open = cur < cur_end;
            }
            q[k] = cur;
            if (open) {
                nq = k + 1;
                if (++cur >= cur_end) open = false;
            }
        }
        if (nq == 0) break;
#pragma unroll
        for (int k = 0; k < 8; ++k) wv[k] = k < nq ? __ldcg(bits + q[k]) : 0u;
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (k < nq && wv[k] != 0) bits[q[k]] = 0;
        for (int k = 0; k < nq; ++k) take_word(q[k], wv[k]);
    }
    flush();
    return acc;
}

// Sequential SIC sum of target t from the factors of emission slot fslot
// (network.cpp:281-299 order: ascending astrocyte, one add per edge).  The
// list entries and their factors are fetched 8 at a time with independent
// loads before the dependent additions.
__device__ __forceinline__ double sic_sum(const InstDev& I, std::uint32_t t, int fslot,
                                          unsigned long long& edges) {
    const std::uint32_t slice = t >> 5, lane = t & 31;
    const std::uint32_t o0 = I.sic_soff[slice], o1 = I.sic_soff[slice + 1];
    const std::uint32_t len = (o1 - o0) >> 5;
    const double* fac = I.fac + static_cast<std::size_t>(fslot) * I.NA;
    double acc = 0.0;
    for (std::uint32_t b0 = 0; b0 < len; b0 += 8) {
        std::uint32_t e[8];
        double f[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) e[k] = b0 + k < len ? __ldg(I.sic_ent + o0 + (b0 + k) * 32 + lane) : 0u;
#pragma unroll
        for (int k = 0; k < 8; ++k) f[k] = (e[k] & 0xFFu) ? __ldcg(fac + (e[k] >> 8)) : 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const std::uint32_t m = e[k] & 0xFFu;
            if (m == 0) return acc;  // padding ends the list
            if (f[k] == 0.0) continue;
            const double c = I.w_a2n * f[k];
            for (std::uint32_t r = 0; r < m; ++r) acc += c;
            edges += m;
        }
    }
    return acc;
}

// One arrival: value at the edge's bit, the bit, the target's summary bit.
__device__ __forceinline__ void push_edge(const InRing& R, int slot, unsigned long long pe,
                                          double value) {
    const std::uint32_t b = static_cast<std::uint32_t>(pe);
    const std::uint32_t t = static_cast<std::uint32_t>(pe >> 32) & 0x3FFFFFFu;
    const std::uint32_t g = static_cast<std::uint32_t>(pe >> 58);
    R.vals[static_cast<std::size_t>(slot) * R.words * 32 + b] = value;
    atomicOr(R.bits + static_cast<std::size_t>(slot) * R.words + (b >> 5), 1u << (b & 31));
    atomicOr(R.sum + static_cast<std::size_t>(slot) * R.n_targets + t, 1ull << g);
}

// Writes `value` at every out-edge of `row` (in-block push, used when a
// spike delay is a single step).
__device__ __forceinline__ void push_row(const std::uint32_t* rs, const InRing& R,
                                         std::uint32_t row, int slot, double value) {
    const std::uint32_t e1 = rs[row + 1];
#pragma unroll 4
    for (std::uint32_t e = rs[row] + threadIdx.x; e < e1; e += blockDim.x)
        push_edge(R, slot, __ldg(R.edge + e), value);
}

__device__ void neuron_role(const InstDev& I, const Work& wk, std::int64_t step) {
    __shared__ std::uint32_t s_spk[kMaxBlock];
    __shared__ double s_val[2 * kMaxBlock];
    __shared__ int s_nspk;
    if (threadIdx.x == 0) s_nspk = 0;
    __syncthreads();

    const std::uint32_t c = wk.first + threadIdx.x;
    if (threadIdx.x < wk.count) {
        const bool exc = c < I.NE;
        const NeuronK& P = exc ? I.pe : I.pi;
        const int slot = static_cast<int>(step % I.slots);

        // Issue every independent load of this cell before any store.
        const std::size_t so = static_cast<std::size_t>(slot);
        unsigned long long* sp_ex = I.ring_ex.sum + so * I.ring_ex.n_targets + c;
        unsigned long long* sp_in = I.ring_in.sum + so * I.ring_in.n_targets + c;
        const unsigned long long g_ex = __ldcg(sp_ex), g_in = __ldcg(sp_in);
        const std::int64_t se = step - I.d_a2n;
        const bool sic_due = se >= 0 && se % I.sic_interval == 0;
        double Isic = (sic_due && !I.fused_sic)
                          ? __ldcg(I.sic_val + static_cast<std::size_t>(step & 1) * I.N + c)
                          : I.Isic[c];
        double V = I.V[c], w = I.w[c], gex = I.gex[c], gin = I.gin[c];
        double dgex = I.dgex[c], dgin = I.dgin[c];
        int refr = I.refr[c];
        const double Vr = I.V_reset[c], bc = I.b[c];

        // apply_arrivals (network.cpp:301-338)
        double exc_in = 0.0, inh_in = 0.0;
        if (g_ex != 0) {
            *sp_ex = 0;
            const double ex = ring_gather<false>(I.ring_ex, slot, c, g_ex);
            if (ex != 0.0) add_syn(ex, exc_in, inh_in);
        }
        if (g_in != 0) {
            *sp_in = 0;
            const double in = ring_gather<true>(I.ring_in, slot, c, g_in);
            if (in != 0.0) add_syn(-in, exc_in, inh_in);
        }
        if (sic_due) {
            if (I.fused_sic) {
                unsigned long long edges = 0;
                Isic = sic_sum(I, c, static_cast<int>(se % I.slots), edges);
                if (edges) atomicAdd(I.counters + 1, edges);
            }
            I.Isic[c] = Isic;
        }

        // Poisson drive and noise (neuron.cpp:228-248)
        if (P.poiss_rate > 0.0) {
            Draws r(I.seed ^ kSaltNeuronPoisson,
                    static_cast<std::uint64_t>(step) * kStreamStride + c);
            const int ev = r.poisson(P.lambda, P.knuth_limit);
            if (ev > 0) exc_in += P.poiss_weight * static_cast<double>(ev);
        }
        double Iext = Isic;
        if (P.noise_std > 0.0) {
            const std::uint64_t idx = static_cast<std::uint64_t>(step / P.steps_per_noise);
            if (P.independent_noise) {
                Draws r(I.seed ^ kSaltNeuronNoise, idx * kNoiseStride + c);
                Iext += 0.0 + P.noise_std * r.normal_first();
            } else {
                Draws r(I.seed ^ (exc ? kSaltSharedExc : kSaltSharedInh), idx);
                Iext += 0.0 + P.noise_std * r.normal_first();
            }
        }

        if (exc_in != 0.0) dgex += exc_in * P.psc_ex;
        if (inh_in != 0.0) dgin += inh_in * P.psc_in;

        const double h = I.ak.h;  // h_step is shared by both models
        const double half_h = I.ak.half_h, h6 = I.ak.h6;
        bool spiked = false;
        for (int s = 0; s < I.ak.substeps; ++s) {
            const double gex1 = P.decay_ex * (gex + h * dgex);
            const double dgex1 = P.decay_ex * dgex;
            const double gin1 = P.decay_in * (gin + h * dgin);
            const double dgin1 = P.decay_in * dgin;
            if (refr > 0) {
                V = Vr;
                const AdexRates r = adex<false>(P, V, w, gex, gin, Iext);
                w += h * r.w;
            } else {
                // RK4 with the conductances at the start, midpoint and end of
                // the substep (neuron.cpp:285-298), stages as a loop; the stage
                // sum k1 + 2 k2 + 2 k3 + k4 accumulates left to right.
                const double gexm = 0.5 * (gex + gex1), ginm = 0.5 * (gin + gin1);
                double sV = 0.0, sw = 0.0, xV = V, xw = w;
#pragma unroll 1
                for (int st = 0; st < 4; ++st) {
                    const double ge = st == 0 ? gex : (st < 3 ? gexm : gex1);
                    const double gi = st == 0 ? gin : (st < 3 ? ginm : gin1);
                    const AdexRates r = adex<true>(P, xV, xw, ge, gi, Iext);
                    if (st == 0) {
                        sV = r.V;
                        sw = r.w;
                    } else if (st < 3) {
                        sV = sV + 2.0 * r.V;
                        sw = sw + 2.0 * r.w;
                    } else {
                        sV = sV + r.V;
                        sw = sw + r.w;
                    }
                    const double stp = st < 2 ? half_h : h;
                    xV = V + stp * r.V;
                    xw = w + stp * r.w;
                }
                V += h6 * sV;
                w += h6 * sw;
            }
            gex = gex1;
            dgex = dgex1;
            gin = gin1;
            dgin = dgin1;
            if (refr > 0) {
                --refr;
            } else if (V >= P.V_peak) {
                V = Vr;
                w += bc;
                refr = P.ref_steps;
                spiked = true;
            }
        }
        I.V[c] = V;
        I.w[c] = w;
        I.gex[c] = gex;
        I.dgex[c] = dgex;
        I.gin[c] = gin;
        I.dgin[c] = dgin;
        I.refr[c] = refr;

        if (spiked) {
            // Tsodyks-Markram update of this source (network.cpp:230-247); the
            // value its edges deliver is w*x*u per set.
            double x = 1.0, u = 1.0;
            if (I.stp_on) {
                const double t_now = static_cast<double>(step) * I.dt;
                const double d = t_now - I.stp_t[c];
                const double xd = exp(div_by(-d, I.tau_rec, I.inv_tau_rec));
                const double ud =
                    I.tau_fac < 1e-10 ? 0.0 : exp(div_by(-d, I.tau_fac, I.inv_tau_fac));
                x = I.stp_x[c];
                u = I.stp_u[c];
                x = 1.0 + (x - x * u - 1.0) * xd;
                u = I.U + u * (1.0 - I.U) * ud;
                I.stp_x[c] = x;
                I.stp_u[c] = u;
                I.stp_t[c] = t_now;
            }
            const double v0 =
                exc ? (I.stp_on ? I.w_e * x * u : I.w_e) : (I.stp_on ? I.w_i * x * u : I.w_i);
            const double v1 = exc ? (I.stp_on ? I.w_n2a * x * u : I.w_n2a) : 0.0;
            if (I.deferred_push) {
                const int ls = static_cast<int>(step % 3);
                std::uint32_t r0, len0, len1;
                if (exc) {
                    r0 = I.exc_rs[c];
                    len0 = I.exc_rs[c + 1] - r0;
                    len1 = I.n2a_rs[c + 1] - I.n2a_rs[c];
                } else {
                    r0 = I.inh_rs[c - I.NE];
                    len0 = I.inh_rs[c - I.NE + 1] - r0;
                    len1 = 0;
                }
                const unsigned long long old = atomicAdd(
                    I.spk_packed + ls, (1ull << 40) | static_cast<unsigned long long>(len0 + len1));
                const std::size_t o = static_cast<std::size_t>(ls) * I.N + (old >> 40);
                I.spk_meta[4 * o + 0] = c;
                I.spk_meta[4 * o + 1] = static_cast<std::uint32_t>(old & 0xFFFFFFFFFFull);
                I.spk_meta[4 * o + 2] = r0;
                I.spk_meta[4 * o + 3] = len0;
                I.spk_val[2 * o] = v0;
                I.spk_val[2 * o + 1] = v1;
            } else {
                s_val[threadIdx.x * 2 + 0] = v0;
                s_val[threadIdx.x * 2 + 1] = v1;
            }
            if (!I.deferred_push) {
                const int pos = atomicAdd(&s_nspk, 1);
                s_spk[pos] = threadIdx.x;
            }
            if (I.rec_spikes && step >= I.rec_from) {
                const unsigned long long li = atomicAdd(I.spike_log_n, 1ULL);
                if (li < I.spike_log_cap) {
                    I.spike_log[li] = (static_cast<unsigned long long>(step) << 32) | c;
                } else {
                    atomicAdd(I.counters + 3, 1ULL);
                }
            }
            unsigned long long edges =
                exc ? (I.exc_rs[c + 1] - I.exc_rs[c]) + (I.n2a_rs[c + 1] - I.n2a_rs[c])
                    : (I.inh_rs[c - I.NE + 1] - I.inh_rs[c - I.NE]);
            atomicAdd(I.counters + 0, edges);
            atomicAdd(I.counters + 2, 1ULL);
        }

        if (I.rec_neuron_max > 0 && c < I.rec_neuron_max && step >= I.rec_from &&
            (step - I.rec_from) % I.rec_every == 0) {
            const std::size_t row =
                static_cast<std::size_t>(((step - I.rec_from) / I.rec_every) % I.rec_rows);
            I.rec_V[row * I.rec_neuron_max + c] = V;
            I.rec_Isic[row * I.rec_neuron_max + c] = Isic;
        }
    }

    // Push the out-edges of this block's spiking sources into the rings of
    // their arrival steps (deliver_spikes, network.cpp:249-279).
    __syncthreads();
    const int nspk = s_nspk;
    for (int q = 0; q < nspk; ++q) {
        const std::uint32_t lane = s_spk[q];
        const std::uint32_t j = wk.first + lane;
        if (j < I.NE) {
            const int as = static_cast<int>((step + I.d_e) % I.slots);
            push_row(I.exc_rs, I.ring_ex, j, as, s_val[2 * lane]);
            push_row(I.n2a_rs, I.ring_as, j, as, s_val[2 * lane + 1]);
        } else {
            const int as = static_cast<int>((step + I.d_i) % I.slots);
            push_row(I.inh_rs, I.ring_in, j - I.NE, as, s_val[2 * lane]);
        }
    }
}

// Deferred push of the spikes of step-1.  The instance's PUSH blocks stride
// over the flat edge space of that step (edge x belongs to the spike whose
// range holds it, found by binary search in shared memory), so the work is
// split evenly whatever the number of spikes.  One thread also clears the
// list slot the next step appends to.
constexpr int kPushBatch = 256;

__device__ void push_role(const InstDev& I, const Work& wk, std::int64_t step) {
    __shared__ std::uint32_t s_off[kPushBatch + 1], s_src[kPushBatch], s_r0[kPushBatch],
        s_len0[kPushBatch];
    __shared__ double s_v[2 * kPushBatch];
    if (wk.first == 0 && threadIdx.x == 0) I.spk_packed[(step + 1) % 3] = 0;
    if (step == 0) return;
    const int ls = static_cast<int>((step - 1) % 3);
    const unsigned long long packed = __ldcg(I.spk_packed + ls);
    const std::uint32_t n = static_cast<std::uint32_t>(packed >> 40);
    const std::uint32_t total = static_cast<std::uint32_t>(packed & 0xFFFFFFFFFFull);
    const std::uint32_t stride = blockDim.x * I.push_blocks;
    const std::uint32_t gtid = wk.first * blockDim.x + threadIdx.x;
    const int as_e = static_cast<int>((step - 1 + I.d_e) % I.slots);
    const int as_i = static_cast<int>((step - 1 + I.d_i) % I.slots);
    const std::size_t base = static_cast<std::size_t>(ls) * I.N;
    for (std::uint32_t b0 = 0; b0 < n; b0 += kPushBatch) {
        const std::uint32_t nb = min(static_cast<std::uint32_t>(kPushBatch), n - b0);
        __syncthreads();
        for (std::uint32_t i = threadIdx.x; i < nb; i += blockDim.x) {
            const std::size_t o = base + b0 + i;
            s_src[i] = __ldcg(I.spk_meta + 4 * o + 0);
            s_off[i] = __ldcg(I.spk_meta + 4 * o + 1);
            s_r0[i] = __ldcg(I.spk_meta + 4 * o + 2);
            s_len0[i] = __ldcg(I.spk_meta + 4 * o + 3);
            s_v[2 * i] = __ldcg(I.spk_val + 2 * o);
            s_v[2 * i + 1] = __ldcg(I.spk_val + 2 * o + 1);
        }
        if (threadIdx.x == 0)
            s_off[nb] = b0 + nb < n ? __ldcg(I.spk_meta + 4 * (base + b0 + nb) + 1) : total;
        __syncthreads();
        // The list order is the atomic order, so offsets ascend along it.
        const std::uint32_t x0 = s_off[0], x1 = s_off[nb];
#pragma unroll 4
        for (std::uint32_t x = x0 + gtid; x < x1; x += stride) {
            std::uint32_t lo = 0, hi = nb;  // last entry with s_off <= x
            while (hi - lo > 1) {
                const std::uint32_t mid = (lo + hi) >> 1;
                if (s_off[mid] <= x) lo = mid; else hi = mid;
            }
            const std::uint32_t j = s_src[lo];
            const std::uint32_t k = x - s_off[lo];
            if (j >= I.NE) {
                push_edge(I.ring_in, as_i, __ldg(I.ring_in.edge + s_r0[lo] + k), s_v[2 * lo]);
            } else if (k < s_len0[lo]) {
                push_edge(I.ring_ex, as_e, __ldg(I.ring_ex.edge + s_r0[lo] + k), s_v[2 * lo]);
            } else {
                push_edge(I.ring_as, as_e, __ldg(I.ring_as.edge + I.n2a_rs[j] + (k - s_len0[lo])),
                          s_v[2 * lo + 1]);
            }
        }
    }
}

__device__ void astro_role(const InstDev& I, const Work& wk, std::int64_t step) {
    if (threadIdx.x >= wk.count) return;
    const std::uint32_t a = wk.first + threadIdx.x;
    const int slot = static_cast<int>(step % I.slots);
    unsigned long long* sp = I.ring_as.sum + static_cast<std::size_t>(slot) * I.ring_as.n_targets + a;
    const unsigned long long g = __ldcg(sp);
    double ca = I.Ca[a], ip3 = I.IP3[a], hh = I.h[a];
    double ip3_in = 0.0;
    if (g != 0) {
        *sp = 0;
        const double v = ring_gather<false>(I.ring_as, slot, a, g);
        if (v != 0.0) ip3_in += v;
    }
    // drive_astrocytes (network.cpp:340-355)
    if (I.a_rate > 0.0) {
        Draws r(I.seed ^ kSaltAstroPoisson, static_cast<std::uint64_t>(step) * kStreamStride + a);
        const int ev = r.poisson(I.a_lambda, I.a_limit);
        if (ev > 0) ip3_in += I.a_weight * static_cast<double>(ev);
    }
    // AstrocytePopulation::update (astrocyte.cpp:307-329)
    double noise = 0.0;
    if (I.a_std > 0.0) {
        const std::uint64_t idx = static_cast<std::uint64_t>(step / I.a_steps_per_noise);
        const std::uint64_t nseed = I.seed ^ kSaltAstroNoise;
        noise = I.a_indep ? I.a_std * normal_clamped(nseed, idx * kStreamStride + a)
                          : I.a_std * normal_clamped(nseed, idx);
    }
    if (I.astro_uniform) {
        astro_rk4<false>(I.ak, I.Ca_tot_u, I.IP3_0_u, I.tau_u, I.inv_tau_u, I.delta_u, ip3_in,
                         noise, ca, ip3, hh);
    } else {
        astro_rk4<false>(I.ak, I.Ca_tot[a], I.IP3_0[a], I.tau[a], I.inv_tau[a], I.delta[a],
                         ip3_in, noise, ca, ip3, hh);
    }
    I.Ca[a] = ca;
    I.IP3[a] = ip3;
    I.h[a] = hh;
    // SIC factor of this step (astrocyte.cpp:331-339), read by the SIC sums
    // of the arrival step.
    if (step % I.sic_interval == 0) {
        const double y = (ca - I.SIC_th) * 1000.0;
        I.fac[static_cast<std::size_t>(slot) * I.NA + a] = y <= 1.0 ? 0.0 : I.SIC_scale * log(y);
    }
    if (I.rec_astro_max > 0 && a < I.rec_astro_max && step >= I.rec_from &&
        (step - I.rec_from) % I.rec_every == 0) {
        const std::size_t row =
            static_cast<std::size_t>(((step - I.rec_from) / I.rec_every) % I.rec_rows);
        I.rec_Ca[row * I.rec_astro_max + a] = ca;
        I.rec_IP3[row * I.rec_astro_max + a] = ip3;
    }
}

// SIC current arriving at step+1 (valid when d_a2n >= 2: its factors were
// written by a launch that has completed).
__device__ void sic_role(const InstDev& I, const Work& wk, std::int64_t step) {
    const std::uint32_t t = wk.first + threadIdx.x;
    const std::int64_t arr = step + 1;
    const std::int64_t se = arr - I.d_a2n;
    unsigned long long edges = 0;
    // Computed even when step+1 lies past this chunk: the next chunk reads it.
    if (threadIdx.x < wk.count && se >= 0 && se % I.sic_interval == 0) {
        I.sic_val[static_cast<std::size_t>(arr & 1) * I.N + t] =
            sic_sum(I, t, static_cast<int>(se % I.slots), edges);
    }
    // one atomic per warp
    for (int o = 16; o > 0; o >>= 1) edges += __shfl_down_sync(0xFFFFFFFFu, edges, o);
    if ((threadIdx.x & 31) == 0 && edges) atomicAdd(I.counters + 1, edges);
}

__global__ void __launch_bounds__(kMaxBlock) step_kernel(const InstDev* __restrict__ insts,
                                                         const Work* __restrict__ work, int k) {
    // Stage this block's instance descriptor in shared memory.
    __shared__ __align__(16) unsigned char s_raw[sizeof(InstDev)];
    const Work wk = work[blockIdx.x];
    {
        const auto* src = reinterpret_cast<const std::uint32_t*>(insts + wk.inst);
        auto* dst = reinterpret_cast<std::uint32_t*>(s_raw);
        for (unsigned i = threadIdx.x; i < sizeof(InstDev) / 4; i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const InstDev& I = *reinterpret_cast<const InstDev*>(s_raw);
    // Programmatic dependent launch: let the next step's grid be scheduled
    // now, and wait here until the previous step's grid has completed and
    // its memory is visible.  The descriptor and work table read above were
    // written before the chunk started.
    asm volatile("griddepcontrol.launch_dependents;");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const std::int64_t step = I.step0 + k;
    if (step >= I.end_step) return;
    if (wk.role == kRoleNeuron) {
        neuron_role(I, wk, step);
    } else if (wk.role == kRoleAstro) {
        astro_role(I, wk, step);
    } else if (wk.role == kRolePush) {
        push_role(I, wk, step);
    } else {
        sic_role(I, wk, step);
    }
}

// Grid-wide barrier of the persistent chunk kernel (all blocks co-resident
// by cooperative launch).  Sense by generation count; every wait is bounded:
// a block that polls kBarrierPolls times without release sets the error word
// and the whole grid stops at its next barrier, so a fault can only end the
// launch early, never hang it.
constexpr unsigned kBarrierPolls = 1u << 24;  // x ~64 ns sleep: ~1 s

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ bool grid_sync(GridBarrier* gb, unsigned nblocks) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned gen = ld_acquire(&gb->gen);
        __threadfence();
        int ok = 1;
        if (atomicAdd(&gb->count, 1u) == nblocks - 1) {
            atomicExch(&gb->count, 0u);
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        } else {
            unsigned polls = 0;
            while (ld_acquire(&gb->gen) == gen) {
                if (++polls > kBarrierPolls || ld_acquire(&gb->error) != 0) {
                    atomicExch(&gb->error, 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (ld_acquire(&gb->error) != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// All `steps` steps of a chunk in one cooperative launch: each block takes
// work items blockIdx.x, blockIdx.x + gridDim.x, ... of every step, with a
// grid barrier between steps.  Data other blocks wrote in earlier steps is
// read through L2 (__ldcg in the roles), never a stale L1 line.
__global__ void __launch_bounds__(kMaxBlock) chunk_kernel(const InstDev* __restrict__ insts,
                                                          const Work* __restrict__ work,
                                                          int n_work, int steps,
                                                          GridBarrier* gb) {
    __shared__ __align__(16) unsigned char s_raw[sizeof(InstDev)];
    __shared__ unsigned s_inst;
    if (threadIdx.x == 0) s_inst = 0xFFFFFFFFu;
    const InstDev& I = *reinterpret_cast<const InstDev*>(s_raw);
    for (int k = 0; k < steps; ++k) {
        for (int wi = blockIdx.x; wi < n_work; wi += gridDim.x) {
            const Work wk = work[wi];
            __syncthreads();
            if (s_inst != wk.inst) {
                const auto* src = reinterpret_cast<const std::uint32_t*>(insts + wk.inst);
                auto* dst = reinterpret_cast<std::uint32_t*>(s_raw);
                for (unsigned i = threadIdx.x; i < sizeof(InstDev) / 4; i += blockDim.x)
                    dst[i] = src[i];
                __syncthreads();
                if (threadIdx.x == 0) s_inst = wk.inst;
                __syncthreads();
            }
            const std::int64_t step = I.step0 + k;
            if (step < I.end_step) {
                if (wk.role == kRoleNeuron) {
                    neuron_role(I, wk, step);
                } else if (wk.role == kRoleAstro) {
                    astro_role(I, wk, step);
                } else if (wk.role == kRolePush) {
                    push_role(I, wk, step);
                } else {
                    sic_role(I, wk, step);
                }
            }
        }
        if (k + 1 < steps && !grid_sync(gb, gridDim.x)) return;
    }
}

// Failure-detection check of the bounded barrier: block 0 never arrives, so
// every other block's wait must run out, set the error word and return.
__global__ void barrier_selftest_kernel(GridBarrier* gb) {
    if (blockIdx.x == 0) return;
    grid_sync(gb, gridDim.x);
}

}  // namespace

cudaError_t barrier_selftest(GridBarrier* gb, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(4);
    cfg.blockDim = dim3(32);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, barrier_selftest_kernel, gb);
}

int persistent_blocks(int block) {
    int per_sm = 0, dev = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, chunk_kernel, block, 0) !=
        cudaSuccess)
        return 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return per_sm * sms;
}

cudaError_t launch_chunk_persistent(const InstDev* insts, const Work* work, int n_work,
                                    int block, int grid, int steps, GridBarrier* gb,
                                    cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(static_cast<unsigned>(block));
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, chunk_kernel, insts, work, n_work, steps, gb);
}

cudaError_t launch_step(const InstDev* insts, const Work* work, int n_work, int block, int k,
                        bool pdl, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(n_work));
    cfg.blockDim = dim3(static_cast<unsigned>(block));
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = pdl ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, step_kernel, insts, work, k);
}

}  // namespace asg
