// Network::run on the B200 engine: the reference-side binding a maintainer
// adds to astrosimgpu behind its compile-time backend switch (one more
// mutually exclusive option beside ASTROSIMGPU_CUDA/OFFLOAD/KOKKOS,
// CMakeLists.txt:16-23).  It replaces the body of Network::run
// (src/network.cpp:357-473): the whole per-timestep loop runs on the GPU
// through the C ABI of include/asg_b200.h, and the host keeps what the
// reference keeps there -- the recorder, the phase profile and the final
// state in the populations.
//
// Built out of tree by integration/Makefile against the reference sources:
// the reference's own main.cpp, network.cpp and the rest, with network.cpp's
// definition of Network::run renamed aside so this one links in its place.
// Inside the reference the same code would sit in network.cpp under
// `#if defined(ASTROSIMGPU_B200)`, with direct access to Network's members;
// out of tree it reaches them the way the test shim does.
#define private public
#include "astrosimgpu/network.hpp"
#undef private

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "asg_b200.h"

namespace astrosimgpu {

namespace {

void check(int status, const char* what) {
    if (status != ASG_OK)
        throw std::runtime_error(std::string("B200 engine: ") + what + ": " + asg_last_error());
}

asg_neuron_params neuron_params(const NeuronParams& p) {
    asg_neuron_params o{};
    o.C_m = p.C_m;
    o.g_L = p.g_L;
    o.E_L = p.E_L;
    o.V_th = p.V_th;
    o.Delta_T = p.Delta_T;
    o.a = p.a;
    o.tau_w = p.tau_w;
    o.V_peak = p.V_peak;
    o.t_ref = p.t_ref;
    o.E_ex = p.E_ex;
    o.E_in = p.E_in;
    o.tau_syn_ex = p.tau_syn_ex;
    o.tau_syn_in = p.tau_syn_in;
    o.I_e = p.I_e;
    return o;
}

asg_input input_params(const InputParams& in, real dt) {
    asg_input o{};
    o.poiss_rate = in.poiss_rate;
    o.poiss_weight = in.poiss_weight;
    o.gauss_noise_std = in.gauss_noise_std;
    o.noise_dt = in.noise_dt > 0.0 ? in.noise_dt : 10.0 * dt;
    o.independent_noise = in.independent_noise ? 1 : 0;
    return o;
}

asg_csr csr_of(const ConnectionSet& c, index_t sources) {
    asg_csr o{};
    o.n_sources = sources;
    o.row_start = c.row_start.data();
    o.target = c.target.data();
    o.weight = c.weight.empty() ? nullptr : c.weight.data();
    o.delay_steps = c.delay_steps.empty() ? nullptr : c.delay_steps.data();
    o.stp_x = c.stp_x.empty() ? nullptr : c.stp_x.data();
    o.stp_u = c.stp_u.empty() ? nullptr : c.stp_u.data();
    o.stp_t_last = c.stp_t_last.empty() ? nullptr : c.stp_t_last.data();
    return o;
}

// Delay of a set in steps: the set's own (every edge carries the same), or
// delay_to_steps's rounding for an empty set (network.cpp:32-35).
int delay_steps(const ConnectionSet& c, real delay_ms, real dt) {
    if (!c.delay_steps.empty()) return c.delay_steps.front();
    return std::max(1, static_cast<int>(delay_ms / dt + 0.5));
}

}  // namespace

void Network::run(Recorder& recorder) {
    const ModelConfig& c = cfg_;
    const std::int64_t pre_steps = c.time.pre_steps();
    const std::int64_t total = pre_steps + c.time.sim_steps();
    const real dt = c.time.dt;
    const index_t N = neurons_.size(), NA = astro_.size();

    // Everything Network::build left: sizes, constants, the four connection
    // sets, per-cell parameters and the initial state.
    std::vector<double> V_reset(N), b(N);
    for (index_t i = 0; i < N; ++i) {
        V_reset[i] = neurons_.p_[i].V_reset;
        b[i] = neurons_.p_[i].b;
    }
    asg_network_desc d{};
    d.n_exc = c.N.N_exc;
    d.n_inh = c.N.N_inh;
    d.n_astro = c.N.N_astro;
    d.dt = dt;
    d.substeps = c.time.substeps;
    d.seed = c.seed;
    d.sic_interval = c.syn.sic_interval;
    d.d_e_steps = delay_steps(exc_primary_, c.syn.d_e, dt);
    d.d_i_steps = delay_steps(inh_primary_, c.syn.d_i, dt);
    d.d_a2n_steps = delay_steps(astro_neuron_, c.syn.d_a2n, dt);
    d.w_e = c.syn.w_e;
    d.w_i = c.syn.w_i;
    d.w_n2a = c.syn.w_n2a;
    d.w_a2n = c.syn.w_a2n;
    d.exc = neuron_params(c.neuron_exc);
    d.inh = neuron_params(c.neuron_inh);
    const AstrocyteParams& a = c.astro;
    d.astro = asg_astro_params{a.Kd_IP3_1, a.Kd_IP3_2,  a.Kd_act,     a.Kd_inh,
                               a.Km_SERCA, a.k_IP3R,    a.rate_IP3R,  a.rate_L,
                               a.rate_SERCA, a.ratio_ER_cyt, a.SIC_scale, a.SIC_th};
    d.input_exc = input_params(c.input_exc, dt);
    d.input_inh = input_params(c.input_inh, dt);
    d.input_astro = input_params(c.input_astro, dt);
    d.stp = asg_stp{c.syn.stp.enabled ? 1 : 0, c.syn.stp.U, c.syn.stp.tau_rec,
                    c.syn.stp.tau_fac};
    d.exc_primary = csr_of(exc_primary_, c.N.N_exc);
    d.inh_primary = csr_of(inh_primary_, c.N.N_inh);
    d.neuron_astro = csr_of(neuron_astro_, c.N.N_exc);
    d.astro_neuron = csr_of(astro_neuron_, c.N.N_astro);
    d.V_reset = V_reset.data();
    d.b = b.data();
    d.Ca_tot = astro_.Ca_tot_.data();
    d.IP3_0 = astro_.IP3_0_.data();
    d.tau_IP3 = astro_.tau_IP3_.data();
    d.delta_IP3 = astro_.delta_IP3_.data();
    d.V = neurons_.V_.data();
    d.w = neurons_.w_.data();
    d.g_ex = neurons_.g_ex_.data();
    d.dg_ex = neurons_.dg_ex_.data();
    d.g_in = neurons_.g_in_.data();
    d.dg_in = neurons_.dg_in_.data();
    d.I_sic = neurons_.I_sic_.data();
    d.refractory = neurons_.refractory_steps_.data();
    d.Ca = astro_.Ca_.data();
    d.IP3 = astro_.IP3_.data();
    d.h = astro_.h_.data();

    // Recording as network.cpp:443-462 does it: spikes from the first
    // recorded step, traces every record_every steps.
    const index_t astro_rec = c.record_astro ? std::min(c.record_astro_max, NA) : 0;
    const index_t neuron_rec = c.record_neuron ? std::min(c.record_neuron_max, N) : 0;
    asg_record_opts rec{};
    rec.record_from_step = pre_steps;
    rec.record_every = c.record_every;
    rec.spikes = c.record_spikes ? 1 : 0;
    rec.astro_max = astro_rec;
    rec.neuron_max = neuron_rec;

    asg_engine_opts opts{};
    asg_network* net = nullptr;
    check(asg_create(&d, &rec, &opts, &net), "create");

    using clock = std::chrono::steady_clock;
    std::vector<std::int64_t> spk_steps, a_steps, n_steps;
    std::vector<std::uint32_t> spk_src;
    std::vector<double> rCa, rIP3, rV, rIsic;
    // Writes what the engine recorded since the last fetch.
    auto drain = [&]() {
        std::int64_t ns = 0, ar = 0, nr = 0;
        check(asg_fetch_spikes(net, nullptr, nullptr, 0, &ns), "fetch_spikes");
        spk_steps.resize(static_cast<std::size_t>(std::max<std::int64_t>(ns, 1)));
        spk_src.resize(spk_steps.size());
        check(asg_fetch_spikes(net, spk_steps.data(), spk_src.data(), ns, &ns), "fetch_spikes");
        for (std::int64_t k = 0; k < ns; ++k)
            recorder.write_spike(static_cast<real>(spk_steps[k]) * dt, spk_src[k]);
        check(asg_fetch_record(net, nullptr, nullptr, nullptr, 0, &ar, nullptr, nullptr, nullptr,
                               0, &nr),
              "fetch_record");
        a_steps.resize(static_cast<std::size_t>(std::max<std::int64_t>(ar, 1)));
        n_steps.resize(static_cast<std::size_t>(std::max<std::int64_t>(nr, 1)));
        rCa.resize(a_steps.size() * std::max<index_t>(astro_rec, 1));
        rIP3.resize(rCa.size());
        rV.resize(n_steps.size() * std::max<index_t>(neuron_rec, 1));
        rIsic.resize(rV.size());
        check(asg_fetch_record(net, a_steps.data(), rCa.data(), rIP3.data(), ar, &ar,
                               n_steps.data(), rV.data(), rIsic.data(), nr, &nr),
              "fetch_record");
        // The reference writes a step's astrocyte rows, then its neuron rows.
        std::int64_t ia = 0, in = 0;
        while (ia < ar || in < nr) {
            const std::int64_t s = ia < ar ? (in < nr ? std::min(a_steps[ia], n_steps[in])
                                                       : a_steps[ia])
                                           : n_steps[in];
            const real t = static_cast<real>(s) * dt;
            if (ia < ar && a_steps[ia] == s) {
                for (index_t k = 0; k < astro_rec; ++k)
                    recorder.write_astro(t, k, rCa[ia * astro_rec + k], rIP3[ia * astro_rec + k]);
                ++ia;
            }
            if (in < nr && n_steps[in] == s) {
                for (index_t k = 0; k < neuron_rec; ++k)
                    recorder.write_neuron(t, k, rV[in * neuron_rec + k],
                                          rIsic[in * neuron_rec + k]);
                ++in;
            }
        }
    };

    // The transient, then the recorded window in calls of up to 10,000 steps
    // (the recorder is fed between calls); the phase profile covers the
    // recorded window only, as in the reference (network.cpp:371-378).
    check(asg_step(net, pre_steps), "step");
    drain();
    const auto t0 = clock::now();
    double device_ms = 0.0;
    for (std::int64_t done = pre_steps; done < total;) {
        const std::int64_t k = std::min<std::int64_t>(10000, total - done);
        check(asg_step(net, k), "step");
        double ms = 0.0;
        std::int64_t kernels = 0;
        check(asg_last_timing(net, &ms, &kernels), "timing");
        device_ms += ms;
        drain();
        done += k;
    }
    profile_.total = std::chrono::duration<double>(clock::now() - t0).count();
    // One fused kernel per step carries every phase; its device time is
    // reported as the neuron update, the rest of the wall time as "other".
    profile_.update_neuron = std::min(profile_.total, device_ms * 1e-3);

    // The final state back into the populations, as device_end does for the
    // reference's CUDA backend.
    asg_state st{};
    st.V = neurons_.V_.data();
    st.w = neurons_.w_.data();
    st.g_ex = neurons_.g_ex_.data();
    st.dg_ex = neurons_.dg_ex_.data();
    st.g_in = neurons_.g_in_.data();
    st.dg_in = neurons_.dg_in_.data();
    st.I_sic = neurons_.I_sic_.data();
    st.refractory = neurons_.refractory_steps_.data();
    st.Ca = astro_.Ca_.data();
    st.IP3 = astro_.IP3_.data();
    st.h = astro_.h_.data();
    check(asg_pull_state(net, &st), "pull_state");
    check(asg_destroy(net), "destroy");
}

}  // namespace astrosimgpu
