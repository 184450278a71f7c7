// Test infrastructure only: a C-callable window onto the REFERENCE simulator's
// own classes, compiled from the reference sources by oracle/Makefile into
// oracle/_ref/libastroref.so.  Only tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py load it, as the checker.  Nothing in the
// product links or calls it.
//
// The reference keeps the per-step phases and the population state private
// (network.hpp:69-110, neuron.hpp:56-82, astrocyte.hpp:51-71).  The shim
// reaches them by re-declaring `private` as `public` for the reference
// headers only; no reference source is copied here.
//
// One step of ref_net_step() runs the phases in the order Network::run does
// (network.cpp:385-431): apply_arrivals, drive_astrocytes, astrocyte update
// (+ clear_inputs), neuron update, deliver_spikes, deliver_sic every
// sic_interval steps.

#define private public
#include "astrosimgpu/network.hpp"
#include "astrosimgpu/analysis.hpp"
#include "astrosimgpu/astrocyte_kernel.hpp"
#undef private

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

using namespace astrosimgpu;

namespace {

struct RefNet {
    ModelConfig cfg;
    Network* net = nullptr;
};

void copy_err(const std::exception& e, char* err, int errlen) {
    if (err != nullptr && errlen > 0) {
        std::snprintf(err, static_cast<std::size_t>(errlen), "%s", e.what());
    }
}

ConnectionSet& set_of(RefNet* r, int which) {
    switch (which) {
        case 0: return r->net->exc_primary_;
        case 1: return r->net->inh_primary_;
        case 2: return r->net->neuron_astro_;
        default: return r->net->astro_neuron_;
    }
}

}  // namespace

extern "C" {

// Config values after load_config + the CLI overrides of main.cpp:216-233
// (negative override = keep the file's value).
void* ref_net_create(const char* config_path, long long seed, double sim_time, double pre_time,
                     long long n_astro, char* err, int errlen) {
    try {
        auto* r = new RefNet;
        r->cfg = load_config(config_path);
        if (seed >= 0) r->cfg.seed = static_cast<std::uint64_t>(seed);
        if (sim_time >= 0.0) r->cfg.time.sim_time = sim_time;
        if (pre_time >= 0.0) r->cfg.time.pre_sim_time = pre_time;
        if (n_astro >= 0) r->cfg.N.N_astro = static_cast<index_t>(n_astro);
        r->net = new Network(r->cfg);
        r->net->build();
        return r;
    } catch (const std::exception& e) {
        copy_err(e, err, errlen);
        return nullptr;
    }
}

// Same, but from JSON text (the caller edits the values it wants changed).
void* ref_net_create_text(const char* json_text, long long seed, char* err, int errlen) {
    try {
        // load_config only reads files; go through a temporary file.
        char path[] = "/tmp/asg_ref_cfg_XXXXXX";
        const int fd = mkstemp(path);
        if (fd < 0) throw std::runtime_error("mkstemp failed");
        FILE* f = fdopen(fd, "w");
        std::fputs(json_text, f);
        std::fclose(f);
        auto* r = new RefNet;
        try {
            r->cfg = load_config(path);
        } catch (...) {
            std::remove(path);
            delete r;
            throw;
        }
        std::remove(path);
        if (seed >= 0) r->cfg.seed = static_cast<std::uint64_t>(seed);
        r->net = new Network(r->cfg);
        r->net->build();
        return r;
    } catch (const std::exception& e) {
        copy_err(e, err, errlen);
        return nullptr;
    }
}

void ref_net_destroy(void* h) {
    auto* r = static_cast<RefNet*>(h);
    if (r == nullptr) return;
    delete r->net;
    delete r;
}

// n_astro, n_exc, n_inh, n_primary_exc, n_primary_inh, n_n2a, n_a2n, ring_slots, sic_delay
void ref_net_stats(void* h, std::int64_t* out) {
    auto* r = static_cast<RefNet*>(h);
    const NetworkStats& s = r->net->stats();
    out[0] = s.n_astro;
    out[1] = s.n_exc;
    out[2] = s.n_inh;
    out[3] = s.n_primary_exc;
    out[4] = s.n_primary_inh;
    out[5] = s.n_neuron_to_astro;
    out[6] = s.n_astro_to_neuron;
    out[7] = r->net->ring_slots_;
    out[8] = r->net->sic_delay_steps_;
}

// Scalars of the resolved config: dt, substeps, seed, pre_steps, sim_steps,
// noise_dt (astro, exc, inh).
void ref_net_time(void* h, double* out) {
    auto* r = static_cast<RefNet*>(h);
    out[0] = r->cfg.time.dt;
    out[1] = r->cfg.time.substeps;
    out[2] = static_cast<double>(r->cfg.seed);
    out[3] = static_cast<double>(r->cfg.time.pre_steps());
    out[4] = static_cast<double>(r->cfg.time.sim_steps());
    out[5] = r->cfg.input_astro.noise_dt;
    out[6] = r->cfg.input_exc.noise_dt;
    out[7] = r->cfg.input_inh.noise_dt;
}

std::int64_t ref_net_table_size(void* h, int which) {
    auto* r = static_cast<RefNet*>(h);
    return set_of(r, which).size();
}

std::int64_t ref_net_table_rows(void* h, int which) {
    auto* r = static_cast<RefNet*>(h);
    return static_cast<std::int64_t>(set_of(r, which).row_start.size()) - 1;
}

// Any pointer may be NULL. STP arrays are left untouched when the set has none.
void ref_net_table(void* h, int which, std::uint32_t* row_start, std::uint32_t* target,
                   double* weight, std::int32_t* delay, double* stp_x, double* stp_u,
                   double* stp_t_last) {
    auto* r = static_cast<RefNet*>(h);
    const ConnectionSet& c = set_of(r, which);
    if (row_start) std::memcpy(row_start, c.row_start.data(), c.row_start.size() * 4);
    if (target) std::memcpy(target, c.target.data(), c.target.size() * 4);
    if (weight) std::memcpy(weight, c.weight.data(), c.weight.size() * 8);
    if (delay) std::memcpy(delay, c.delay_steps.data(), c.delay_steps.size() * 4);
    if (stp_x && !c.stp_x.empty()) std::memcpy(stp_x, c.stp_x.data(), c.stp_x.size() * 8);
    if (stp_u && !c.stp_u.empty()) std::memcpy(stp_u, c.stp_u.data(), c.stp_u.size() * 8);
    if (stp_t_last && !c.stp_t_last.empty())
        std::memcpy(stp_t_last, c.stp_t_last.data(), c.stp_t_last.size() * 8);
}

// Per-cell parameters drawn at build time.
void ref_net_cells(void* h, double* V_reset, double* b, double* Ca_tot, double* IP3_0,
                   double* tau_IP3, double* delta_IP3) {
    auto* r = static_cast<RefNet*>(h);
    const NeuronPopulation& n = r->net->neurons_;
    for (std::size_t i = 0; i < n.p_.size(); ++i) {
        V_reset[i] = n.p_[i].V_reset;
        b[i] = n.p_[i].b;
    }
    const AstrocytePopulation& a = r->net->astro_;
    std::memcpy(Ca_tot, a.Ca_tot_.data(), a.Ca_tot_.size() * 8);
    std::memcpy(IP3_0, a.IP3_0_.data(), a.IP3_0_.size() * 8);
    std::memcpy(tau_IP3, a.tau_IP3_.data(), a.tau_IP3_.size() * 8);
    std::memcpy(delta_IP3, a.delta_IP3_.data(), a.delta_IP3_.size() * 8);
}

// Neuron state (7 doubles per cell, in the order V, w, g_ex, dg_ex, g_in,
// dg_in, I_sic, each an array of n_neurons) + refractory counters, and
// astrocyte state (Ca, IP3, h).
void ref_net_state(void* h, double* neuron7, std::int32_t* refractory, double* astro3) {
    auto* r = static_cast<RefNet*>(h);
    const NeuronPopulation& n = r->net->neurons_;
    const std::size_t N = n.V_.size();
    const vec<real>* arrs[7] = {&n.V_, &n.w_, &n.g_ex_, &n.dg_ex_, &n.g_in_, &n.dg_in_, &n.I_sic_};
    for (int k = 0; k < 7; ++k) std::memcpy(neuron7 + k * N, arrs[k]->data(), N * 8);
    std::memcpy(refractory, n.refractory_steps_.data(), N * 4);
    const AstrocytePopulation& a = r->net->astro_;
    const std::size_t NA = a.Ca_.size();
    std::memcpy(astro3, a.Ca_.data(), NA * 8);
    std::memcpy(astro3 + NA, a.IP3_.data(), NA * 8);
    std::memcpy(astro3 + 2 * NA, a.h_.data(), NA * 8);
}

// Ring contents: which 0 exc, 1 inh, 2 sic, 3 astro; out is [slots][cells].
void ref_net_ring(void* h, int which, double* out) {
    auto* r = static_cast<RefNet*>(h);
    const vec<vec<real>>* ring = which == 0   ? &r->net->ring_exc_
                                 : which == 1 ? &r->net->ring_inh_
                                 : which == 2 ? &r->net->ring_sic_
                                              : &r->net->ring_astro_;
    std::size_t off = 0;
    for (const auto& slot : *ring) {
        std::memcpy(out + off, slot.data(), slot.size() * 8);
        off += slot.size();
    }
}

// One step of Network::run's loop body (network.cpp:385-431), no recording.
// Writes the sorted spike sources to `spikes` (up to cap) and returns the
// number emitted.
int ref_net_step(void* h, std::int64_t step, std::uint32_t* spikes, int cap) {
    auto* r = static_cast<RefNet*>(h);
    Network& net = *r->net;
    net.apply_arrivals(step);
    net.drive_astrocytes(step);
    net.astro_.update(net.cfg_.time, step, net.cfg_.seed);
    net.astro_.clear_inputs(net.astro_input_sinks_);
    net.spike_buffer_.clear();
    net.neurons_.update(net.cfg_.time, step, net.cfg_.seed, net.spike_buffer_);
    net.deliver_spikes(net.spike_buffer_, step);
    if (step % net.cfg_.syn.sic_interval == 0) {
        net.deliver_sic(step);
    }
    const int n = static_cast<int>(net.spike_buffer_.size());
    for (int i = 0; i < n && i < cap; ++i) spikes[i] = net.spike_buffer_[i].source;
    return n;
}

// Runs steps [first, first+count) and appends (step, source) of every spike
// to the two arrays; returns the total spike count (may exceed cap).
std::int64_t ref_net_run(void* h, std::int64_t first, std::int64_t count, std::int64_t* spk_step,
                         std::uint32_t* spk_src, std::int64_t cap) {
    auto* r = static_cast<RefNet*>(h);
    std::int64_t total = 0;
    std::vector<std::uint32_t> buf(static_cast<std::size_t>(r->net->neurons_.size()) + 1);
    for (std::int64_t s = first; s < first + count; ++s) {
        const int n = ref_net_step(h, s, buf.data(), static_cast<int>(buf.size()));
        for (int i = 0; i < n; ++i) {
            if (total < cap) {
                spk_step[total] = s;
                spk_src[total] = buf[i];
            }
            ++total;
        }
    }
    return total;
}

// SIC factor per astrocyte (astrocyte.cpp:331-339) from the current Ca.
void ref_net_sic_factors(void* h, double* out) {
    auto* r = static_cast<RefNet*>(h);
    for (index_t a = 0; a < r->net->astro_.size(); ++a) out[a] = r->net->astro_.sic_factor(a);
}

// Overwrites the dynamic state (the layout of ref_net_state).  Used to start
// the reference from a state another simulator reached, or to perturb it.
void ref_net_set_state(void* h, const double* neuron7, const std::int32_t* refractory,
                       const double* astro3) {
    auto* r = static_cast<RefNet*>(h);
    NeuronPopulation& n = r->net->neurons_;
    const std::size_t N = n.V_.size();
    vec<real>* arrs[7] = {&n.V_, &n.w_, &n.g_ex_, &n.dg_ex_, &n.g_in_, &n.dg_in_, &n.I_sic_};
    for (int k = 0; k < 7; ++k) std::memcpy(arrs[k]->data(), neuron7 + k * N, N * 8);
    std::memcpy(n.refractory_steps_.data(), refractory, N * 4);
    AstrocytePopulation& a = r->net->astro_;
    const std::size_t NA = a.Ca_.size();
    std::memcpy(a.Ca_.data(), astro3, NA * 8);
    std::memcpy(a.IP3_.data(), astro3 + NA, NA * 8);
    std::memcpy(a.h_.data(), astro3 + 2 * NA, NA * 8);
}

// Replaces connection set `which` (0 exc, 1 inh, 2 neuron->astro, 3
// astro->neuron) by another CSR grouped by source -- e.g. the product's
// fixed-in-degree tables, which the reference's Bernoulli builder cannot
// make -- with the set's uniform weight and delay and fresh STP state (the
// set's own finalise, as build_primary_connections does), then re-derives
// what Network::build computes from the sets (network.cpp:64-98): the edge
// counts, the SIC sources and the astrocyte input sinks.  Returns 0, or -1
// when the row count does not match the set's sources.
int ref_net_load_table(void* h, int which, std::int64_t n_rows, const std::uint32_t* row_start,
                       const std::uint32_t* target) {
    auto* r = static_cast<RefNet*>(h);
    Network& net = *r->net;
    const ModelConfig& c = net.cfg_;
    const index_t sources[4] = {c.N.N_exc, c.N.N_inh, c.N.N_exc, c.N.N_astro};
    if (which < 0 || which > 3 || n_rows != static_cast<std::int64_t>(sources[which])) return -1;
    ConnectionSet& set = set_of(r, which);
    const std::size_t m = row_start[n_rows];
    set = ConnectionSet{};
    set.row_start.assign(row_start, row_start + n_rows + 1);
    set.target.assign(target, target + m);
    const double weights[4] = {c.syn.w_e, c.syn.w_i, c.syn.w_n2a, c.syn.w_a2n};
    const double delays_ms[4] = {c.syn.d_e, c.syn.d_i, c.syn.d_e, c.syn.d_a2n};
    const int delay = std::max(1, static_cast<int>(delays_ms[which] / c.time.dt + 0.5));
    set.weight.assign(m, weights[which]);
    set.delay_steps.assign(m, delay);
    StpParams none;
    none.enabled = false;
    set.finalise(sources[which], which == 3 ? none : c.syn.stp);

    net.stats_.n_primary_exc = net.exc_primary_.size();
    net.stats_.n_primary_inh = net.inh_primary_.size();
    net.stats_.n_neuron_to_astro = net.neuron_astro_.size();
    net.stats_.n_astro_to_neuron = net.astro_neuron_.size();
    net.sic_sources_.clear();
    for (index_t a = 0; a < c.N.N_astro; ++a)
        if (net.astro_neuron_.row_start[a] < net.astro_neuron_.row_start[a + 1])
            net.sic_sources_.push_back(a);
    vec<char> seen(c.N.N_astro, 0);
    net.astro_input_sinks_.clear();
    for (const index_t t : net.neuron_astro_.target)
        if (!seen[t]) {
            seen[t] = 1;
            net.astro_input_sinks_.push_back(t);
        }
    std::sort(net.astro_input_sinks_.begin(), net.astro_input_sinks_.end());
    return 0;
}

// ---- Free functions of the reference, exposed for known-answer checks ----

std::uint64_t ref_rng_bits(std::uint64_t seed, std::uint64_t stream, std::uint64_t counter) {
    return rng_bits(seed, stream, counter);
}
double ref_rng_uniform(std::uint64_t seed, std::uint64_t stream, std::uint64_t counter) {
    return rng_uniform(seed, stream, counter);
}
double ref_rng_normal(std::uint64_t seed, std::uint64_t stream) { return rng_normal(seed, stream); }

// CounterRng(seed, stream) then `n` calls of the method `kind`
// (0 uniform, 1 normal, 2 poisson(lambda)), results into out.
void ref_counter_rng(std::uint64_t seed, std::uint64_t stream, int kind, double lambda, int n,
                     double* out) {
    CounterRng r(seed, stream);
    for (int i = 0; i < n; ++i) {
        out[i] = kind == 0 ? r.uniform() : kind == 1 ? r.normal() : r.poisson(lambda);
    }
}

// astro_advance (astrocyte_kernel.hpp:71-103) on arrays, one call per cell.
// consts: Kd_IP3_1, Kd_IP3_2, Kd_act, Kd_inh, Km_SERCA, k_IP3R, rate_IP3R,
// rate_L, rate_SERCA, ratio_ER_cyt.
void ref_astro_advance(const double* consts, std::int64_t n, const double* Ca_tot,
                       const double* IP3_0, const double* tau_IP3, const double* delta_IP3,
                       const double* input, const double* noise, double h_step, int substeps,
                       double* Ca, double* IP3, double* h) {
    AstroConstants c{consts[0], consts[1], consts[2], consts[3], consts[4],
                     consts[5], consts[6], consts[7], consts[8], consts[9]};
    for (std::int64_t i = 0; i < n; ++i) {
        astro_advance(c, Ca_tot[i], IP3_0[i], tau_IP3[i], delta_IP3[i], input[i],
                      noise ? noise[i] : 0.0, h_step, substeps, Ca[i], IP3[i], h[i]);
    }
}

// The astrocyte kernel-scaling workload on the host, through the reference's
// own astro_advance, parallel over cells like astrocyte.cpp:307: N
// independent cells with uniform parameters, state at x0*(1+0.1*(2U-1)),
// U = rng_uniform(seed, cell, k) for k = 0,1,2 (Ca, IP3, h), and per step an
// input event of `weight` when rng_uniform(seed, cell, 1000+step) < p.
// Steps are [first, first+count).  Returns the wall seconds of the loop.
double ref_astro_scaling(const double* consts, double Ca_tot, double IP3_0, double tau_IP3,
                         double delta_IP3, double h_step, int substeps, std::uint64_t seed,
                         double p, double weight, std::int64_t first, std::int64_t count,
                         std::int64_t n, double* Ca, double* IP3, double* h, int threads) {
    AstroConstants c{consts[0], consts[1], consts[2], consts[3], consts[4],
                     consts[5], consts[6], consts[7], consts[8], consts[9]};
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
    const double t0 = omp_get_wtime();
#else
    (void)threads;
    const double t0 = 0.0;
#endif
    for (std::int64_t s = first; s < first + count; ++s) {
#pragma omp parallel for schedule(static)
        for (std::int64_t i = 0; i < n; ++i) {
            const std::uint64_t cell = static_cast<std::uint64_t>(i);
            const double in = rng_uniform(seed, cell, 1000 + static_cast<std::uint64_t>(s)) < p
                                  ? weight
                                  : 0.0;
            astro_advance(c, Ca_tot, IP3_0, tau_IP3, delta_IP3, in, 0.0, h_step, substeps,
                          Ca[i], IP3[i], h[i]);
        }
    }
#ifdef _OPENMP
    return omp_get_wtime() - t0;
#else
    return 0.0;
#endif
}

int ref_omp_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// ---- Analysis (analysis.cpp), for the long-run statistics ----

// detect_events + pairwise_correlation + summarise as main.cpp:266-315 drives
// them.  `times`/`ca` hold n_cells traces of n_samples each (row-major).
// out: active, transients, mean duration, pairs, mean pairwise correlation.
void ref_calcium_analysis(const double* times, const double* ca, int n_cells, int n_samples,
                          double threshold, double merge_gap, double win_start, double win_end,
                          double width, double shift, double* out) {
    vec<vec<real>> onsets;
    vec<real> durations;
    std::size_t active = 0;
    for (int c = 0; c < n_cells; ++c) {
        vec<real> t(times + static_cast<std::size_t>(c) * n_samples,
                    times + static_cast<std::size_t>(c + 1) * n_samples);
        vec<real> v(ca + static_cast<std::size_t>(c) * n_samples,
                    ca + static_cast<std::size_t>(c + 1) * n_samples);
        const EventTrain ev = detect_events(t, v, threshold, true, merge_gap);
        onsets.push_back(ev.onset);
        durations.insert(durations.end(), ev.duration.begin(), ev.duration.end());
        if (!ev.onset.empty()) ++active;
    }
    Interval window{win_start, win_end};
    const PairwiseCorrelation corr = pairwise_correlation(onsets, window, width, shift);
    const Summary dur = summarise(durations);
    out[0] = static_cast<double>(active);
    out[1] = static_cast<double>(dur.count);
    out[2] = dur.mean;
    out[3] = static_cast<double>(corr.coefficient.size());
    out[4] = corr.mean();
}

}  // extern "C"
