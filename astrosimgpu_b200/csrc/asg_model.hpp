// Host-side model: configuration (the reference's JSON schema), the network
// builder, and the counter-based fixed-in-degree generator.  These are the
// callers of the engine's C ABI in the standalone build; in the reference
// they are load_config (parameters.cpp:85-205) and Network::build
// (network.cpp:56-228).
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "asg_b200.h"

namespace asg {

// ---------------------------------------------------------------- JSON
// Minimal JSON reader with '//' line comments and lookup tracking: every key
// looked up is remembered, and unused() lists the ones nobody asked for
// (reference behaviour, json.cpp:258-282).
class JValue {
public:
    enum class Kind { Null, Bool, Number, String, Array, Object };
    static JValue parse(const std::string& text);  // throws std::runtime_error

    Kind kind() const { return kind_; }
    bool is_object() const { return kind_ == Kind::Object; }
    const JValue& at(const std::string& key) const;  // records the lookup
    template <typename T> void read(const std::string& key, T& out) const;
    void read(const std::string& key, bool& out) const;
    void read(const std::string& key, std::string& out) const;
    void unused(const std::string& prefix, std::vector<std::string>& out) const;

    Kind kind_ = Kind::Null;
    bool b_ = false;
    double num_ = 0.0;
    std::string str_;
    std::vector<JValue> arr_;
    std::map<std::string, JValue> obj_;
    mutable std::vector<std::string> looked_up_;
};

template <typename T> void JValue::read(const std::string& key, T& out) const {
    const JValue& v = at(key);
    if (v.kind_ == Kind::Number) out = static_cast<T>(v.num_);
}

// ------------------------------------------------------------- config
struct NeuronPop {
    double C_m = 281.0, g_L = 30.0, E_L = -70.6, V_th = -50.4, Delta_T = 2.0, a = 4.0, b = 80.5,
           tau_w = 144.0, V_reset = -60.0, V_peak = 0.0, t_ref = 0.0, E_ex = 0.0, E_in = -85.0,
           tau_syn_ex = 0.2, tau_syn_in = 2.0, I_e = 0.0, V_m_init = -70.6;
};

struct AstroPop {
    double Ca_tot = 2.0, IP3_0 = 0.16, Kd_IP3_1 = 0.13, Kd_IP3_2 = 0.9434, Kd_act = 0.08234,
           Kd_inh = 1.049, Km_SERCA = 0.1, SIC_scale = 1.0, SIC_th = 0.19669, delta_IP3 = 0.0002,
           k_IP3R = 0.0002, rate_IP3R = 0.006, rate_L = 0.00011, rate_SERCA = 0.0009,
           ratio_ER_cyt = 0.185, tau_IP3 = 7142.0, Ca_init = 0.073, h_init = 0.793,
           IP3_init = 0.16;
};

struct Drive {
    double poiss_rate = 0.0, poiss_weight = 1.0, noise_std = 0.0, noise_dt = 0.0;
    bool independent = true;
};

struct Spread {
    bool enabled = false;
    double lower = 1.0, upper = 1.0, var = 0.0;
};

struct ModelConfig {
    std::uint32_t N_A = 100, N_E = 400, N_I = 100;
    double dt = 0.1, pre_sim_time = 0.0, sim_time = 0.0;
    int substeps = 1;
    std::uint64_t seed = 1;
    AstroPop astro;
    NeuronPop exc, inh;
    double w_e = 5.0, w_i = -5.0, w_n2a = 0.2, w_a2n = 1.0, d_e = 1.0, d_i = 1.0, d_a2n = 1.0;
    int sic_interval = 1;
    bool stp_on = true;
    double U = 0.5, tau_rec = 800.0, tau_fac = 0.0;
    double p_primary = 0.2, p_third = 0.2;
    int pool_size = 1;
    bool pool_random = false, autapses = false, unique_third = false;
    Drive in_astro, in_exc, in_inh;
    Spread rnd_astro, rnd_neuron;
    bool analysis = true;
    double ca_threshold = -1.0, merge_gap = 2000.0, hist_window = 2000.0, hist_shift = 400.0;
    bool record_spikes = true, record_astro = true, record_neuron = false;
    int record_every = 10;
    std::uint32_t record_astro_max = 100, record_neuron_max = 50;
    std::string output_dir = "results";

    std::int64_t pre_steps() const { return static_cast<std::int64_t>(pre_sim_time / dt + 0.5); }
    std::int64_t sim_steps() const { return static_cast<std::int64_t>(sim_time / dt + 0.5); }
};

// Throws std::runtime_error on malformed text, bad values or unknown keys.
ModelConfig config_from_json(const std::string& text, const std::string& where);

int delay_steps(double ms, double dt);

// ------------------------------------------------------------- network
struct HostCsr {
    std::vector<std::uint32_t> row_start, target;
};

struct Model {
    ModelConfig cfg;
    bool built = false;
    HostCsr exc, inh, n2a, a2n;
    std::vector<double> V_reset, b, Ca_tot, IP3_0, tau_IP3, delta_IP3;
    std::vector<std::uint32_t> zero_row;  // placeholder row_start for empty sets
};

// Network::build (network.cpp:56-228): one sequential counter stream
// (seed, 0x5EED) drawn in the reference's order.
void build_reference(Model& m);
// Per-cell parameters only (the sequential stream of the reference builder).
void build_fixed_indegree_host_cells(Model& m);
// Counter-based fixed in-degree generator (host form).
void build_fixed_indegree_host(Model& m, std::uint32_t k_in);
// Same tables, generated on the device.
int build_fixed_indegree_device(Model& m, std::uint32_t k_in, int device);

void fill_desc(const Model& m, asg_network_desc& d);

}  // namespace asg
