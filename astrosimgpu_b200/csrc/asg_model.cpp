// Host-side model: JSON configuration in the reference's schema, the
// bit-exact network builder, the fixed-in-degree generator (host form) and
// the asg_model_* C ABI.

#include "asg_model.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <unordered_set>

#include "asg_common.hpp"
#include "asg_device.cuh"

namespace asg {

// ================================================================= JSON

namespace {

const JValue& null_value() {
    static const JValue v;
    return v;
}

class Reader {
public:
    explicit Reader(const std::string& t) : t_(t) {}

    JValue document() {
        space();
        JValue v = value();
        space();
        if (p_ != t_.size()) error("unexpected characters after the document");
        return v;
    }

private:
    [[noreturn]] void error(const char* what) const {
        std::ostringstream os;
        os << "JSON error at byte " << p_ << ": " << what;
        throw std::runtime_error(os.str());
    }
    void space() {
        for (;;) {
            while (p_ < t_.size() && std::isspace(static_cast<unsigned char>(t_[p_]))) ++p_;
            if (p_ + 1 < t_.size() && t_[p_] == '/' && t_[p_ + 1] == '/') {
                while (p_ < t_.size() && t_[p_] != '\n') ++p_;  // line comment
                continue;
            }
            return;
        }
    }
    char peek() const {
        if (p_ >= t_.size()) error("unexpected end of input");
        return t_[p_];
    }
    JValue value() {
        const char c = peek();
        if (c == '{') return object();
        if (c == '[') return array();
        if (c == '"') {
            JValue v;
            v.kind_ = JValue::Kind::String;
            v.str_ = string();
            return v;
        }
        if (t_.compare(p_, 4, "true") == 0) return boolean(true, 4);
        if (t_.compare(p_, 5, "false") == 0) return boolean(false, 5);
        if (t_.compare(p_, 4, "null") == 0) {
            p_ += 4;
            return JValue{};
        }
        return number();
    }
    JValue boolean(bool b, std::size_t len) {
        p_ += len;
        JValue v;
        v.kind_ = JValue::Kind::Bool;
        v.b_ = b;
        return v;
    }
    JValue number() {
        const std::size_t s = p_;
        while (p_ < t_.size() && (std::isdigit(static_cast<unsigned char>(t_[p_])) ||
                                  std::strchr("+-.eE", t_[p_]) != nullptr))
            ++p_;
        if (p_ == s) error("expected a value");
        JValue v;
        v.kind_ = JValue::Kind::Number;
        v.num_ = std::strtod(t_.substr(s, p_ - s).c_str(), nullptr);
        return v;
    }
    std::string string() {
        ++p_;  // opening quote
        std::string out;
        while (peek() != '"') {
            char c = t_[p_++];
            if (c == '\\') {
                const char e = peek();
                ++p_;
                switch (e) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'r': out += '\r'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'u': p_ += 4; out += '?'; break;
                    default: out += e;
                }
            } else {
                out += c;
            }
        }
        ++p_;
        return out;
    }
    JValue array() {
        ++p_;
        JValue v;
        v.kind_ = JValue::Kind::Array;
        space();
        if (peek() == ']') {
            ++p_;
            return v;
        }
        for (;;) {
            space();
            v.arr_.push_back(value());
            space();
            const char c = peek();
            ++p_;
            if (c == ']') return v;
            if (c != ',') error("expected ',' or ']'");
        }
    }
    JValue object() {
        ++p_;
        JValue v;
        v.kind_ = JValue::Kind::Object;
        space();
        if (peek() == '}') {
            ++p_;
            return v;
        }
        for (;;) {
            space();
            if (peek() != '"') error("expected a key");
            std::string k = string();
            space();
            if (peek() != ':') error("expected ':'");
            ++p_;
            space();
            v.obj_[k] = value();
            space();
            const char c = peek();
            ++p_;
            if (c == '}') return v;
            if (c != ',') error("expected ',' or '}'");
        }
    }

    const std::string& t_;
    std::size_t p_ = 0;
};

}  // namespace

JValue JValue::parse(const std::string& text) { return Reader(text).document(); }

const JValue& JValue::at(const std::string& key) const {
    if (kind_ != Kind::Object) return null_value();
    if (std::find(looked_up_.begin(), looked_up_.end(), key) == looked_up_.end())
        looked_up_.push_back(key);
    auto it = obj_.find(key);
    return it == obj_.end() ? null_value() : it->second;
}

void JValue::read(const std::string& key, bool& out) const {
    const JValue& v = at(key);
    if (v.kind_ == Kind::Bool) out = v.b_;
}

void JValue::read(const std::string& key, std::string& out) const {
    const JValue& v = at(key);
    if (v.kind_ == Kind::String) out = v.str_;
}

void JValue::unused(const std::string& prefix, std::vector<std::string>& out) const {
    if (kind_ != Kind::Object) return;
    for (const auto& kv : obj_) {
        const std::string path = prefix.empty() ? kv.first : prefix + "." + kv.first;
        if (std::find(looked_up_.begin(), looked_up_.end(), kv.first) == looked_up_.end()) {
            out.push_back(path);
        } else {
            kv.second.unused(path, out);
        }
    }
}

// =============================================================== config

namespace {

void read_astro(const JValue& j, AstroPop& a) {
    if (!j.is_object()) return;
    j.read("Ca_tot", a.Ca_tot);
    j.read("IP3_0", a.IP3_0);
    j.read("Kd_IP3_1", a.Kd_IP3_1);
    j.read("Kd_IP3_2", a.Kd_IP3_2);
    j.read("Kd_act", a.Kd_act);
    j.read("Kd_inh", a.Kd_inh);
    j.read("Km_SERCA", a.Km_SERCA);
    j.read("SIC_scale", a.SIC_scale);
    j.read("SIC_th", a.SIC_th);
    j.read("delta_IP3", a.delta_IP3);
    j.read("k_IP3R", a.k_IP3R);
    j.read("rate_IP3R", a.rate_IP3R);
    j.read("rate_L", a.rate_L);
    j.read("rate_SERCA", a.rate_SERCA);
    j.read("ratio_ER_cyt", a.ratio_ER_cyt);
    j.read("tau_IP3", a.tau_IP3);
    j.read("Ca_init", a.Ca_init);
    j.read("h_init", a.h_init);
    j.read("IP3", a.IP3_init);  // alias of IP3_init
    j.read("IP3_init", a.IP3_init);
}

void read_neuron(const JValue& j, NeuronPop& p) {
    if (!j.is_object()) return;
    j.read("C_m", p.C_m);
    j.read("g_L", p.g_L);
    j.read("E_L", p.E_L);
    j.read("V_th", p.V_th);
    j.read("Delta_T", p.Delta_T);
    j.read("a", p.a);
    j.read("b", p.b);
    j.read("tau_w", p.tau_w);
    j.read("V_reset", p.V_reset);
    j.read("V_peak", p.V_peak);
    j.read("t_ref", p.t_ref);
    j.read("E_ex", p.E_ex);
    j.read("E_in", p.E_in);
    j.read("tau_syn_ex", p.tau_syn_ex);
    j.read("tau_syn_in", p.tau_syn_in);
    j.read("I_e", p.I_e);
    j.read("V_m", p.V_m_init);  // the schema names the initial potential V_m
}

void read_drive(const JValue& j, Drive& d) {
    if (!j.is_object()) return;
    j.read("poiss_rate", d.poiss_rate);
    j.read("poiss_weight", d.poiss_weight);
    j.read("gauss_noise_var", d.noise_std);  // historical name; the value is a std
    j.read("gauss_noise_std", d.noise_std);
    j.read("noise_dt", d.noise_dt);
    j.read("independent_noise", d.independent);
}

void read_spread(const JValue& j, Spread& s) {
    if (!j.is_object()) return;
    s.enabled = true;  // an object turns the spread on unless it says otherwise
    j.read("enabled", s.enabled);
    j.read("lower", s.lower);
    j.read("upper", s.upper);
    j.read("var", s.var);
}

}  // namespace

ModelConfig config_from_json(const std::string& text, const std::string& where) {
    const JValue root = JValue::parse(text);
    if (!root.is_object()) throw std::runtime_error("configuration root must be an object: " + where);
    ModelConfig c;
    if (const JValue& n = root.at("N"); n.is_object()) {
        n.read("N_A", c.N_A);
        n.read("N_E", c.N_E);
        n.read("N_I", c.N_I);
    }
    if (const JValue& s = root.at("simulation"); s.is_object()) {
        s.read("dt", c.dt);
        s.read("substeps", c.substeps);
        s.read("pre_sim_time", c.pre_sim_time);
        s.read("sim_time", c.sim_time);
        s.read("seed", c.seed);
        s.read("output_dir", c.output_dir);
        s.read("record_spikes", c.record_spikes);
        s.read("record_astro", c.record_astro);
        s.read("record_neuron", c.record_neuron);
        s.read("record_every", c.record_every);
        s.read("record_astro_max", c.record_astro_max);
        s.read("record_neuron_max", c.record_neuron_max);
    }
    read_astro(root.at("astrocyte"), c.astro);
    read_neuron(root.at("neuron_exc"), c.exc);
    read_neuron(root.at("neuron_inh"), c.inh);
    read_drive(root.at("input_astro"), c.in_astro);
    read_drive(root.at("input_exc"), c.in_exc);
    read_drive(root.at("input_inh"), c.in_inh);
    read_spread(root.at("randomize_astro"), c.rnd_astro);
    read_spread(root.at("randomize_neuron"), c.rnd_neuron);
    if (const JValue& s = root.at("synapse"); s.is_object()) {
        s.read("w_e", c.w_e);
        s.read("w_i", c.w_i);
        s.read("w_n2a", c.w_n2a);
        s.read("w_a2n", c.w_a2n);
        s.read("d_e", c.d_e);
        s.read("d_i", c.d_i);
        s.read("d_a2n", c.d_a2n);
        s.read("sic_interval", c.sic_interval);
        if (const JValue& t = s.at("stp"); t.is_object()) {
            t.read("enabled", c.stp_on);
            t.read("U", c.U);
            t.read("tau_rec", c.tau_rec);
            t.read("tau_fac", c.tau_fac);
        }
    }
    if (const JValue& a = root.at("analysis"); a.is_object()) {
        a.read("enabled", c.analysis);
        a.read("ca_threshold", c.ca_threshold);
        a.read("merge_gap", c.merge_gap);
        a.read("hist_window", c.hist_window);
        a.read("hist_shift", c.hist_shift);
    }
    if (const JValue& k = root.at("connectivity"); k.is_object()) {
        k.read("p_primary", c.p_primary);
        k.read("p_third_if_primary", c.p_third);
        k.read("pool_size", c.pool_size);
        k.read("allow_autapses", c.autapses);
        k.read("unique_third_out", c.unique_third);
        std::string pool = "block";
        k.read("pool_type", pool);
        if (pool == "block") {
            c.pool_random = false;
        } else if (pool == "random") {
            c.pool_random = true;
        } else {
            throw std::runtime_error("unknown pool_type '" + pool +
                                     "' (expected \"block\" or \"random\")");
        }
    }
    for (Drive* d : {&c.in_astro, &c.in_exc, &c.in_inh})
        if (d->noise_dt <= 0.0) d->noise_dt = 10.0 * c.dt;  // noise_generator default
    if (c.substeps < 1) throw std::runtime_error("simulation.substeps must be at least 1");
    if (c.dt <= 0.0) throw std::runtime_error("simulation.dt must be positive");
    if (c.record_every < 1) throw std::runtime_error("simulation.record_every must be at least 1");
    if (c.sic_interval < 1) throw std::runtime_error("synapse.sic_interval must be at least 1");
    if (c.pool_size < 1) throw std::runtime_error("connectivity.pool_size must be at least 1");
    std::vector<std::string> extra;
    root.unused("", extra);
    if (!extra.empty()) {
        std::string msg = "unrecognised keys in " + where + ":";
        for (const auto& k : extra) msg += "\n  " + k;
        throw std::runtime_error(msg);
    }
    return c;
}

int delay_steps(double ms, double dt) {
    const int s = static_cast<int>(ms / dt + 0.5);
    return s < 1 ? 1 : s;
}

// ============================================================== builder

namespace {

// The model's sequential counter stream (CounterRng, rng.hpp:53-143).
class Stream {
public:
    Stream(std::uint64_t seed, std::uint64_t stream) : seed_(seed), stream_(stream) {}
    double uniform() { return uniform_at(seed_, stream_, counter_++); }
    double normal() {
        if (spare_ok_) {
            spare_ok_ = false;
            return spare_;
        }
        double u1;
        do {
            u1 = uniform();
        } while (u1 <= 1e-300);
        const double u2 = uniform();
        const double r = std::sqrt(-2.0 * std::log(u1));
        const double th = kTwoPi * u2;
        spare_ = r * std::sin(th);
        spare_ok_ = true;
        return r * std::cos(th);
    }
    double normal_within(double mean, double sd, double lo, double hi) {
        for (int i = 0; i < 1000; ++i) {
            const double v = mean + sd * normal();
            if (v >= lo && v <= hi) return v;
        }
        return std::min(std::max(mean, lo), hi);
    }

private:
    std::uint64_t seed_, stream_, counter_ = 0;
    bool spare_ok_ = false;
    double spare_ = 0.0;
};

// Per-cell parameter spread: Gaussian with sd = var*|mean|, redrawn until it
// lies in [lower*mean, upper*mean] (bounds swapped for negative means).
double spread(double mean, const Spread& s, Stream& r) {
    if (!s.enabled || s.var <= 0.0) return mean;
    const double lo = mean < 0.0 ? mean * s.upper : mean * s.lower;
    const double hi = mean < 0.0 ? mean * s.lower : mean * s.upper;
    return r.normal_within(mean, s.var * std::abs(mean), lo, hi);
}

void to_csr(std::vector<std::vector<std::uint32_t>>& rows, HostCsr& out) {
    out.row_start.assign(rows.size() + 1, 0);
    std::size_t total = 0;
    for (std::size_t i = 0; i < rows.size(); ++i) {
        out.row_start[i] = static_cast<std::uint32_t>(total);
        total += rows[i].size();
    }
    out.row_start[rows.size()] = static_cast<std::uint32_t>(total);
    out.target.clear();
    out.target.reserve(total);
    for (auto& r : rows) {
        out.target.insert(out.target.end(), r.begin(), r.end());
        std::vector<std::uint32_t>().swap(r);
    }
}

void build_cells(Model& m, Stream& rng) {
    const ModelConfig& c = m.cfg;
    const std::uint32_t NA = c.N_A, N = c.N_E + c.N_I;
    m.Ca_tot.resize(NA);
    m.IP3_0.resize(NA);
    m.tau_IP3.resize(NA);
    m.delta_IP3.resize(NA);
    for (std::uint32_t i = 0; i < NA; ++i) {
        m.Ca_tot[i] = spread(c.astro.Ca_tot, c.rnd_astro, rng);
        m.IP3_0[i] = spread(c.astro.IP3_0, c.rnd_astro, rng);
        m.tau_IP3[i] = spread(c.astro.tau_IP3, c.rnd_astro, rng);
        m.delta_IP3[i] = spread(c.astro.delta_IP3, c.rnd_astro, rng);
    }
    m.V_reset.resize(N);
    m.b.resize(N);
    for (std::uint32_t i = 0; i < N; ++i) {
        const NeuronPop& p = i < c.N_E ? c.exc : c.inh;
        m.V_reset[i] = spread(p.V_reset, c.rnd_neuron, rng);
        m.b[i] = spread(p.b, c.rnd_neuron, rng);
    }
}

}  // namespace

void build_reference(Model& m) {
    const ModelConfig& c = m.cfg;
    Stream rng(c.seed, 0x5EED);
    build_cells(m, rng);

    const std::uint32_t NE = c.N_E, NI = c.N_I, N = NE + NI, NA = c.N_A;
    // Astrocyte pools of each postsynaptic neuron, per population block.
    std::vector<std::vector<std::uint32_t>> pool(N);
    std::vector<std::uint32_t> cand;
    for (int blk = 0; blk < 2; ++blk) {
        const std::uint32_t off = blk ? NE : 0, cnt = blk ? NI : NE;
        for (std::uint32_t l = 0; l < cnt; ++l) {
            auto& p = pool[off + l];
            if (!c.pool_random) {
                const std::uint32_t start =
                    NA == 0 ? 0
                            : static_cast<std::uint32_t>((static_cast<std::uint64_t>(l) * NA) /
                                                         std::max<std::uint32_t>(cnt, 1));
                for (int k = 0; k < c.pool_size; ++k)
                    p.push_back(NA == 0 ? 0 : (start + static_cast<std::uint32_t>(k)) % NA);
            } else {
                cand.resize(NA);
                for (std::uint32_t i = 0; i < NA; ++i) cand[i] = i;
                const int take = std::min<int>(c.pool_size, static_cast<int>(NA));
                for (int k = 0; k < take; ++k) {
                    const std::size_t pick =
                        static_cast<std::size_t>(rng.uniform() *
                                                 static_cast<double>(cand.size() - k)) +
                        static_cast<std::size_t>(k);
                    std::swap(cand[k], cand[std::min(pick, cand.size() - 1)]);
                    p.push_back(cand[k]);
                }
            }
        }
    }
    std::vector<std::vector<std::uint32_t>> exc(NE), ast(NE), a2n(NA), inh(NI);
    std::unordered_set<std::uint64_t> seen;
    for (int blk = 0; blk < 2; ++blk) {
        const std::uint32_t off = blk ? NE : 0, cnt = blk ? NI : NE;
        for (std::uint32_t pre = 0; pre < NE; ++pre) {
            for (std::uint32_t l = 0; l < cnt; ++l) {
                const std::uint32_t post = off + l;
                if (!c.autapses && pre == post) continue;
                if (rng.uniform() >= c.p_primary) continue;
                exc[pre].push_back(post);
                if (NA == 0 || rng.uniform() >= c.p_third) continue;
                const auto& p = pool[post];
                const std::uint32_t a =
                    p[static_cast<std::size_t>(rng.uniform() * static_cast<double>(p.size())) %
                      p.size()];
                ast[pre].push_back(a);
                if (!c.unique_third ||
                    seen.insert((static_cast<std::uint64_t>(a) << 32) | post).second)
                    a2n[a].push_back(post);
            }
        }
    }
    for (std::uint32_t pre = 0; pre < NI; ++pre) {
        const std::uint32_t g = NE + pre;
        for (std::uint32_t post = 0; post < N; ++post) {
            if (!c.autapses && g == post) continue;
            if (rng.uniform() < c.p_primary) inh[pre].push_back(post);
        }
    }
    to_csr(exc, m.exc);
    to_csr(inh, m.inh);
    to_csr(ast, m.n2a);
    to_csr(a2n, m.a2n);
    m.built = true;
}

// Fixed in-degree generator.  For target t (stream t of seed ^ salt): k_in
// presynaptic neurons, draw k at counter 3k, uniform over the other N-1
// neurons (multapses allowed, as NEST's fixed_indegree by default); an
// excitatory source recruits, when the draw at counter 3k+1 is below
// p_third_if_primary, the astrocyte of t's pool picked by counter 3k+2.
// Pools are the block or random pools of the config, the random ones drawn
// from stream N+t.  Rows are emitted in (target, k) order.
constexpr std::uint64_t kGenSalt = 0x6A09E667F3BCC909ULL;

void build_fixed_indegree_host_cells(Model& m) {
    Stream rng(m.cfg.seed, 0x5EED);
    build_cells(m, rng);
}

void build_fixed_indegree_host(Model& m, std::uint32_t k_in) {
    const ModelConfig& c = m.cfg;
    build_fixed_indegree_host_cells(m);
    const std::uint32_t NE = c.N_E, NI = c.N_I, N = NE + NI, NA = c.N_A;
    const std::uint64_t gseed = c.seed ^ kGenSalt;
    const int psz = NA == 0 ? 0 : std::min<int>(c.pool_size, static_cast<int>(NA));
    std::vector<std::uint32_t> src(static_cast<std::size_t>(N) * k_in),
        ast(static_cast<std::size_t>(N) * k_in, 0xFFFFFFFFu);
    std::vector<std::uint32_t> exc_deg(NE + 1, 0), inh_deg(NI + 1, 0), n2a_deg(NE + 1, 0),
        a2n_deg(NA + 1, 0);
    for (std::uint32_t t = 0; t < N; ++t) {
        for (std::uint32_t k = 0; k < k_in; ++k) {
            const double u = uniform_at(gseed, t, 3ull * k);
            std::uint32_t s = static_cast<std::uint32_t>(u * static_cast<double>(N - 1));
            if (s >= N - 1) s = N - 2;
            if (s >= t) ++s;
            const std::size_t e = static_cast<std::size_t>(t) * k_in + k;
            src[e] = s;
            if (s < NE) {
                exc_deg[s + 1]++;
                if (NA > 0 && uniform_at(gseed, t, 3ull * k + 1) < c.p_third) {
                    const double v = uniform_at(gseed, t, 3ull * k + 2);
                    const std::uint32_t pick =
                        std::min<std::uint32_t>(static_cast<std::uint32_t>(v * psz), psz - 1);
                    std::uint32_t a;
                    if (!c.pool_random) {
                        const std::uint32_t start = static_cast<std::uint32_t>(
                            (static_cast<std::uint64_t>(t) * NA) / std::max<std::uint32_t>(N, 1));
                        a = (start + pick) % NA;
                    } else {
                        // pool entry `pick` of t: a uniform draw of stream N+t
                        a = static_cast<std::uint32_t>(uniform_at(gseed, N + t, pick) * NA);
                        if (a >= NA) a = NA - 1;
                    }
                    ast[e] = a;
                    n2a_deg[s + 1]++;
                    a2n_deg[a + 1]++;
                }
            } else {
                inh_deg[s - NE + 1]++;
            }
        }
    }
    auto scan = [](std::vector<std::uint32_t>& v) {
        for (std::size_t i = 1; i < v.size(); ++i) v[i] += v[i - 1];
    };
    scan(exc_deg);
    scan(inh_deg);
    scan(n2a_deg);
    scan(a2n_deg);
    m.exc.row_start = exc_deg;
    m.inh.row_start = inh_deg;
    m.n2a.row_start = n2a_deg;
    m.a2n.row_start = a2n_deg;
    m.exc.target.assign(exc_deg.back(), 0);
    m.inh.target.assign(inh_deg.back(), 0);
    m.n2a.target.assign(n2a_deg.back(), 0);
    m.a2n.target.assign(a2n_deg.back(), 0);
    std::vector<std::uint32_t> fe(exc_deg.begin(), exc_deg.end() - 1),
        fi(inh_deg.begin(), inh_deg.end() - 1), fn(n2a_deg.begin(), n2a_deg.end() - 1),
        fa(a2n_deg.begin(), a2n_deg.end() - 1);
    for (std::uint32_t t = 0; t < N; ++t) {
        for (std::uint32_t k = 0; k < k_in; ++k) {
            const std::size_t e = static_cast<std::size_t>(t) * k_in + k;
            const std::uint32_t s = src[e];
            if (s < NE) {
                m.exc.target[fe[s]++] = t;
                if (ast[e] != 0xFFFFFFFFu) {
                    m.n2a.target[fn[s]++] = ast[e];
                    m.a2n.target[fa[ast[e]]++] = t;
                }
            } else {
                m.inh.target[fi[s - NE]++] = t;
            }
        }
    }
    m.built = true;
}

void fill_desc(const Model& m, asg_network_desc& d) {
    const ModelConfig& c = m.cfg;
    std::memset(&d, 0, sizeof d);
    d.n_exc = c.N_E;
    d.n_inh = c.N_I;
    d.n_astro = c.N_A;
    d.dt = c.dt;
    d.substeps = c.substeps;
    d.seed = c.seed;
    d.sic_interval = c.sic_interval;
    d.d_e_steps = delay_steps(c.d_e, c.dt);
    d.d_i_steps = delay_steps(c.d_i, c.dt);
    d.d_a2n_steps = delay_steps(c.d_a2n, c.dt);
    d.w_e = c.w_e;
    d.w_i = c.w_i;
    d.w_n2a = c.w_n2a;
    d.w_a2n = c.w_a2n;
    auto pop = [](const NeuronPop& p, asg_neuron_params& o) {
        o.C_m = p.C_m; o.g_L = p.g_L; o.E_L = p.E_L; o.V_th = p.V_th; o.Delta_T = p.Delta_T;
        o.a = p.a; o.tau_w = p.tau_w; o.V_peak = p.V_peak; o.t_ref = p.t_ref; o.E_ex = p.E_ex;
        o.E_in = p.E_in; o.tau_syn_ex = p.tau_syn_ex; o.tau_syn_in = p.tau_syn_in; o.I_e = p.I_e;
    };
    pop(c.exc, d.exc);
    pop(c.inh, d.inh);
    const AstroPop& a = c.astro;
    d.astro = asg_astro_params{a.Kd_IP3_1, a.Kd_IP3_2, a.Kd_act, a.Kd_inh, a.Km_SERCA, a.k_IP3R,
                               a.rate_IP3R, a.rate_L, a.rate_SERCA, a.ratio_ER_cyt, a.SIC_scale,
                               a.SIC_th};
    auto drive = [](const Drive& s, asg_input& o) {
        o.poiss_rate = s.poiss_rate;
        o.poiss_weight = s.poiss_weight;
        o.gauss_noise_std = s.noise_std;
        o.noise_dt = s.noise_dt;
        o.independent_noise = s.independent ? 1 : 0;
    };
    drive(c.in_exc, d.input_exc);
    drive(c.in_inh, d.input_inh);
    drive(c.in_astro, d.input_astro);
    d.stp = asg_stp{c.stp_on ? 1 : 0, c.U, c.tau_rec, c.tau_fac};
    auto csr = [](const HostCsr& h, std::uint32_t n, asg_csr& o) {
        o.n_sources = n;
        o.row_start = h.row_start.empty() ? nullptr : h.row_start.data();
        o.target = h.target.data();
    };
    csr(m.exc, c.N_E, d.exc_primary);
    csr(m.inh, c.N_I, d.inh_primary);
    csr(m.n2a, c.N_E, d.neuron_astro);
    csr(m.a2n, c.N_A, d.astro_neuron);
    d.V_reset = m.V_reset.data();
    d.b = m.b.data();
    d.Ca_tot = m.Ca_tot.data();
    d.IP3_0 = m.IP3_0.data();
    d.tau_IP3 = m.tau_IP3.data();
    d.delta_IP3 = m.delta_IP3.data();
    d.Ca_tot_u = a.Ca_tot;
    d.IP3_0_u = a.IP3_0;
    d.tau_IP3_u = a.tau_IP3;
    d.delta_IP3_u = a.delta_IP3;
    d.V_m_init_exc = c.exc.V_m_init;
    d.V_m_init_inh = c.inh.V_m_init;
    d.Ca_init = a.Ca_init;
    d.IP3_init = a.IP3_init;
    d.h_init = a.h_init;
}

}  // namespace asg

// ================================================================ C ABI

using asg::Model;

extern "C" {

static int model_from_text(const std::string& text, const std::string& where, int64_t seed,
                           double sim_time, double pre_time, int64_t n_astro, asg_model** out) {
    if (out == nullptr) return asg::fail(ASG_ERR_ARG, "out is NULL");
    *out = nullptr;
    try {
        auto* m = new Model;
        m->cfg = asg::config_from_json(text, where);
        if (seed >= 0) m->cfg.seed = static_cast<std::uint64_t>(seed);
        if (sim_time >= 0.0) m->cfg.sim_time = sim_time;
        if (pre_time >= 0.0) m->cfg.pre_sim_time = pre_time;
        if (n_astro >= 0) m->cfg.N_A = static_cast<std::uint32_t>(n_astro);
        *out = reinterpret_cast<asg_model*>(m);
        return ASG_OK;
    } catch (const std::exception& e) {
        return asg::fail(ASG_ERR_CONFIG, "%s", e.what());
    }
}

int asg_model_from_json(const char* json_text, int64_t seed, double sim_time, double pre_time,
                        int64_t n_astro, asg_model** out) {
    asg::clear_error();
    if (json_text == nullptr) return asg::fail(ASG_ERR_ARG, "json_text is NULL");
    return model_from_text(json_text, "<text>", seed, sim_time, pre_time, n_astro, out);
}

int asg_model_from_file(const char* path, int64_t seed, double sim_time, double pre_time,
                        int64_t n_astro, asg_model** out) {
    asg::clear_error();
    if (path == nullptr) return asg::fail(ASG_ERR_ARG, "path is NULL");
    std::ifstream in(path);
    if (!in) return asg::fail(ASG_ERR_CONFIG, "cannot open configuration file: %s", path);
    std::ostringstream buf;
    buf << in.rdbuf();
    return model_from_text(buf.str(), path, seed, sim_time, pre_time, n_astro, out);
}

int asg_model_build(asg_model* mp) {
    asg::clear_error();
    if (mp == nullptr) return asg::fail(ASG_ERR_ARG, "model is NULL");
    try {
        asg::build_reference(*reinterpret_cast<Model*>(mp));
    } catch (const std::exception& e) {
        return asg::fail(ASG_ERR_OOM, "build failed: %s", e.what());
    }
    return ASG_OK;
}

int asg_model_build_fixed_indegree(asg_model* mp, uint32_t k_in, int32_t device) {
    asg::clear_error();
    if (mp == nullptr) return asg::fail(ASG_ERR_ARG, "model is NULL");
    Model& m = *reinterpret_cast<Model*>(mp);
    const std::uint32_t N = m.cfg.N_E + m.cfg.N_I;
    if (N < 2) return asg::fail(ASG_ERR_ARG, "fixed in-degree needs at least two neurons");
    try {
        if (device >= 0) return asg::build_fixed_indegree_device(m, k_in, device);
        asg::build_fixed_indegree_host(m, k_in);
    } catch (const std::exception& e) {
        return asg::fail(ASG_ERR_OOM, "build failed: %s", e.what());
    }
    return ASG_OK;
}

int asg_model_desc(asg_model* mp, asg_network_desc* out) {
    asg::clear_error();
    if (mp == nullptr || out == nullptr) return asg::fail(ASG_ERR_ARG, "NULL argument");
    Model& m = *reinterpret_cast<Model*>(mp);
    if (!m.built) return asg::fail(ASG_ERR_STATE, "model is not built");
    asg::fill_desc(m, *out);
    return ASG_OK;
}

int asg_model_record_opts(asg_model* mp, asg_record_opts* out) {
    asg::clear_error();
    if (mp == nullptr || out == nullptr) return asg::fail(ASG_ERR_ARG, "NULL argument");
    const asg::ModelConfig& c = reinterpret_cast<Model*>(mp)->cfg;
    out->record_from_step = c.pre_steps();
    out->record_every = c.record_every;
    out->spikes = c.record_spikes ? 1 : 0;
    out->astro_max = c.record_astro ? c.record_astro_max : 0;
    out->neuron_max = c.record_neuron ? c.record_neuron_max : 0;
    return ASG_OK;
}

int asg_model_scalars(asg_model* mp, double* o) {
    asg::clear_error();
    if (mp == nullptr || o == nullptr) return asg::fail(ASG_ERR_ARG, "NULL argument");
    const asg::ModelConfig& c = reinterpret_cast<Model*>(mp)->cfg;
    o[0] = c.dt;
    o[1] = c.substeps;
    o[2] = static_cast<double>(c.seed);
    o[3] = static_cast<double>(c.pre_steps());
    o[4] = static_cast<double>(c.sim_steps());
    o[5] = c.record_every;
    o[6] = c.pre_sim_time;
    o[7] = c.sim_time;
    o[8] = c.ca_threshold >= 0.0 ? c.ca_threshold : c.astro.SIC_th;
    o[9] = c.merge_gap;
    o[10] = c.hist_window;
    o[11] = c.hist_shift;
    return ASG_OK;
}

int asg_model_stats(asg_model* mp, int64_t* o) {
    asg::clear_error();
    if (mp == nullptr || o == nullptr) return asg::fail(ASG_ERR_ARG, "NULL argument");
    const Model& m = *reinterpret_cast<Model*>(mp);
    const asg::ModelConfig& c = m.cfg;
    o[0] = static_cast<int64_t>(m.exc.target.size());
    o[1] = static_cast<int64_t>(m.inh.target.size());
    o[2] = static_cast<int64_t>(m.n2a.target.size());
    o[3] = static_cast<int64_t>(m.a2n.target.size());
    o[4] = std::max({1, asg::delay_steps(c.d_e, c.dt), asg::delay_steps(c.d_i, c.dt),
                     asg::delay_steps(c.d_a2n, c.dt)}) + 1;
    return ASG_OK;
}

int asg_model_free(asg_model* mp) {
    asg::clear_error();
    delete reinterpret_cast<Model*>(mp);
    return ASG_OK;
}

}  // extern "C"
