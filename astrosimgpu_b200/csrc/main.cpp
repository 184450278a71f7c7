// astrosim_b200: command-line driver over the C ABI (include/asg_b200.h).
//
// Same options, outputs and summary as the reference CLI (main.cpp:26-41,
// 76-161, 165-329): build the network from a JSON config, run the recorded
// window on the B200, write spikes.csv / astrocytes.csv / neurons.csv with
// default 6-significant-digit formatting, read the calcium traces back and
// run the transient analysis, and write run.txt with a phase table and the
// backend line "B200 native (sm_100a, FP64)".

#include <chrono>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "asg_b200.h"

namespace {

void usage(const char* argv0) {
    std::cout << "Usage: " << argv0 << " [options]\n\n"
              << "Runs the neuron-astrocyte model of a JSON parameter file with every\n"
              << "timestep on one B200 GPU, writes the spike and trace files, and prints\n"
              << "the firing and astrocyte-calcium summary.\n\n"
              << "Options:\n"
              << "  -c, --config PATH     parameter file (JSON)   [config/use_case.json]\n"
              << "  -o, --output DIR      output directory        [from config]\n"
              << "  -s, --seed N          random seed             [from config]\n"
              << "  -t, --sim-time MS     recorded duration       [from config]\n"
              << "  -p, --pre-time MS     discarded transient     [from config]\n"
              << "  -a, --astrocytes N    override the astrocyte count [from config]\n"
              << "      --chunk N         steps per captured CUDA graph [by network size]\n"
              << "      --astro-fp32      astrocyte update in FP32 (precision study) [FP64]\n"
              << "      --no-analysis     skip the post-run summary\n"
              << "  -h, --help            show this message\n";
}

bool ok(int st, const char* what) {
    if (st != ASG_OK) {
        std::cerr << "error: " << what << ": " << asg_last_error() << "\n";
        return false;
    }
    return true;
}

}  // namespace

int main(int argc, char** argv) {
    std::string config = "config/use_case.json", out_override;
    long long seed = -1, astro = -1;
    double sim = -1.0, pre = -1.0;
    bool analysis = true;
    int chunk = 0;  // 0: the engine's default for the network size
    bool astro_fp32 = false;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&]() -> std::string {
            if (i + 1 >= argc) {
                std::cerr << "missing value for " << a << "\n";
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "-h" || a == "--help") {
            usage(argv[0]);
            return 0;
        } else if (a == "-c" || a == "--config") {
            config = next();
        } else if (a == "-o" || a == "--output") {
            out_override = next();
        } else if (a == "-s" || a == "--seed") {
            seed = std::stoll(next());
        } else if (a == "-t" || a == "--sim-time") {
            sim = std::stod(next());
        } else if (a == "-p" || a == "--pre-time") {
            pre = std::stod(next());
        } else if (a == "-a" || a == "--astrocytes") {
            astro = std::stoll(next());
        } else if (a == "--chunk") {
            chunk = std::stoi(next());
        } else if (a == "--astro-fp32") {
            astro_fp32 = true;
        } else if (a == "--no-analysis") {
            analysis = false;
        } else {
            std::cerr << "unknown option: " << a << "\n\n";
            usage(argv[0]);
            return 2;
        }
    }

    asg_model* model = nullptr;
    if (!ok(asg_model_from_file(config.c_str(), seed, sim, pre, astro, &model), "config")) return 1;
    std::cout << "Building network from " << config << " ...\n";
    if (!ok(asg_model_build(model), "build")) return 1;
    asg_network_desc desc;
    asg_record_opts rec;
    double sc[12];
    int64_t st5[5];
    asg_model_desc(model, &desc);
    asg_model_record_opts(model, &rec);
    asg_model_scalars(model, sc);
    asg_model_stats(model, st5);
    const double dt = sc[0];
    const int64_t pre_steps = static_cast<int64_t>(sc[3]), sim_steps = static_cast<int64_t>(sc[4]);
    const uint32_t N = desc.n_exc + desc.n_inh, NA = desc.n_astro;
    std::cout << "  " << NA << " astrocytes, " << desc.n_exc << " excitatory, " << desc.n_inh
              << " inhibitory neurons\n  " << st5[0] + st5[1] << " neuron-neuron synapses, "
              << st5[2] << " neuron-astrocyte, " << st5[3] << " astrocyte-neuron\n";

    // Output directory from the config's simulation.output_dir unless overridden.
    std::string out_dir = out_override;
    if (out_dir.empty()) {
        std::ifstream in(config);
        std::stringstream ss;
        ss << in.rdbuf();
        const std::string text = ss.str();
        const auto k = text.find("\"output_dir\"");
        out_dir = "results";
        if (k != std::string::npos) {
            const auto q1 = text.find('"', text.find(':', k) + 1);
            const auto q2 = text.find('"', q1 + 1);
            if (q1 != std::string::npos && q2 != std::string::npos) out_dir = text.substr(q1 + 1, q2 - q1 - 1);
        }
    }
    std::error_code ec;
    std::filesystem::create_directories(out_dir, ec);
    std::ofstream spikes_csv, astro_csv, neuron_csv;
    if (rec.spikes) {
        spikes_csv.open(out_dir + "/spikes.csv");
        spikes_csv << "time_ms,neuron\n";
    }
    if (rec.astro_max) {
        astro_csv.open(out_dir + "/astrocytes.csv");
        astro_csv << "time_ms,astrocyte,Ca,IP3\n";
    }
    if (rec.neuron_max) {
        neuron_csv.open(out_dir + "/neurons.csv");
        neuron_csv << "time_ms,neuron,V_m,I_SIC\n";
    }

    asg_engine_opts opts;
    std::memset(&opts, 0, sizeof opts);
    opts.chunk_steps = chunk;
    opts.astro_precision = astro_fp32 ? 32 : 64;
    asg_network* net = nullptr;
    if (!ok(asg_create(&desc, &rec, &opts, &net), "create")) return 1;
    std::cout << "Simulating " << sc[6] << " ms transient + " << sc[7] << " ms recorded ...\n";

    const auto t0 = std::chrono::steady_clock::now();
    if (!ok(asg_step(net, pre_steps), "transient")) return 1;
    double dev_ms_transient = 0.0;
    asg_last_timing(net, &dev_ms_transient, nullptr);
    const auto t_rec = std::chrono::steady_clock::now();
    double dev_ms = 0.0;
    int64_t kernels = 0, spikes_recorded = 0;
    const uint32_t am = std::min(rec.astro_max, NA), nm = std::min(rec.neuron_max, N);
    std::vector<int64_t> sst, ast, nst;
    std::vector<uint32_t> ssrc;
    std::vector<double> ca, ip3, v, isic;
    const int64_t block = 20000;
    for (int64_t done = 0; done < sim_steps; done += block) {
        const int64_t n = std::min(block, sim_steps - done);
        if (!ok(asg_step(net, n), "step")) return 1;
        double ms = 0.0;
        int64_t k = 0;
        asg_last_timing(net, &ms, &k);
        dev_ms += ms;
        kernels += k;
        int64_t cnt = 0, ar = 0, nr = 0;
        asg_fetch_spikes(net, nullptr, nullptr, 0, &cnt);
        sst.resize(cnt);
        ssrc.resize(cnt);
        if (!ok(asg_fetch_spikes(net, sst.data(), ssrc.data(), cnt, &cnt), "spikes")) return 1;
        for (int64_t i = 0; i < cnt; ++i) {
            if (sst[i] < pre_steps) continue;
            spikes_csv << static_cast<double>(sst[i]) * dt << ',' << ssrc[i] << '\n';
            ++spikes_recorded;
        }
        asg_fetch_record(net, nullptr, nullptr, nullptr, 0, &ar, nullptr, nullptr, nullptr, 0, &nr);
        ast.resize(ar);
        ca.resize(ar * am);
        ip3.resize(ar * am);
        nst.resize(nr);
        v.resize(nr * nm);
        isic.resize(nr * nm);
        if (!ok(asg_fetch_record(net, ast.data(), ca.data(), ip3.data(), ar, &ar, nst.data(),
                                 v.data(), isic.data(), nr, &nr),
                "record"))
            return 1;
        for (int64_t r = 0; r < ar; ++r)
            for (uint32_t a = 0; a < am; ++a)
                astro_csv << static_cast<double>(ast[r]) * dt << ',' << a << ',' << ca[r * am + a]
                          << ',' << ip3[r * am + a] << '\n';
        for (int64_t r = 0; r < nr; ++r)
            for (uint32_t i = 0; i < nm; ++i)
                neuron_csv << static_cast<double>(nst[r]) * dt << ',' << i << ',' << v[r * nm + i]
                           << ',' << isic[r * nm + i] << '\n';
    }
    const auto t1 = std::chrono::steady_clock::now();
    const double wall = std::chrono::duration<double>(t1 - t0).count();
    const double rec_wall = std::chrono::duration<double>(t1 - t_rec).count();
    int64_t spike_edges = 0, sic_edges = 0, n_spikes = 0;
    asg_counters(net, &spike_edges, &sic_edges, &n_spikes);
    asg_destroy(net);
    astro_csv.close();
    spikes_csv.close();
    neuron_csv.close();

    std::string analysis_text;
    if (analysis && am > 0) {
        // Read the traces back from the CSV, as the reference does
        // (main.cpp:46-74): the analysis sees 6-significant-digit values.
        std::map<uint32_t, std::vector<double>> times, calcium;
        std::ifstream in(out_dir + "/astrocytes.csv");
        std::string line;
        std::getline(in, line);
        while (std::getline(in, line)) {
            std::istringstream ls(line);
            std::string f;
            if (!std::getline(ls, f, ',')) continue;
            const double t = std::strtod(f.c_str(), nullptr);
            if (!std::getline(ls, f, ',')) continue;
            const uint32_t cell = static_cast<uint32_t>(std::strtoul(f.c_str(), nullptr, 10));
            if (!std::getline(ls, f, ',')) continue;
            times[cell].push_back(t);
            calcium[cell].push_back(std::strtod(f.c_str(), nullptr));
        }
        std::size_t ns = 0;
        for (auto& kv : times) ns = std::max(ns, kv.second.size());
        std::vector<double> T, Cv;
        for (auto& kv : calcium) {
            auto tt = times[kv.first];
            tt.resize(ns, tt.empty() ? 0.0 : tt.back());
            auto cc = kv.second;
            cc.resize(ns, cc.empty() ? 0.0 : cc.back());
            T.insert(T.end(), tt.begin(), tt.end());
            Cv.insert(Cv.end(), cc.begin(), cc.end());
        }
        double width = sc[10], shift = sc[11];
        if (width >= sc[7] && sc[7] > 0.0) {
            width = sc[7] / 10.0;
            shift = width / 5.0;
        }
        double o[5] = {0, 0, 0, 0, 0};
        asg_calcium_analysis(T.data(), Cv.data(), static_cast<int32_t>(calcium.size()),
                             static_cast<int32_t>(ns), sc[8], sc[9], sc[6], sc[6] + sc[7], width,
                             shift, o);
        std::ostringstream os;
        os << std::fixed << std::setprecision(4);
        os << "Calcium analysis (threshold " << sc[8] << " uM, window " << width << "/" << shift
           << " ms)\n-----------------------------------\n";
        os << "astrocytes with transients  " << static_cast<long long>(o[0]) << " / "
           << calcium.size() << "\n";
        os << "transients detected         " << static_cast<long long>(o[1]) << "\n";
        os << "mean duration               " << o[2] << " ms\n";
        os << "pairs correlated            " << static_cast<long long>(o[3]) << "\n";
        os << "mean pairwise correlation   " << o[4] << "\n";
        analysis_text = os.str();
    }

    std::ostringstream os;
    os << std::fixed << std::setprecision(4);
    os << "Tripartite neuron-astrocyte network\n-----------------------------------\n";
    os << "astrocytes            " << NA << "\n";
    os << "excitatory neurons    " << desc.n_exc << "\n";
    os << "inhibitory neurons    " << desc.n_inh << "\n";
    os << "exc -> neuron synapses " << st5[0] << "\n";
    os << "inh -> neuron synapses " << st5[1] << "\n";
    os << "neuron -> astrocyte    " << st5[2] << "\n";
    os << "astrocyte -> neuron    " << st5[3] << "\n\n";
    os << "dt                    " << dt << " ms (" << desc.substeps << " substeps)\n";
    os << "astrocyte backend     B200 native (sm_100a, "
       << (astro_fp32 ? "FP64 neurons, FP32 astrocytes: precision study" : "FP64")
       << "), whole step on the GPU\n";
    os << "transient             " << sc[6] << " ms\n";
    os << "recorded              " << sc[7] << " ms\n";
    os << "seed                  " << static_cast<unsigned long long>(sc[2]) << "\n\n";
    os << "wall clock            " << wall << " s\n";
    os << "spikes recorded       " << spikes_recorded << "\n";
    if (sc[7] > 0.0 && N > 0)
        os << "mean firing rate      "
           << static_cast<double>(spikes_recorded) * 1000.0 / (sc[7] * static_cast<double>(N))
           << " Hz\n";
    os << "\nState propagation (recorded window)\n-----------------------------------\n";
    os << "device time           " << dev_ms * 1e-3 << " s (" << kernels << " step launches)\n";
    os << "host wall             " << rec_wall << " s (incl. CSV output)\n";
    if (sim_steps > 0) {
        os << "device us per step    " << dev_ms * 1e3 / static_cast<double>(sim_steps) << "\n";
        os << "real-time factor      " << (dev_ms * 1e-3) / (sc[7] * 1e-3) << "\n";
        os << "neuron-updates/s      " << std::scientific << std::setprecision(3)
           << static_cast<double>(N) * sim_steps / (dev_ms * 1e-3) << "\n";
        os << "synaptic events/s     " << static_cast<double>(spike_edges + sic_edges) / ((dev_ms + dev_ms_transient) * 1e-3)
           << std::fixed << std::setprecision(4) << "\n";
    }
    if (!analysis_text.empty()) os << "\n" << analysis_text;
    std::ofstream(out_dir + "/run.txt") << os.str();
    std::cout << "\n" << os.str() << "\nOutput written to " << out_dir << "/\n";
    asg_model_free(model);
    return 0;
}
