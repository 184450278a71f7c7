// Host side of the network engine: one Engine holds any number of resident
// network instances (a plain run is an engine with one instance, a sweep is
// a batch, serving adds and removes instances at step boundaries) and
// advances them together, one fused kernel launch per step, K steps per
// captured CUDA graph ("chunk").
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "asg_b200.h"
#include "asg_common.hpp"
#include "asg_engine.cuh"

namespace asg {

struct SpikeRec {
    std::int64_t step;
    std::uint32_t source;
};

// One resident instance.
struct Instance {
    int id = -1;
    InstDev dev{};             // host copy of the device descriptor
    DevBuf arena;              // every device array of the instance
    std::size_t arena_bytes = 0;
    std::int64_t step = 0;     // next step to run
    std::int64_t end = INT64_MAX;
    bool done() const { return step >= end; }
    // outputs gathered on the host
    std::vector<SpikeRec> spikes;
    std::vector<std::int64_t> astro_rec_steps, neuron_rec_steps;
    std::vector<double> rec_Ca, rec_IP3, rec_V, rec_Isic;
    std::int64_t spike_edges = 0, sic_edges = 0, n_spikes = 0;
    // mapped host buffers for logs and record rows, two per parity
    unsigned long long* log_h[2] = {nullptr, nullptr};
    unsigned long long* log_d[2] = {nullptr, nullptr};
    double* rec_h[2] = {nullptr, nullptr};  // Ca | IP3 | V | Isic rows
    double* rec_d[2] = {nullptr, nullptr};
    std::uint32_t log_cap = 0;
    std::uint32_t rec_rows = 0;
    std::int64_t chunk_first[2] = {0, 0};   // first step of the chunk written to parity p
    std::int64_t chunk_last[2] = {0, 0};
    bool keep_spikes = true;
    int max_chunk = 0;  // longest chunk the output buffers were sized for
    ~Instance();
};

struct EngineConfig {
    int device = 0;
    int chunk_steps = 32;
    int block = 128;
    int use_graphs = 1;  // 1 graphs of per-step launches, -1 plain launches, 2 persistent
    int sic_mode = 0;  // 0 auto, 1 fused, 2 split
    bool pdl = true;   // programmatic dependent launch between steps
    int push_mode = 0; // 0 deferred push when delays allow, 1 always in the spiking block
    std::uint64_t mem_budget = 0;
    int occupancy = 0;  // 0 auto, 1 latency form, 2 high-occupancy form of the step kernel
    bool large_total = false;  // the engine will hold 2^16+ neurons in all (auto SIC form)
    bool astro_fp32 = false;   // precision study: astrocyte update in FP32
    bool item_loop = true;     // high-occupancy form: one wave, several items per block
};

class Engine {
public:
    explicit Engine(const EngineConfig& cfg);
    ~Engine();
    int init();

    // Adds an instance from a descriptor; it runs steps [first, end).
    // add = prepare + commit.
    int add(const asg_network_desc& d, const asg_record_opts* rec, std::int64_t first,
            std::int64_t end, bool keep_spikes, int* id);
    // Validates the descriptor, builds the instance's tables and uploads its
    // arena on the upload stream.  Uses nothing the chunks in flight use, so
    // it may run on another host thread while run_chunk steps (one prepare
    // at a time).  check_budget: refuse beyond cfg.mem_budget (a caller that
    // accounts for memory itself passes false).
    int prepare(const asg_network_desc& d, const asg_record_opts* rec, std::int64_t first,
                std::int64_t end, bool keep_spikes, bool check_budget,
                std::unique_ptr<Instance>* out);
    // Joins a prepared instance at this chunk boundary (same thread as run).
    int commit(std::unique_ptr<Instance> inst, int* id);
    int remove(int id);
    Instance* find(int id);
    // Bytes an instance of this descriptor would hold on the device.
    static int footprint(const asg_network_desc& d, int chunk_steps, std::uint64_t* bytes);

    // Runs chunks until every instance advanced by n_steps (or reached its
    // end).  Outputs are gathered into each Instance.  A call runs as equal
    // chunks of at most chunk_steps (1000 steps at chunk 512: two of 500),
    // each one captured graph.
    int run(std::int64_t n_steps);
    // One chunk of up to chunk_steps (serving loop granularity).
    int run_chunk(std::int64_t max_steps);

    // Waits for every chunk in flight and gathers its outputs.
    int flush() { return finish_pending(); }

    int pull_state(int id, asg_state* out);
    int pull_stp(int id, double* x, double* u, double* t);

    EngineConfig cfg;
    std::vector<std::unique_ptr<Instance>> insts;
    double last_ms = 0.0;
    std::int64_t last_kernels = 0;
    double total_ms = 0.0;
    std::int64_t total_kernels = 0;
    std::int64_t chunks = 0;
    double chunk_device_ms = 0.0;  // sum over collected chunks (serving)
    std::int64_t launched_kernels = 0;
    std::uint64_t resident_bytes = 0;
    cudaStream_t stream = nullptr;
    int sms = 148;

    // The next chunk first recomputes the SIC values of the arrival steps
    // step .. step+lead-1 (after a restore: the ring may come from another
    // launch mode).
    void mark_side_prime() { side_prime = true; }

    int set_block(int block);
    int set_chunk(int chunk);
    int set_mode(int use_graphs);

private:
    int rebuild();          // work table + graph after the instance set changed
    cudaError_t issue_steps(int steps);  // step launches + side-stream SIC batches
    int launch_chunk(int parity, int steps);
    int collect(int parity);
    int finish_pending();

    DevBuf d_insts, d_work;
    InstDev* h_insts[2] = {nullptr, nullptr};  // pinned staging
    unsigned long long* h_stats[2] = {nullptr, nullptr};  // pinned: per inst log_n + counters
    DevBuf d_stats;        // [n][8]: log_n, spike_edges, sic_edges, spikes, overflow
    DevBuf d_barrier;      // GridBarrier of the persistent chunk kernel
    unsigned* h_barrier_err[2] = {nullptr, nullptr};  // pinned copy of its error word
    int persistent_grid = 0;
    std::size_t cap_insts = 0;
    std::vector<Work> work;
    std::vector<int> order;  // instance index per device slot
    // Captured chunk graphs by length, most recently used first: the
    // chunk_steps graph and the lengths run() splits its calls into.
    static constexpr std::size_t kMaxGraphs = 4;
    std::vector<std::pair<int, cudaGraphExec_t>> graphs;
    bool graph_mode() const { return cfg.use_graphs == 0 || cfg.use_graphs == 1; }
    bool wide = false;  // launches use the high-occupancy form of the step kernel
    int wide_grid = 0;  // its grid: one wave of resident blocks (0: one block per item)
    cudaGraphExec_t find_graph(int steps);
    int capture_graph(int steps);
    void drop_graphs();
    bool dirty = true;
    // side-stream SIC batches (instances with InstDev::sic_side)
    static constexpr int kSideEvents = 8;
    cudaStream_t side = nullptr;
    cudaStream_t upload = nullptr;  // table uploads of add(), beside the chunks in flight
    std::vector<Work> side_work;
    DevBuf d_side_work;
    int side_lead = 0, side_lead_max = 0;
    bool side_prime = true;
    cudaError_t prime_side();
    cudaEvent_t ev_side_fork = nullptr, ev_side_join = nullptr;
    cudaEvent_t ev_side_pre[kSideEvents] = {}, ev_side_done[kSideEvents] = {};
    cudaEvent_t ev_start = nullptr, ev_end = nullptr;
    cudaEvent_t ev_chunk[2] = {nullptr, nullptr};
    cudaEvent_t ev_chunk0[2] = {nullptr, nullptr};
    bool pending[2] = {false, false};
    std::size_t launched_insts[2] = {0, 0};
    int next_parity = 0;
    int next_id = 0;
};

}  // namespace asg
