// C ABI of the network engine: the single-network handle (asg_*) and the
// batched sweep (asg_batch_*).  Both are thin shells over asg::Engine; a
// plain network is an engine holding one instance.

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "asg_engine.hpp"

namespace asg {

EngineConfig config_from(const asg_engine_opts* o) {
    EngineConfig c;
    if (o != nullptr) {
        c.device = o->device;
        if (o->chunk_steps > 0) c.chunk_steps = o->chunk_steps;
        if (o->block > 0) c.block = o->block;
        if (o->use_graphs != 0) c.use_graphs = o->use_graphs;  // -1 plain, 2 persistent
        c.sic_mode = o->sic_mode;
        c.pdl = o->pdl >= 0;
        c.push_mode = o->push_mode;
        c.mem_budget = o->mem_budget;
        c.occupancy = o->occupancy;
        c.astro_fp32 = o->astro_precision == 32;
    }
    return c;
}

// Default chunk of a single network: about 2^23 neuron-steps per chunk, a
// power of two in [32, 512].  Longer chunks cost fewer chunk boundaries (a
// descriptor copy, a counter copy and reset, a graph launch and a first step
// without early launch: ~20 us of device time each), while the per-chunk
// spike log (N * chunk / 8 entries, two pinned buffers) stays at most 8 MB.
int default_chunk(std::uint64_t n_neurons) {
    const std::uint64_t want = (1ull << 23) / std::max<std::uint64_t>(n_neurons, 1);
    int c = 32;
    while (c < 512 && static_cast<std::uint64_t>(c) * 2 <= want) c *= 2;
    return c;
}

namespace {

int fetch_spikes_from(Instance* I, int64_t* steps, uint32_t* sources, int64_t cap,
                      int64_t* count) {
    const int64_t n = static_cast<int64_t>(I->spikes.size());
    if (count) *count = n;
    if (steps == nullptr && sources == nullptr) return ASG_OK;  // size query
    if (n > cap) return fail(ASG_ERR_OVERFLOW, "%lld spikes pending, buffer holds %lld",
                             static_cast<long long>(n), static_cast<long long>(cap));
    for (int64_t i = 0; i < n; ++i) {
        if (steps) steps[i] = I->spikes[i].step;
        if (sources) sources[i] = I->spikes[i].source;
    }
    I->spikes.clear();
    return ASG_OK;
}

int fetch_record_from(Instance* I, int64_t* astro_steps, double* Ca, double* IP3,
                      int64_t astro_cap, int64_t* astro_rows, int64_t* neuron_steps, double* V,
                      double* Isic, int64_t neuron_cap, int64_t* neuron_rows) {
    const int64_t na = static_cast<int64_t>(I->astro_rec_steps.size());
    const int64_t nn = static_cast<int64_t>(I->neuron_rec_steps.size());
    if (astro_rows) *astro_rows = na;
    if (neuron_rows) *neuron_rows = nn;
    const bool want_a = astro_steps || Ca || IP3;
    const bool want_n = neuron_steps || V || Isic;
    if (want_a && na > astro_cap)
        return fail(ASG_ERR_OVERFLOW, "%lld astrocyte rows pending, buffer holds %lld",
                    static_cast<long long>(na), static_cast<long long>(astro_cap));
    if (want_n && nn > neuron_cap)
        return fail(ASG_ERR_OVERFLOW, "%lld neuron rows pending, buffer holds %lld",
                    static_cast<long long>(nn), static_cast<long long>(neuron_cap));
    if (want_a) {
        if (astro_steps) std::copy(I->astro_rec_steps.begin(), I->astro_rec_steps.end(), astro_steps);
        if (Ca) std::copy(I->rec_Ca.begin(), I->rec_Ca.end(), Ca);
        if (IP3) std::copy(I->rec_IP3.begin(), I->rec_IP3.end(), IP3);
        I->astro_rec_steps.clear();
        I->rec_Ca.clear();
        I->rec_IP3.clear();
    }
    if (want_n) {
        if (neuron_steps) std::copy(I->neuron_rec_steps.begin(), I->neuron_rec_steps.end(), neuron_steps);
        if (V) std::copy(I->rec_V.begin(), I->rec_V.end(), V);
        if (Isic) std::copy(I->rec_Isic.begin(), I->rec_Isic.end(), Isic);
        I->neuron_rec_steps.clear();
        I->rec_V.clear();
        I->rec_Isic.clear();
    }
    return ASG_OK;
}

}  // namespace

struct NetworkHandle {
    std::unique_ptr<Engine> eng;
    int id = -1;
};

struct BatchHandle {
    std::unique_ptr<Engine> eng;
    std::vector<int> ids;
};

// Times candidate launch shapes on a snapshot of every instance (device
// arena + host bookkeeping restored after each trial, so the simulation is
// not advanced) and keeps the fastest: chunk length x block size x launch
// mode (CUDA graph of per-step launches or the persistent chunk kernel).
int autotune_engine(Engine& e, int32_t steps, asg_engine_opts* chosen) {
    ASG_TRY(e.flush());
    // Snapshot every instance (device arena + host-side bookkeeping).
    struct Snap {
        DevBuf copy;
        int64_t step;
        std::size_t spikes, arows, nrows, ca, ip3, v, isic;
        int64_t se, sic, ns;
    };
    std::vector<Snap> snaps(e.insts.size());
    for (std::size_t i = 0; i < e.insts.size(); ++i) {
        Instance& I = *e.insts[i];
        Snap& s = snaps[i];
        ASG_TRY(s.copy.alloc(I.arena_bytes, false));
        ASG_CUDA(cudaMemcpyAsync(s.copy.get(), I.arena.get(), I.arena_bytes,
                                 cudaMemcpyDeviceToDevice, e.stream));
        s.step = I.step;
        s.spikes = I.spikes.size();
        s.arows = I.astro_rec_steps.size();
        s.nrows = I.neuron_rec_steps.size();
        s.ca = I.rec_Ca.size();
        s.ip3 = I.rec_IP3.size();
        s.v = I.rec_V.size();
        s.isic = I.rec_Isic.size();
        s.se = I.spike_edges;
        s.sic = I.sic_edges;
        s.ns = I.n_spikes;
    }
    ASG_CUDA(cudaStreamSynchronize(e.stream));
    auto restore = [&]() -> int {
        ASG_TRY(e.flush());
        for (std::size_t i = 0; i < e.insts.size(); ++i) {
            Instance& I = *e.insts[i];
            Snap& s = snaps[i];
            ASG_CUDA(cudaMemcpyAsync(I.arena.get(), s.copy.get(), I.arena_bytes,
                                     cudaMemcpyDeviceToDevice, e.stream));
            I.step = s.step;
            I.spikes.resize(s.spikes);
            I.astro_rec_steps.resize(s.arows);
            I.neuron_rec_steps.resize(s.nrows);
            I.rec_Ca.resize(s.ca);
            I.rec_IP3.resize(s.ip3);
            I.rec_V.resize(s.v);
            I.rec_Isic.resize(s.isic);
            I.spike_edges = s.se;
            I.sic_edges = s.sic;
            I.n_spikes = s.ns;
        }
        ASG_CUDA(cudaStreamSynchronize(e.stream));
        return ASG_OK;
    };
    const int block0 = e.cfg.block, chunk0 = e.cfg.chunk_steps, mode0 = e.cfg.use_graphs;
    int best_block = block0, best_chunk = chunk0, best_mode = mode0;
    double best = 1e300;
    for (int mode : {1, 2}) {
        for (int chunk : {32, 64, 128, 256, 512}) {  // up to the chunk the instances were sized for
            if (e.set_chunk(chunk) != ASG_OK) continue;
            for (int block : {128, 256, 512}) {
                ASG_TRY(e.set_block(block));
                ASG_TRY(e.set_mode(mode));
                ASG_TRY(e.run(std::max(steps / 4, 1)));  // warm: graph build, caches
                ASG_TRY(restore());
                ASG_TRY(e.run(steps));
                const double per = e.last_ms / steps;
                if (per < best) {
                    best = per;
                    best_block = block;
                    best_chunk = chunk;
                    best_mode = mode;
                }
                ASG_TRY(restore());
            }
        }
    }
    clear_error();
    ASG_TRY(e.set_chunk(best_chunk));
    ASG_TRY(e.set_block(best_block));
    ASG_TRY(e.set_mode(best_mode));
    if (chosen != nullptr) {
        std::memset(chosen, 0, sizeof *chosen);
        chosen->device = e.cfg.device;
        chosen->chunk_steps = best_chunk;
        chosen->block = best_block;
        chosen->use_graphs = best_mode;
        chosen->sic_mode = e.cfg.sic_mode;
        chosen->pdl = e.cfg.pdl ? 0 : -1;
        chosen->push_mode = e.cfg.push_mode;
        chosen->mem_budget = e.cfg.mem_budget;
        chosen->occupancy = e.cfg.occupancy;
    }
    (void)block0;
    (void)mode0;
    return ASG_OK;
}


}  // namespace asg

using asg::BatchHandle;
using asg::Engine;
using asg::NetworkHandle;

extern "C" {

int asg_create(const asg_network_desc* desc, const asg_record_opts* rec,
               const asg_engine_opts* opts, asg_network** out) {
    asg::clear_error();
    if (desc == nullptr || out == nullptr) return asg::fail(ASG_ERR_ARG, "asg_create: NULL argument");
    *out = nullptr;
    auto h = std::make_unique<NetworkHandle>();
    asg::EngineConfig cfg = asg::config_from(opts);
    if (opts == nullptr || opts->chunk_steps <= 0)
        cfg.chunk_steps = asg::default_chunk(static_cast<std::uint64_t>(desc->n_exc) + desc->n_inh);
    h->eng = std::make_unique<Engine>(cfg);
    ASG_TRY(h->eng->init());
    ASG_TRY(h->eng->add(*desc, rec, 0, INT64_MAX, true, &h->id));
    *out = reinterpret_cast<asg_network*>(h.release());
    return ASG_OK;
}

int asg_step(asg_network* net, int64_t n_steps) {
    asg::clear_error();
    if (net == nullptr) return asg::fail(ASG_ERR_ARG, "asg_step: NULL handle");
    return reinterpret_cast<NetworkHandle*>(net)->eng->run(n_steps);
}

int asg_current_step(asg_network* net, int64_t* step) {
    asg::clear_error();
    if (net == nullptr || step == nullptr) return asg::fail(ASG_ERR_ARG, "asg_current_step: NULL");
    auto* h = reinterpret_cast<NetworkHandle*>(net);
    *step = h->eng->find(h->id)->step;
    return ASG_OK;
}

int asg_fetch_spikes(asg_network* net, int64_t* steps, uint32_t* sources, int64_t cap,
                     int64_t* count) {
    asg::clear_error();
    if (net == nullptr) return asg::fail(ASG_ERR_ARG, "asg_fetch_spikes: NULL handle");
    auto* h = reinterpret_cast<NetworkHandle*>(net);
    return asg::fetch_spikes_from(h->eng->find(h->id), steps, sources, cap, count);
}

int asg_fetch_record(asg_network* net, int64_t* astro_steps, double* Ca, double* IP3,
                     int64_t astro_cap_rows, int64_t* astro_rows, int64_t* neuron_steps,
                     double* V, double* I_sic, int64_t neuron_cap_rows, int64_t* neuron_rows) {
    asg::clear_error();
    if (net == nullptr) return asg::fail(ASG_ERR_ARG, "asg_fetch_record: NULL handle");
    auto* h = reinterpret_cast<NetworkHandle*>(net);
    return asg::fetch_record_from(h->eng->find(h->id), astro_steps, Ca, IP3, astro_cap_rows,
                                  astro_rows, neuron_steps, V, I_sic, neuron_cap_rows,
                                  neuron_rows);
}

int asg_pull_state(asg_network* net, asg_state* out) {
    asg::clear_error();
    if (net == nullptr || out == nullptr) return asg::fail(ASG_ERR_ARG, "asg_pull_state: NULL");
    auto* h = reinterpret_cast<NetworkHandle*>(net);
    return h->eng->pull_state(h->id, out);
}

int asg_pull_stp(asg_network* net, double* x, double* u, double* t_last) {
    asg::clear_error();
    if (net == nullptr) return asg::fail(ASG_ERR_ARG, "asg_pull_stp: NULL handle");
    auto* h = reinterpret_cast<NetworkHandle*>(net);
    return h->eng->pull_stp(h->id, x, u, t_last);
}

int asg_counters(asg_network* net, int64_t* spike_edges, int64_t* sic_edges, int64_t* spikes) {
    asg::clear_error();
    if (net == nullptr) return asg::fail(ASG_ERR_ARG, "asg_counters: NULL handle");
    auto* h = reinterpret_cast<NetworkHandle*>(net);
    const asg::Instance* I = h->eng->find(h->id);
    if (spike_edges) *spike_edges = I->spike_edges;
    if (sic_edges) *sic_edges = I->sic_edges;
    if (spikes) *spikes = I->n_spikes;
    return ASG_OK;
}

int asg_last_timing(asg_network* net, double* device_ms, int64_t* kernels) {
    asg::clear_error();
    if (net == nullptr) return asg::fail(ASG_ERR_ARG, "asg_last_timing: NULL handle");
    auto* h = reinterpret_cast<NetworkHandle*>(net);
    if (device_ms) *device_ms = h->eng->last_ms;
    if (kernels) *kernels = h->eng->last_kernels;
    return ASG_OK;
}

int asg_checkpoint_size(asg_network* net, uint64_t* bytes) {
    asg::clear_error();
    if (net == nullptr || bytes == nullptr) return asg::fail(ASG_ERR_ARG, "asg_checkpoint_size: NULL");
    auto* h = reinterpret_cast<NetworkHandle*>(net);
    *bytes = h->eng->find(h->id)->arena_bytes + sizeof(int64_t);
    return ASG_OK;
}

int asg_checkpoint(asg_network* net, void* host_buf, uint64_t bytes) {
    asg::clear_error();
    if (net == nullptr || host_buf == nullptr) return asg::fail(ASG_ERR_ARG, "asg_checkpoint: NULL");
    auto* h = reinterpret_cast<NetworkHandle*>(net);
    asg::Instance* I = h->eng->find(h->id);
    if (bytes < I->arena_bytes + sizeof(int64_t))
        return asg::fail(ASG_ERR_OVERFLOW, "checkpoint needs %zu bytes", I->arena_bytes + 8);
    ASG_CUDA(cudaStreamSynchronize(h->eng->stream));
    std::memcpy(host_buf, &I->step, sizeof(int64_t));
    ASG_CUDA(cudaMemcpy(static_cast<char*>(host_buf) + 8, I->arena.get(), I->arena_bytes,
                        cudaMemcpyDeviceToHost));
    return ASG_OK;
}

int asg_restore(asg_network* net, const void* host_buf, uint64_t bytes) {
    asg::clear_error();
    if (net == nullptr || host_buf == nullptr) return asg::fail(ASG_ERR_ARG, "asg_restore: NULL");
    auto* h = reinterpret_cast<NetworkHandle*>(net);
    asg::Instance* I = h->eng->find(h->id);
    if (bytes != I->arena_bytes + sizeof(int64_t))
        return asg::fail(ASG_ERR_ARG, "checkpoint size %llu does not match this network (%zu)",
                         static_cast<unsigned long long>(bytes), I->arena_bytes + 8);
    ASG_CUDA(cudaStreamSynchronize(h->eng->stream));
    std::memcpy(&I->step, host_buf, sizeof(int64_t));
    ASG_CUDA(cudaMemcpy(I->arena.get(), static_cast<const char*>(host_buf) + 8, I->arena_bytes,
                        cudaMemcpyHostToDevice));
    I->spikes.clear();
    I->dev.noise_from = I->step;  // noise terms drawn afresh at the first step
    h->eng->mark_side_prime();
    return ASG_OK;
}

int asg_destroy(asg_network* net) {
    asg::clear_error();
    delete reinterpret_cast<NetworkHandle*>(net);
    return ASG_OK;
}

// ------------------------------------------------------------------ batch

int asg_batch_create(int32_t n, const asg_network_desc* const* descs, const asg_record_opts* rec,
                     const asg_engine_opts* opts, asg_batch** out) {
    asg::clear_error();
    if (out == nullptr || (n > 0 && descs == nullptr) || n < 0)
        return asg::fail(ASG_ERR_ARG, "asg_batch_create: bad arguments");
    *out = nullptr;
    auto h = std::make_unique<BatchHandle>();
    asg::EngineConfig cfg = asg::config_from(opts);
    // A batch of 2^16+ neurons in all runs throughput-bound steps: its
    // instances with short SIC lists sum SIC in their neuron threads.
    std::uint64_t total = 0;
    for (int32_t i = 0; i < n; ++i)
        if (descs[i] != nullptr) total += static_cast<std::uint64_t>(descs[i]->n_exc) + descs[i]->n_inh;
    cfg.large_total = total >= (1u << 16);
    h->eng = std::make_unique<Engine>(cfg);
    ASG_TRY(h->eng->init());
    for (int32_t i = 0; i < n; ++i) {
        if (descs[i] == nullptr) return asg::fail(ASG_ERR_ARG, "asg_batch_create: descs[%d] NULL", i);
        int id = -1;
        const int st = h->eng->add(*descs[i], rec, 0, INT64_MAX, true, &id);
        if (st != ASG_OK) return st;
        h->ids.push_back(id);
    }
    *out = reinterpret_cast<asg_batch*>(h.release());
    return ASG_OK;
}

static asg::Instance* batch_inst(asg_batch* b, int32_t inst) {
    auto* h = reinterpret_cast<BatchHandle*>(b);
    if (inst < 0 || inst >= static_cast<int32_t>(h->ids.size())) return nullptr;
    return h->eng->find(h->ids[inst]);
}

int asg_batch_step(asg_batch* b, int64_t n_steps) {
    asg::clear_error();
    if (b == nullptr) return asg::fail(ASG_ERR_ARG, "asg_batch_step: NULL handle");
    return reinterpret_cast<BatchHandle*>(b)->eng->run(n_steps);
}

int asg_batch_fetch_spikes(asg_batch* b, int32_t inst, int64_t* steps, uint32_t* sources,
                           int64_t cap, int64_t* count) {
    asg::clear_error();
    if (b == nullptr) return asg::fail(ASG_ERR_ARG, "asg_batch_fetch_spikes: NULL handle");
    asg::Instance* I = batch_inst(b, inst);
    if (I == nullptr) return asg::fail(ASG_ERR_NOT_FOUND, "no instance %d", inst);
    return asg::fetch_spikes_from(I, steps, sources, cap, count);
}

int asg_batch_fetch_record(asg_batch* b, int32_t inst, int64_t* astro_steps, double* Ca,
                           double* IP3, int64_t astro_cap_rows, int64_t* astro_rows,
                           int64_t* neuron_steps, double* V, double* I_sic,
                           int64_t neuron_cap_rows, int64_t* neuron_rows) {
    asg::clear_error();
    if (b == nullptr) return asg::fail(ASG_ERR_ARG, "asg_batch_fetch_record: NULL handle");
    asg::Instance* I = batch_inst(b, inst);
    if (I == nullptr) return asg::fail(ASG_ERR_NOT_FOUND, "no instance %d", inst);
    return asg::fetch_record_from(I, astro_steps, Ca, IP3, astro_cap_rows, astro_rows,
                                  neuron_steps, V, I_sic, neuron_cap_rows, neuron_rows);
}

int asg_batch_pull_state(asg_batch* b, int32_t inst, asg_state* out) {
    asg::clear_error();
    if (b == nullptr || out == nullptr) return asg::fail(ASG_ERR_ARG, "asg_batch_pull_state: NULL");
    auto* h = reinterpret_cast<BatchHandle*>(b);
    if (inst < 0 || inst >= static_cast<int32_t>(h->ids.size()))
        return asg::fail(ASG_ERR_NOT_FOUND, "no instance %d", inst);
    return h->eng->pull_state(h->ids[inst], out);
}

int asg_batch_counters(asg_batch* b, int32_t inst, int64_t* spike_edges, int64_t* sic_edges,
                       int64_t* spikes) {
    asg::clear_error();
    if (b == nullptr) return asg::fail(ASG_ERR_ARG, "asg_batch_counters: NULL handle");
    asg::Instance* I = batch_inst(b, inst);
    if (I == nullptr) return asg::fail(ASG_ERR_NOT_FOUND, "no instance %d", inst);
    if (spike_edges) *spike_edges = I->spike_edges;
    if (sic_edges) *sic_edges = I->sic_edges;
    if (spikes) *spikes = I->n_spikes;
    return ASG_OK;
}

int asg_batch_last_timing(asg_batch* b, double* device_ms, int64_t* kernels) {
    asg::clear_error();
    if (b == nullptr) return asg::fail(ASG_ERR_ARG, "asg_batch_last_timing: NULL handle");
    auto* h = reinterpret_cast<BatchHandle*>(b);
    if (device_ms) *device_ms = h->eng->last_ms;
    if (kernels) *kernels = h->eng->last_kernels;
    return ASG_OK;
}

int asg_batch_autotune(asg_batch* b, int32_t steps, asg_engine_opts* chosen) {
    asg::clear_error();
    if (b == nullptr || steps <= 0) return asg::fail(ASG_ERR_ARG, "asg_batch_autotune: bad arguments");
    return asg::autotune_engine(*reinterpret_cast<BatchHandle*>(b)->eng, steps, chosen);
}

int asg_autotune(asg_network* net, int32_t steps, asg_engine_opts* chosen) {
    asg::clear_error();
    if (net == nullptr || steps <= 0) return asg::fail(ASG_ERR_ARG, "asg_autotune: bad arguments");
    return asg::autotune_engine(*reinterpret_cast<NetworkHandle*>(net)->eng, steps, chosen);
}

int asg_batch_destroy(asg_batch* b) {
    asg::clear_error();
    delete reinterpret_cast<BatchHandle*>(b);
    return ASG_OK;
}

}  // extern "C"

extern "C" int asg_selftest_barrier_timeout(int32_t* timed_out, double* wait_ms) {
    asg::clear_error();
    if (timed_out == nullptr) return asg::fail(ASG_ERR_ARG, "asg_selftest_barrier_timeout: NULL");
    asg::DevBuf gb;
    ASG_TRY(gb.alloc(sizeof(asg::GridBarrier)));
    cudaEvent_t a, b;
    ASG_CUDA(cudaEventCreate(&a));
    ASG_CUDA(cudaEventCreate(&b));
    ASG_CUDA(cudaEventRecord(a, nullptr));
    ASG_CUDA(asg::barrier_selftest(gb.as<asg::GridBarrier>(), nullptr));
    ASG_CUDA(cudaEventRecord(b, nullptr));
    ASG_CUDA(cudaEventSynchronize(b));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    asg::GridBarrier h{};
    ASG_CUDA(cudaMemcpy(&h, gb.get(), sizeof h, cudaMemcpyDeviceToHost));
    *timed_out = h.error != 0;
    if (wait_ms) *wait_ms = ms;
    return ASG_OK;
}
