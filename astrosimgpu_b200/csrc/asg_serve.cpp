// Serving: continuous batching of simulation requests over one Engine, and
// the launch-shape autotuner of the batched sweep.
//
// Two host threads share the engine.  The admission thread prepares queued
// requests in arrival order while their device footprint fits the budget
// (validation, device in-edge numbering, arena upload: everything that does
// not touch the running batch) and stages them.  The stepping thread, at
// each chunk boundary, joins the staged requests, removes cancelled ones,
// runs one chunk of steps for every resident request, and retires requests
// that reached their last step, recording submit->admit and submit->done
// latency.  Requests join and leave only at chunk boundaries, so a request's
// arithmetic is the same alone and in any mix.

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "asg_engine.hpp"

namespace asg {

EngineConfig config_from(const asg_engine_opts* o);

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// Deep copy of a descriptor: the caller's arrays may be freed after submit.
struct DescCopy {
    asg_network_desc d{};
    std::vector<std::vector<std::uint32_t>> u32;
    std::vector<std::vector<double>> f64;
    std::vector<std::vector<std::int32_t>> i32;

    template <typename T, typename Store>
    const T* keep(const T* p, std::size_t n, Store& s) {
        if (p == nullptr || n == 0) return nullptr;
        s.emplace_back(p, p + n);
        return s.back().data();
    }

    explicit DescCopy(const asg_network_desc& src) : d(src) {
        u32.reserve(16);
        f64.reserve(32);
        i32.reserve(8);
        const std::size_t N = src.n_exc + src.n_inh, NA = src.n_astro;
        auto csr = [&](asg_csr& c) {
            if (c.n_sources == 0 || c.row_start == nullptr) return;
            const std::size_t m = c.row_start[c.n_sources];
            c.row_start = keep(c.row_start, c.n_sources + 1, u32);
            c.target = keep(c.target, m, u32);
            c.weight = keep(c.weight, m, f64);
            c.delay_steps = keep(c.delay_steps, m, i32);
            c.stp_x = keep(c.stp_x, m, f64);
            c.stp_u = keep(c.stp_u, m, f64);
            c.stp_t_last = keep(c.stp_t_last, m, f64);
        };
        csr(d.exc_primary);
        csr(d.inh_primary);
        csr(d.neuron_astro);
        csr(d.astro_neuron);
        d.V_reset = keep(src.V_reset, N, f64);
        d.b = keep(src.b, N, f64);
        d.Ca_tot = keep(src.Ca_tot, NA, f64);
        d.IP3_0 = keep(src.IP3_0, NA, f64);
        d.tau_IP3 = keep(src.tau_IP3, NA, f64);
        d.delta_IP3 = keep(src.delta_IP3, NA, f64);
        d.V = keep(src.V, N, f64);
        d.w = keep(src.w, N, f64);
        d.g_ex = keep(src.g_ex, N, f64);
        d.dg_ex = keep(src.dg_ex, N, f64);
        d.g_in = keep(src.g_in, N, f64);
        d.dg_in = keep(src.dg_in, N, f64);
        d.I_sic = keep(src.I_sic, N, f64);
        d.refractory = keep(src.refractory, N, i32);
        d.Ca = keep(src.Ca, NA, f64);
        d.IP3 = keep(src.IP3, NA, f64);
        d.h = keep(src.h, NA, f64);
    }
};

enum class ReqState { Queued, Preparing, Staged, Running, Done };

struct Request {
    std::int64_t id = 0;
    std::unique_ptr<DescCopy> desc;
    std::int64_t n_steps = 0;
    bool keep_spikes = true;
    ReqState state = ReqState::Queued;
    bool cancel = false;
    int inst = -1;
    std::uint64_t footprint = 0;
    Clock::time_point t_submit, t_admit, t_done;
    asg_request_result result{};
    std::vector<SpikeRec> spikes;
    std::unique_ptr<Instance> prepared;  // built by the admission thread, not yet joined
    std::string error;                   // text of a failed admission
};

}  // namespace

struct Server {
    std::unique_ptr<Engine> eng;
    std::uint64_t budget = 0;
    int max_instances = 256;
    std::mutex mu;
    // cv_work wakes the stepping loop (staged requests, cancels, stop);
    // cv_admit the admission thread (submits, retirements, cancels, stop).
    std::condition_variable cv_work, cv_admit, cv_done;
    std::deque<std::int64_t> queue;   // submitted, waiting for admission
    std::deque<std::int64_t> staged;  // prepared, waiting for a chunk boundary
    std::map<std::int64_t, std::unique_ptr<Request>> reqs;
    std::int64_t next_id = 1;
    bool stop = false;
    int loop_status = ASG_OK;
    std::string loop_error;
    std::int32_t resident = 0, peak_resident = 0;
    std::int32_t in_admission = 0;       // preparing or staged
    std::uint64_t resident_bytes = 0;    // footprints of running requests
    std::uint64_t reserved_bytes = 0;    // footprints of requests in admission
    std::int64_t retirements = 0;        // bumps whenever device memory frees up
    std::thread thread, admit_thread;

    void loop();
    void admit_loop();
    void retire(Request& r, int status);
};

void Server::retire(Request& r, int status) {
    Instance* I = r.inst >= 0 ? eng->find(r.inst) : nullptr;
    r.t_done = Clock::now();
    r.result.status = status;
    if (I != nullptr) {
        r.result.n_spikes = I->n_spikes;
        r.result.spike_edges = I->spike_edges;
        r.result.sic_edges = I->sic_edges;
        const double sim_ms = static_cast<double>(r.n_steps) * r.desc->d.dt;
        const double n = static_cast<double>(r.desc->d.n_exc + r.desc->d.n_inh);
        r.result.mean_rate_hz = sim_ms > 0.0 && n > 0.0
                                    ? static_cast<double>(I->n_spikes) * 1000.0 / (sim_ms * n)
                                    : 0.0;
        if (r.keep_spikes) r.spikes.swap(I->spikes);
        resident_bytes -= r.footprint;
        eng->remove(r.inst);
        --resident;
        ++retirements;
        cv_admit.notify_all();
    }
    r.result.submit_to_admit_ms = r.state == ReqState::Running
                                      ? ms_between(r.t_submit, r.t_admit)
                                      : ms_between(r.t_submit, r.t_done);
    r.result.submit_to_done_ms = ms_between(r.t_submit, r.t_done);
    r.state = ReqState::Done;
    r.desc.reset();  // host copy no longer needed
    r.prepared.reset();
}

// Admission, off the stepping loop: takes queued requests in arrival order
// while their footprint fits the budget beside the resident and staged ones,
// and prepares each (validation, in-edge numbering on the GPU, SIC lists,
// arena upload) without holding the server lock, while the loop keeps
// stepping the resident requests.  Prepared requests are staged; the loop
// joins them at its next chunk boundary.
void Server::admit_loop() {
    cudaSetDevice(eng->cfg.device);  // this thread's calls go to the server's GPU
    std::unique_lock<std::mutex> lk(mu);
    while (!stop) {
        if (queue.empty()) {
            cv_admit.wait(lk, [&] { return stop || !queue.empty(); });
            continue;
        }
        Request& r = *reqs[queue.front()];
        if (r.cancel) {
            queue.pop_front();
            retire(r, ASG_ERR_CANCELLED);
            cv_done.notify_all();
            continue;
        }
        if (resident + in_admission >= max_instances ||
            resident_bytes + reserved_bytes + r.footprint > budget) {
            const std::int64_t seen = retirements;
            cv_admit.wait(lk, [&] { return stop || retirements != seen || r.cancel; });
            continue;
        }
        queue.pop_front();
        r.state = ReqState::Preparing;
        reserved_bytes += r.footprint;
        ++in_admission;
        const std::int64_t seen = retirements;
        const asg_network_desc* d = &r.desc->d;
        lk.unlock();
        asg_record_opts ro{};
        ro.record_every = 1;
        ro.spikes = r.keep_spikes ? 1 : 0;
        std::unique_ptr<Instance> inst;
        const int st = eng->prepare(*d, &ro, 0, r.n_steps, r.keep_spikes, false, &inst);
        const std::string err = st != ASG_OK ? asg_last_error() : std::string();
        lk.lock();
        if (stop) {  // the server is shutting down or the loop failed
            inst.reset();
            reserved_bytes -= r.footprint;
            --in_admission;
            retire(r, loop_status != ASG_OK ? loop_status : ASG_ERR_CANCELLED);
            cv_done.notify_all();
            break;
        }
        if (st == ASG_ERR_OOM && (resident > 0 || in_admission > 1)) {
            // the device is short of memory now: retry once something leaves
            inst.reset();
            reserved_bytes -= r.footprint;
            --in_admission;
            r.state = ReqState::Queued;
            queue.push_front(r.id);
            cv_admit.wait(lk, [&] { return stop || retirements != seen || r.cancel; });
            continue;
        }
        if (st != ASG_OK) {
            reserved_bytes -= r.footprint;
            --in_admission;
            r.error = err;
            retire(r, st);
            cv_done.notify_all();
            continue;
        }
        r.prepared = std::move(inst);
        r.state = ReqState::Staged;
        staged.push_back(r.id);
        cv_work.notify_one();
    }
}

// Stepping: at each chunk boundary retire cancelled requests and join the
// staged ones, run one chunk of steps for every resident request, and retire
// those that reached their last step.  Requests join and leave only at chunk
// boundaries, so a request's arithmetic is the same alone and in any mix.
void Server::loop() {
    cudaSetDevice(eng->cfg.device);  // this thread's calls go to the server's GPU
    std::unique_lock<std::mutex> lk(mu);
    while (!stop) {
        for (auto& kv : reqs) {
            Request& r = *kv.second;
            if (r.cancel && r.state == ReqState::Running) retire(r, ASG_ERR_CANCELLED);
        }
        std::vector<Request*> joining;
        while (!staged.empty()) {
            Request& r = *reqs[staged.front()];
            staged.pop_front();
            reserved_bytes -= r.footprint;
            --in_admission;
            if (r.cancel) {
                retire(r, ASG_ERR_CANCELLED);
                continue;
            }
            joining.push_back(&r);
        }
        if (!joining.empty()) {
            // the join waits for the chunks in flight: outside the lock
            std::vector<int> ids(joining.size(), -1), sts(joining.size(), ASG_OK);
            std::vector<std::string> errs(joining.size());
            std::vector<std::unique_ptr<Instance>> prepared;
            for (Request* r : joining) prepared.push_back(std::move(r->prepared));
            lk.unlock();
            for (std::size_t k = 0; k < joining.size(); ++k) {
                sts[k] = eng->commit(std::move(prepared[k]), &ids[k]);
                if (sts[k] != ASG_OK) errs[k] = asg_last_error();
            }
            lk.lock();
            for (std::size_t k = 0; k < joining.size(); ++k) {
                Request& r = *joining[k];
                if (sts[k] != ASG_OK) {
                    r.error = errs[k];
                    retire(r, sts[k]);
                    continue;
                }
                r.inst = ids[k];
                r.state = ReqState::Running;
                r.t_admit = Clock::now();
                resident_bytes += r.footprint;
                peak_resident = std::max(peak_resident, ++resident);
            }
        }
        cv_done.notify_all();
        if (resident == 0) {
            cv_work.wait(lk, [&] { return stop || !staged.empty(); });
            continue;
        }
        // one chunk for every resident request, outside the lock
        lk.unlock();
        int st = eng->run_chunk(eng->cfg.chunk_steps);
        bool finishing = false;
        for (auto& p : eng->insts) finishing = finishing || p->done();
        // retiring requests need the outputs of every chunk still in flight
        if (st == ASG_OK && finishing) st = eng->flush();
        lk.lock();
        if (st != ASG_OK) {
            loop_status = st;
            loop_error = asg_last_error();
            // every request not being prepared right now ends with the error
            // (the admission thread ends the one it is preparing)
            for (auto& kv : reqs)
                if (kv.second->state != ReqState::Done && kv.second->state != ReqState::Preparing)
                    retire(*kv.second, st);
            queue.clear();
            staged.clear();
            stop = true;
            cv_admit.notify_all();
            break;
        }
        for (auto& kv : reqs) {
            Request& r = *kv.second;
            if (r.state != ReqState::Running) continue;
            Instance* I = eng->find(r.inst);
            if (I != nullptr && I->done()) retire(r, ASG_OK);
        }
    }
    cv_done.notify_all();
}

}  // namespace asg

using asg::Server;

extern "C" {

int asg_serve_create(const asg_serve_opts* opts, asg_server** out) {
    asg::clear_error();
    if (out == nullptr) return asg::fail(ASG_ERR_ARG, "asg_serve_create: out is NULL");
    *out = nullptr;
    auto s = std::make_unique<Server>();
    asg::EngineConfig cfg = asg::config_from(opts ? &opts->engine : nullptr);
    if (opts == nullptr || opts->engine.chunk_steps <= 0) cfg.chunk_steps = 64;
    s->eng = std::make_unique<asg::Engine>(cfg);
    ASG_TRY(s->eng->init());
    if (opts != nullptr && opts->mem_budget > 0) {
        s->budget = opts->mem_budget;
    } else {
        std::size_t fr = 0, tot = 0;
        ASG_CUDA(cudaMemGetInfo(&fr, &tot));
        s->budget = static_cast<std::uint64_t>(0.8 * static_cast<double>(fr));
    }
    s->eng->cfg.mem_budget = s->budget + (1ull << 30);
    if (opts != nullptr && opts->max_instances > 0) s->max_instances = opts->max_instances;
    Server* raw = s.get();
    s->thread = std::thread([raw] { raw->loop(); });
    s->admit_thread = std::thread([raw] { raw->admit_loop(); });
    *out = reinterpret_cast<asg_server*>(s.release());
    return ASG_OK;
}

int asg_serve_submit(asg_server* sp, const asg_network_desc* desc, int64_t n_steps,
                     int32_t keep_spikes, int64_t* request_id) {
    asg::clear_error();
    if (sp == nullptr || desc == nullptr || request_id == nullptr || n_steps < 0)
        return asg::fail(ASG_ERR_ARG, "asg_serve_submit: bad arguments");
    auto* s = reinterpret_cast<Server*>(sp);
    std::uint64_t fp = 0;
    asg::Engine::footprint(*desc, s->eng->cfg.chunk_steps, &fp);
    if (fp > s->budget)
        return asg::fail(ASG_ERR_OOM, "request needs ~%llu device bytes, budget is %llu",
                         static_cast<unsigned long long>(fp),
                         static_cast<unsigned long long>(s->budget));
    auto r = std::make_unique<asg::Request>();
    r->desc = std::make_unique<asg::DescCopy>(*desc);
    r->n_steps = n_steps;
    r->keep_spikes = keep_spikes != 0;
    r->footprint = fp;
    r->t_submit = asg::Clock::now();
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->stop)
            return asg::fail(ASG_ERR_STATE, "server stopped: %s", s->loop_error.c_str());
        r->id = s->next_id++;
        *request_id = r->id;
        s->queue.push_back(r->id);
        s->reqs[r->id] = std::move(r);
    }
    s->cv_admit.notify_all();
    return ASG_OK;
}

int asg_serve_poll(asg_server* sp, int64_t id, int32_t* done, asg_request_result* res) {
    asg::clear_error();
    if (sp == nullptr || done == nullptr) return asg::fail(ASG_ERR_ARG, "asg_serve_poll: NULL");
    auto* s = reinterpret_cast<Server*>(sp);
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return asg::fail(ASG_ERR_NOT_FOUND, "no request %lld", (long long)id);
    *done = it->second->state == asg::ReqState::Done;
    if (*done && res) *res = it->second->result;
    return ASG_OK;
}

int asg_serve_wait(asg_server* sp, int64_t id, double timeout_ms, asg_request_result* res) {
    asg::clear_error();
    if (sp == nullptr) return asg::fail(ASG_ERR_ARG, "asg_serve_wait: NULL handle");
    auto* s = reinterpret_cast<Server*>(sp);
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return asg::fail(ASG_ERR_NOT_FOUND, "no request %lld", (long long)id);
    asg::Request* r = it->second.get();
    auto pred = [&] { return r->state == asg::ReqState::Done; };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, pred);
    } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms),
                                    pred)) {
        return asg::fail(ASG_ERR_TIMEOUT, "request %lld not done after %.1f ms", (long long)id,
                         timeout_ms);
    }
    if (res) *res = r->result;
    return r->result.status == ASG_OK || r->result.status == ASG_ERR_CANCELLED
               ? ASG_OK
               : asg::fail(r->result.status, "request %lld failed: %s", (long long)id,
                           r->error.empty() ? s->loop_error.c_str() : r->error.c_str());
}

int asg_serve_fetch_spikes(asg_server* sp, int64_t id, int64_t* steps, uint32_t* sources,
                           int64_t cap, int64_t* count) {
    asg::clear_error();
    if (sp == nullptr) return asg::fail(ASG_ERR_ARG, "asg_serve_fetch_spikes: NULL handle");
    auto* s = reinterpret_cast<Server*>(sp);
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return asg::fail(ASG_ERR_NOT_FOUND, "no request %lld", (long long)id);
    asg::Request& r = *it->second;
    if (r.state != asg::ReqState::Done) return asg::fail(ASG_ERR_STATE, "request still running");
    const int64_t n = static_cast<int64_t>(r.spikes.size());
    if (count) *count = n;
    if (steps == nullptr && sources == nullptr) return ASG_OK;
    if (n > cap) return asg::fail(ASG_ERR_OVERFLOW, "%lld spikes, buffer holds %lld", (long long)n,
                                  (long long)cap);
    for (int64_t i = 0; i < n; ++i) {
        if (steps) steps[i] = r.spikes[i].step;
        if (sources) sources[i] = r.spikes[i].source;
    }
    return ASG_OK;
}

int asg_serve_cancel(asg_server* sp, int64_t id) {
    asg::clear_error();
    if (sp == nullptr) return asg::fail(ASG_ERR_ARG, "asg_serve_cancel: NULL handle");
    auto* s = reinterpret_cast<Server*>(sp);
    {
        std::lock_guard<std::mutex> g(s->mu);
        auto it = s->reqs.find(id);
        if (it == s->reqs.end())
            return asg::fail(ASG_ERR_NOT_FOUND, "no request %lld", (long long)id);
        it->second->cancel = true;
    }
    s->cv_work.notify_one();
    s->cv_admit.notify_all();
    return ASG_OK;
}

int asg_serve_stats(asg_server* sp, int64_t* chunks, int64_t* kernels, double* device_ms,
                    int32_t* resident, int32_t* peak) {
    asg::clear_error();
    if (sp == nullptr) return asg::fail(ASG_ERR_ARG, "asg_serve_stats: NULL handle");
    auto* s = reinterpret_cast<Server*>(sp);
    std::lock_guard<std::mutex> g(s->mu);
    if (chunks) *chunks = s->eng->chunks;
    if (kernels) *kernels = s->eng->launched_kernels;
    if (device_ms) *device_ms = s->eng->chunk_device_ms;
    if (resident) *resident = s->resident;
    if (peak) *peak = s->peak_resident;
    return ASG_OK;
}

int asg_serve_destroy(asg_server* sp) {
    asg::clear_error();
    if (sp == nullptr) return ASG_OK;
    auto* s = reinterpret_cast<Server*>(sp);
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->cv_admit.notify_all();
    if (s->admit_thread.joinable()) s->admit_thread.join();
    if (s->thread.joinable()) s->thread.join();
    delete s;
    return ASG_OK;
}

}  // extern "C"
