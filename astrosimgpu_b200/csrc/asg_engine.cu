// Host side of the network engine (see asg_engine.hpp / asg_engine.cuh):
// descriptor validation, table preprocessing, the per-instance device arena,
// the work table, captured chunks and output collection.

#include "asg_engine.hpp"

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

namespace asg {

namespace {

constexpr double kE = 2.7182818284590452353602874713527;

int delay_ok(int d) { return d >= 1; }

// Derived constants of one neuron population (values the reference forms at
// run time are formed here with the same IEEE operations).
NeuronK make_neuron_k(const asg_neuron_params& p, const asg_input& in, double dt, double h) {
    NeuronK k{};
    k.C_m = p.C_m;
    k.g_L = p.g_L;
    k.E_L = p.E_L;
    k.V_th = p.V_th;
    k.Delta_T = p.Delta_T;
    k.a = p.a;
    k.tau_w = p.tau_w;
    k.V_peak = p.V_peak;
    k.E_ex = p.E_ex;
    k.E_in = p.E_in;
    k.I_e = p.I_e;
    k.inv_C_m = 1.0 / p.C_m;
    k.inv_Delta_T = 1.0 / p.Delta_T;
    k.inv_tau_w = 1.0 / p.tau_w;
    k.neg_g_L = -p.g_L;
    k.gl_dt = p.g_L * p.Delta_T;
    k.psc_ex = kE / p.tau_syn_ex;
    k.psc_in = kE / p.tau_syn_in;
    k.decay_ex = std::exp(-h / p.tau_syn_ex);
    k.decay_in = std::exp(-h / p.tau_syn_in);
    k.ref_steps = static_cast<int>(p.t_ref / h + 0.5);
    k.poiss_rate = in.poiss_rate;
    k.poiss_weight = in.poiss_weight;
    k.lambda = in.poiss_rate * dt * 1e-3;
    k.knuth_limit = std::exp(-k.lambda);
    k.noise_std = in.gauss_noise_std;
    k.independent_noise = in.independent_noise != 0;
    k.steps_per_noise = std::max(1, static_cast<int>(std::llround(in.noise_dt / dt)));
    return k;
}

AstroK make_astro_k(const asg_astro_params& a, double h, int substeps) {
    AstroK k{};
    k.Kd_IP3_1 = a.Kd_IP3_1;
    k.Kd_IP3_2 = a.Kd_IP3_2;
    k.Kd_act = a.Kd_act;
    k.ratio_ER_cyt = a.ratio_ER_cyt;
    k.inv_ratio = 1.0 / a.ratio_ER_cyt;
    k.chan = a.ratio_ER_cyt * a.rate_IP3R;
    k.serca = a.rate_SERCA;
    k.km2 = a.Km_SERCA * a.Km_SERCA;
    k.leak = a.ratio_ER_cyt * a.rate_L;
    k.ah = a.k_IP3R * a.Kd_inh;
    k.k_IP3R = a.k_IP3R;
    k.half_h = 0.5 * h;
    k.h = h;
    k.h6 = h / 6.0;
    k.substeps = substeps;
    return k;
}

// Device memory from the stream-ordered allocator: freeing it does not wait
// for the device (cudaFree would, and stall the chunks in flight).
struct AsyncBuf {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    cudaError_t alloc(std::size_t bytes, cudaStream_t st) {
        s = st;
        return cudaMallocAsync(&p, std::max<std::size_t>(bytes, 16), st);
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
    ~AsyncBuf() {
        if (p) cudaFreeAsync(p, s);
    }
};

// Transposed in-edge structure of one set, built on the device.  A target's
// in-edges are numbered p = 0.. in (source, row position) order; bit p of the
// target's words marks an arrival on that edge.
struct InRingDev {
    AsyncBuf wbase;  // [n_targets + 1] first bitmap word of each target
    AsyncBuf edge;   // [m] bit | target << 32 | dense << 57 | summary bit << 58
    std::uint32_t words = 0, m = 0;
};

__global__ void ring_count_kernel(const std::uint32_t* __restrict__ tg, std::uint32_t m,
                                  std::uint32_t* __restrict__ deg) {
    for (std::uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m;
         e += gridDim.x * blockDim.x)
        atomicAdd(deg + tg[e], 1u);
}

// words[t] = ceil(deg[t] / 32); words[n] = 0 (so the scan's last entry is the total)
__global__ void ring_words_kernel(const std::uint32_t* __restrict__ deg, std::uint32_t n,
                                  std::uint32_t* __restrict__ words) {
    for (std::uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t <= n;
         t += gridDim.x * blockDim.x)
        words[t] = t < n ? (deg[t] + 31) / 32 : 0u;
}

__global__ void ring_iota_kernel(std::uint32_t* __restrict__ v, std::uint32_t m) {
    for (std::uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m;
         e += gridDim.x * blockDim.x)
        v[e] = e;
}

// Sorted position i holds edge se[i] to target st[i]; the sort is stable, so
// the edges of one target sit in (source, row position) order and the
// edge's number is i - seg[t].
__global__ void ring_pack_kernel(const std::uint32_t* __restrict__ st,
                                 const std::uint32_t* __restrict__ se, std::uint32_t m,
                                 const std::uint32_t* __restrict__ seg,
                                 const std::uint32_t* __restrict__ wbase,
                                 unsigned long long* __restrict__ edge) {
    for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += gridDim.x * blockDim.x) {
        const std::uint32_t t = st[i];
        const std::uint32_t p = i - seg[t];
        const std::uint32_t nw = wbase[t + 1] - wbase[t];
        const std::uint32_t G = (nw + 63) / 64;
        const unsigned long long bit = static_cast<unsigned long long>(wbase[t]) * 32 + p;
        // A target of at most 32 words reads all its words at once and never
        // its summary: its pushes skip the summary update.
        const unsigned long long dense = nw <= 32 ? 1ull : 0ull;
        edge[se[i]] = bit | (static_cast<unsigned long long>(t) << 32) | (dense << 57) |
                      (static_cast<unsigned long long>((p / 32) / G) << 58);
    }
}

// The in-edge numbering of one set (n_src sources, CSR rs / tg on the host)
// on `st`: in-degrees, word bases and segment starts by exclusive scans,
// then a stable radix sort of (target, edge) pairs and the packing.  Returns
// with r.words known (the stream synchronised once for it).
int build_in_ring(std::uint32_t n_src, const std::uint32_t* rs, const std::uint32_t* tg,
                  std::uint32_t n_targets, cudaStream_t st, InRingDev& r) {
    NvtxRange nvtx("admission: in-edge numbering (arrival rings)");
    const std::uint32_t m = rs[n_src];
    const std::uint32_t n = n_targets;
    r.m = m;
    if (m >= (1u << 31)) return fail(ASG_ERR_UNSUPPORTED, "a set of %u edges (at most 2^31-1)", m);
    // Scratch beyond the arena: a failed allocation reports ASG_ERR_OOM (a
    // server then waits for memory to free up).
    auto need = [&](AsyncBuf& buf, std::size_t bytes) -> int {
        const cudaError_t e = buf.alloc(bytes, st);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            return fail(ASG_ERR_OOM, "in-edge numbering: %zu device bytes unavailable", bytes);
        }
        return e == cudaSuccess ? ASG_OK : cuda_fail(e, "cudaMallocAsync", __FILE__, __LINE__);
    };
    ASG_TRY(need(r.wbase, (static_cast<std::size_t>(n) + 1) * 4));
    ASG_TRY(need(r.edge, static_cast<std::size_t>(m) * 8));
    if (m == 0) {
        ASG_CUDA(cudaMemsetAsync(r.wbase.p, 0, (static_cast<std::size_t>(n) + 1) * 4, st));
        r.words = 0;
        return ASG_OK;
    }
    AsyncBuf keys, keys_out, vals, vals_out, deg, seg, words, tmp;
    for (AsyncBuf* buf : {&keys, &keys_out, &vals, &vals_out})
        ASG_TRY(need(*buf, static_cast<std::size_t>(m) * 4));
    for (AsyncBuf* buf : {&deg, &seg, &words})
        ASG_TRY(need(*buf, (static_cast<std::size_t>(n) + 1) * 4));
    ASG_CUDA(cudaMemcpyAsync(keys.p, tg, static_cast<std::size_t>(m) * 4, cudaMemcpyDefault, st));
    ASG_CUDA(cudaMemsetAsync(deg.p, 0, (static_cast<std::size_t>(n) + 1) * 4, st));
    const unsigned blocks = 4096;
    ring_count_kernel<<<blocks, 256, 0, st>>>(keys.as<std::uint32_t>(), m, deg.as<std::uint32_t>());
    ring_words_kernel<<<blocks, 256, 0, st>>>(deg.as<std::uint32_t>(), n, words.as<std::uint32_t>());
    ring_iota_kernel<<<blocks, 256, 0, st>>>(vals.as<std::uint32_t>(), m);
    ASG_CUDA(cudaGetLastError());
    int end_bit = 1;
    while (end_bit < 32 && (1ull << end_bit) < n) ++end_bit;
    std::size_t b_scan = 0, b_sort = 0;
    ASG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b_scan, deg.as<std::uint32_t>(),
                                           seg.as<std::uint32_t>(), static_cast<int>(n) + 1, st));
    ASG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b_sort, keys.as<std::uint32_t>(),
                                             keys_out.as<std::uint32_t>(), vals.as<std::uint32_t>(),
                                             vals_out.as<std::uint32_t>(), static_cast<int>(m), 0,
                                             end_bit, st));
    std::size_t b = std::max(b_scan, b_sort);
    ASG_TRY(need(tmp, b));
    ASG_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, b, deg.as<std::uint32_t>(),
                                           seg.as<std::uint32_t>(), static_cast<int>(n) + 1, st));
    b = std::max(b_scan, b_sort);
    ASG_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, b, words.as<std::uint32_t>(),
                                           r.wbase.as<std::uint32_t>(), static_cast<int>(n) + 1, st));
    b = std::max(b_scan, b_sort);
    ASG_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, b, keys.as<std::uint32_t>(),
                                             keys_out.as<std::uint32_t>(), vals.as<std::uint32_t>(),
                                             vals_out.as<std::uint32_t>(), static_cast<int>(m), 0,
                                             end_bit, st));
    ring_pack_kernel<<<blocks, 256, 0, st>>>(keys_out.as<std::uint32_t>(), vals_out.as<std::uint32_t>(),
                                            m, seg.as<std::uint32_t>(), r.wbase.as<std::uint32_t>(),
                                            r.edge.as<unsigned long long>());
    ASG_CUDA(cudaGetLastError());
    ASG_CUDA(cudaMemcpyAsync(&r.words, r.wbase.as<std::uint32_t>() + n, 4, cudaMemcpyDeviceToHost, st));
    ASG_CUDA(cudaStreamSynchronize(st));
    return ASG_OK;
}

// Compressed SIC lists in sliced ELL (32 targets per slice), each target's
// list cut into `parts` consecutive pieces of about equal edge count (an
// (astrocyte, multiplicity) pair that straddles a cut is split in two: m1
// then m2 equal additions are the m additions).
struct SicHost {
    std::vector<std::uint32_t> soff, ent;
    std::uint32_t max_edges = 0;  // largest number of SIC edges of one target
};

constexpr std::uint32_t kSicEdgesPerPart = 160;
constexpr std::uint32_t kPushCells = 256;

// Longest SIC edge list of one target (sets the number of parts).
std::uint32_t sic_max_edges(std::uint32_t NA, const std::uint32_t* rs, const std::uint32_t* tg,
                            std::uint32_t N) {
    std::vector<std::uint32_t> deg(N, 0);
    for (std::uint32_t e = 0; e < rs[NA]; ++e) deg[tg[e]]++;
    std::uint32_t mx = 0;
    for (std::uint32_t d : deg) mx = std::max(mx, d);
    return mx;
}

SicHost make_sic(std::uint32_t NA, const std::uint32_t* rs, const std::uint32_t* tg,
                 std::uint32_t N, std::uint32_t parts, std::uint32_t npad) {
    // per target: (astro, mult) in ascending astro order
    std::vector<std::vector<std::uint32_t>> lists(N);
    for (std::uint32_t a = 0; a < NA; ++a) {
        for (std::uint32_t e = rs[a]; e < rs[a + 1]; ++e) {
            auto& l = lists[tg[e]];
            if (!l.empty() && (l.back() >> 8) == a && (l.back() & 0xFFu) < 255u) {
                l.back() += 1;
            } else {
                l.push_back((a << 8) | 1u);
            }
        }
    }
    // Split each target's list at edge counts floor(p * E / parts).
    const std::uint32_t V = parts * npad;
    std::vector<std::vector<std::uint32_t>> vl(V);
    SicHost s;
    for (std::uint32_t t = 0; t < N; ++t) {
        std::uint32_t E = 0;
        for (std::uint32_t x : lists[t]) E += x & 0xFFu;
        s.max_edges = std::max(s.max_edges, E);
        std::uint32_t done = 0, p = 0;
        for (std::uint32_t x : lists[t]) {
            std::uint32_t m = x & 0xFFu;
            const std::uint32_t a = x >> 8;
            while (m > 0) {
                // end (exclusive, in edges) of part p
                std::uint32_t end = static_cast<std::uint32_t>(
                    (static_cast<std::uint64_t>(p + 1) * E) / parts);
                while (done >= end && p + 1 < parts) {
                    ++p;
                    end = static_cast<std::uint32_t>((static_cast<std::uint64_t>(p + 1) * E) / parts);
                }
                const std::uint32_t take = std::min(m, end - done);
                vl[p * npad + t].push_back((a << 8) | take);
                done += take;
                m -= take;
            }
        }
    }
    const std::uint32_t slices = V / 32;
    s.soff.assign(slices + 1, 0);
    for (std::uint32_t sl = 0; sl < slices; ++sl) {
        std::size_t len = 0;
        for (std::uint32_t v = sl * 32; v < sl * 32 + 32; ++v) len = std::max(len, vl[v].size());
        s.soff[sl + 1] = s.soff[sl] + static_cast<std::uint32_t>(len * 32);
    }
    s.ent.assign(std::max<std::uint32_t>(s.soff[slices], 1), 0u);
    for (std::uint32_t v = 0; v < V; ++v) {
        const std::uint32_t sl = v / 32, lane = v % 32;
        for (std::size_t q = 0; q < vl[v].size(); ++q)
            s.ent[s.soff[sl] + q * 32 + lane] = vl[v][q];
    }
    return s;
}

// The first index e in [0, m) with bad(e), or m; large ranges are scanned
// on all of the host's cores.
template <class Bad>
std::uint32_t first_bad(std::uint32_t m, Bad bad) {
    std::uint32_t first = m;
#pragma omp parallel for reduction(min : first) schedule(static) if (m >= (1u << 16))
    for (std::int64_t e = 0; e < static_cast<std::int64_t>(m); ++e)
        if (bad(static_cast<std::uint32_t>(e)) && static_cast<std::uint32_t>(e) < first)
            first = static_cast<std::uint32_t>(e);
    return first;
}

int check_csr(const char* name, const asg_csr& c, std::uint32_t n_src, std::uint32_t n_tgt) {
    if (c.n_sources != n_src)
        return fail(ASG_ERR_ARG, "%s: n_sources %u, expected %u", name, c.n_sources, n_src);
    if (n_src > 0 && (c.row_start == nullptr))
        return fail(ASG_ERR_ARG, "%s: row_start is NULL", name);
    if (n_src == 0) return ASG_OK;
    if (c.row_start[0] != 0) return fail(ASG_ERR_ARG, "%s: row_start[0] != 0", name);
    const std::uint32_t s =
        first_bad(n_src, [&](std::uint32_t i) { return c.row_start[i + 1] < c.row_start[i]; });
    if (s < n_src) return fail(ASG_ERR_ARG, "%s: row_start decreases at %u", name, s);
    const std::uint32_t m = c.row_start[n_src];
    if (m > 0 && c.target == nullptr) return fail(ASG_ERR_ARG, "%s: target is NULL", name);
    const std::uint32_t e = first_bad(m, [&](std::uint32_t i) { return c.target[i] >= n_tgt; });
    if (e < m)
        return fail(ASG_ERR_ARG, "%s: target[%u] = %u out of range (%u)", name, e, c.target[e],
                    n_tgt);
    return ASG_OK;
}

int check_uniform(const char* name, const asg_csr& c, std::uint32_t n_src, double w, int d,
                  const asg_stp& stp) {
    if (n_src == 0) return ASG_OK;
    const std::uint32_t m = c.row_start[n_src];
    const std::uint32_t e = first_bad(m, [&](std::uint32_t i) {
        return (c.weight && c.weight[i] != w) || (c.delay_steps && c.delay_steps[i] != d);
    });
    if (e < m && c.weight && c.weight[e] != w)
        return fail(ASG_ERR_UNSUPPORTED,
                    "%s: per-edge weight %g differs from the set weight %g (the engine "
                    "takes one weight per set, as the reference builds them)",
                    name, c.weight[e], w);
    if (e < m)
        return fail(ASG_ERR_UNSUPPORTED, "%s: per-edge delay %d differs from the set delay %d",
                    name, c.delay_steps[e], d);
    if (stp.enabled && (c.stp_x || c.stp_u || c.stp_t_last)) {
        for (std::uint32_t s = 0; s < n_src; ++s) {
            for (std::uint32_t e = c.row_start[s]; e < c.row_start[s + 1]; ++e) {
                const std::uint32_t f = c.row_start[s];
                if ((c.stp_x && c.stp_x[e] != c.stp_x[f]) || (c.stp_u && c.stp_u[e] != c.stp_u[f]) ||
                    (c.stp_t_last && c.stp_t_last[e] != c.stp_t_last[f]))
                    return fail(ASG_ERR_UNSUPPORTED,
                                "%s: STP state differs along the row of source %u", name, s);
            }
        }
    }
    return ASG_OK;
}

bool all_equal(const double* a, std::uint32_t n) {
    for (std::uint32_t i = 1; i < n; ++i)
        if (std::memcmp(&a[i], &a[0], sizeof(double)) != 0) return false;
    return true;
}

// Arena layout: a list of (destination pointer, bytes, host source) entries
// placed at 256-byte boundaries in one allocation.
struct Seg {
    void* dst;  // address of the pointer field to set
    std::size_t bytes;
    const void* src;  // nullptr: zero-filled
};

std::size_t align256(std::size_t x) { return (x + 255) & ~static_cast<std::size_t>(255); }

}  // namespace

Instance::~Instance() {
    for (int p = 0; p < 2; ++p) {
        if (log_h[p]) cudaFreeHost(log_h[p]);
        if (rec_h[p]) cudaFreeHost(rec_h[p]);
    }
}

Engine::Engine(const EngineConfig& c) : cfg(c) {}

Engine::~Engine() {
    if (stream) cudaStreamSynchronize(stream);
    drop_graphs();
    for (int p = 0; p < 2; ++p) {
        if (h_insts[p]) cudaFreeHost(h_insts[p]);
        if (h_stats[p]) cudaFreeHost(h_stats[p]);
        if (h_barrier_err[p]) cudaFreeHost(h_barrier_err[p]);
        if (ev_chunk[p]) cudaEventDestroy(ev_chunk[p]);
        if (ev_chunk0[p]) cudaEventDestroy(ev_chunk0[p]);
    }
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_end) cudaEventDestroy(ev_end);
    if (ev_side_fork) cudaEventDestroy(ev_side_fork);
    if (ev_side_join) cudaEventDestroy(ev_side_join);
    for (int q = 0; q < kSideEvents; ++q) {
        if (ev_side_pre[q]) cudaEventDestroy(ev_side_pre[q]);
        if (ev_side_done[q]) cudaEventDestroy(ev_side_done[q]);
    }
    insts.clear();
    if (side) cudaStreamDestroy(side);
    if (upload) cudaStreamDestroy(upload);
    if (stream) cudaStreamDestroy(stream);
}

int Engine::init() {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return fail(ASG_ERR_NO_DEVICE, "no CUDA device visible");
    if (cfg.device < 0 || cfg.device >= count)
        return fail(ASG_ERR_ARG, "device %d out of range (%d devices)", cfg.device, count);
    ASG_CUDA(cudaSetDevice(cfg.device));
    ASG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cfg.device));
    if (cfg.chunk_steps <= 0) cfg.chunk_steps = 32;
    if (cfg.block <= 0) cfg.block = 128;
    if (cfg.block > 512 || cfg.block % 32 != 0)
        return fail(ASG_ERR_ARG, "block size %d must be a multiple of 32 in [32, 512]", cfg.block);
    if (cfg.mem_budget == 0) {
        std::size_t fr = 0, tot = 0;
        ASG_CUDA(cudaMemGetInfo(&fr, &tot));
        cfg.mem_budget = static_cast<std::uint64_t>(0.9 * static_cast<double>(fr));
    }
    ASG_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    ASG_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    ASG_CUDA(cudaStreamCreateWithFlags(&upload, cudaStreamNonBlocking));
    ASG_CUDA(cudaEventCreateWithFlags(&ev_side_fork, cudaEventDisableTiming));
    ASG_CUDA(cudaEventCreateWithFlags(&ev_side_join, cudaEventDisableTiming));
    for (int q = 0; q < kSideEvents; ++q) {
        ASG_CUDA(cudaEventCreateWithFlags(&ev_side_pre[q], cudaEventDisableTiming));
        ASG_CUDA(cudaEventCreateWithFlags(&ev_side_done[q], cudaEventDisableTiming));
    }
    ASG_CUDA(cudaEventCreate(&ev_start));
    ASG_CUDA(cudaEventCreate(&ev_end));
    for (int p = 0; p < 2; ++p) {
        ASG_CUDA(cudaEventCreate(&ev_chunk[p]));
        ASG_CUDA(cudaEventCreate(&ev_chunk0[p]));
        ASG_CUDA(cudaHostAlloc(&h_barrier_err[p], sizeof(unsigned), cudaHostAllocDefault));
        *h_barrier_err[p] = 0;
    }
    ASG_TRY(d_barrier.alloc(sizeof(GridBarrier)));
    return ASG_OK;
}

Instance* Engine::find(int id) {
    for (auto& p : insts)
        if (p->id == id) return p.get();
    return nullptr;
}

int Engine::footprint(const asg_network_desc& d, int chunk_steps, std::uint64_t* bytes) {
    // Upper estimate from sizes alone (no preprocessing), used for admission.
    const std::uint64_t N = d.n_exc + d.n_inh, NA = d.n_astro;
    const int md = std::max({1, d.d_e_steps, d.d_i_steps, d.d_a2n_steps});
    const std::uint64_t slots = md + 1;
    auto edges = [](const asg_csr& c) -> std::uint64_t {
        return c.n_sources && c.row_start ? c.row_start[c.n_sources] : 0;
    };
    const std::uint64_t Ee = edges(d.exc_primary), Ei = edges(d.inh_primary),
                        Ea = edges(d.neuron_astro), Es = edges(d.astro_neuron);
    std::uint64_t b = 0;
    b += N * (7 * 8 + 4 + 16 + 24) + NA * (7 * 8);  // state, params, STP
    const std::uint64_t words = (Ee + Ei + Ea) / 32 + 2 * N + NA;  // upper bound
    b += (Ee + Ei + Ea) * 9 + (N * 3 + NA) * 8;       // out lists, bit positions, word bases
    b += slots * words * (4 + 32 * 8) + slots * (2 * N + NA) * 8;  // bits, values, summaries
    b += slots * (2 * N + NA) * (4 + kListCap * 12);                // counters, short lists
    b += Es * 4 + N * 8 + slots * NA * 8 + 2 * N * 8;  // SIC (upper bound), factors, values
    b += (N + 32) * (kMaxSicParts * 8 + 2 * kMaxSicParts * 8);  // part cuts, partial sums
    b += N * 8 * kSicRing;                                        // SIC value ring
    b += 256 * 64;                                     // alignment slack
    (void)chunk_steps;
    *bytes = b;
    return ASG_OK;
}

int Engine::add(const asg_network_desc& d, const asg_record_opts* rec, std::int64_t first,
                std::int64_t end, bool keep_spikes, int* id_out) {
    std::unique_ptr<Instance> inst;
    ASG_TRY(prepare(d, rec, first, end, keep_spikes, true, &inst));
    return commit(std::move(inst), id_out);
}

int Engine::commit(std::unique_ptr<Instance> inst, int* id_out) {
    // The chunks in flight are collected before the instance list changes,
    // since they report statistics by instance position.
    ASG_TRY(finish_pending());
    inst->id = next_id++;
    resident_bytes += inst->arena_bytes;
    *id_out = inst->id;
    insts.push_back(std::move(inst));
    dirty = true;
    return ASG_OK;
}

int Engine::prepare(const asg_network_desc& d, const asg_record_opts* rec, std::int64_t first,
                    std::int64_t end, bool keep_spikes, bool check_budget,
                    std::unique_ptr<Instance>* out) {
    NvtxRange nvtx("admission: prepare instance");
    // Touches no state the chunks in flight use: the tables are prepared and
    // uploaded on the upload stream into a new arena, so a serving loop can
    // run this on another thread while the engine's stream keeps stepping.
    const std::uint32_t NE = d.n_exc, NI = d.n_inh, N = NE + NI, NA = d.n_astro;
    if (d.dt <= 0.0) return fail(ASG_ERR_ARG, "dt must be positive");
    if (d.substeps < 1) return fail(ASG_ERR_ARG, "substeps must be at least 1");
    if (d.sic_interval < 1) return fail(ASG_ERR_ARG, "sic_interval must be at least 1");
    if (!delay_ok(d.d_e_steps) || !delay_ok(d.d_i_steps) || !delay_ok(d.d_a2n_steps))
        return fail(ASG_ERR_ARG, "delays must be at least one step");
    if (NA >= (1u << 24)) return fail(ASG_ERR_UNSUPPORTED, "at most 2^24-1 astrocytes");
    if (NE + NI >= (1u << 25)) return fail(ASG_ERR_UNSUPPORTED, "at most 2^25-1 neurons");
    if (N > 0 && (d.V_reset == nullptr || d.b == nullptr))
        return fail(ASG_ERR_ARG, "per-cell V_reset and b are required");
    if (first < 0 || end < first) return fail(ASG_ERR_ARG, "bad step range");
    ASG_TRY(check_csr("exc_primary", d.exc_primary, NE, N));
    ASG_TRY(check_csr("inh_primary", d.inh_primary, NI, N));
    ASG_TRY(check_csr("neuron_astro", d.neuron_astro, NE, std::max(NA, 1u)));
    ASG_TRY(check_csr("astro_neuron", d.astro_neuron, NA, N));
    if (NA == 0 && d.neuron_astro.n_sources && d.neuron_astro.row_start &&
        d.neuron_astro.row_start[NE] > 0)
        return fail(ASG_ERR_ARG, "neuron_astro has edges but there are no astrocytes");
    ASG_TRY(check_uniform("exc_primary", d.exc_primary, NE, d.w_e, d.d_e_steps, d.stp));
    ASG_TRY(check_uniform("inh_primary", d.inh_primary, NI, d.w_i, d.d_i_steps, d.stp));
    ASG_TRY(check_uniform("neuron_astro", d.neuron_astro, NE, d.w_n2a, d.d_e_steps, d.stp));
    asg_stp nostp{};
    ASG_TRY(check_uniform("astro_neuron", d.astro_neuron, NA, d.w_a2n, d.d_a2n_steps, nostp));
    // Divisors taken through their host-rounded reciprocals (div_by) must lie
    // in the range where that division is exact: magnitudes in [2^-46, 2^63].
    {
        auto divisor_ok = [](double b) {
            const double m = std::fabs(b);
            return m >= 0x1p-46 && m <= 0x1p63;
        };
        const std::pair<const char*, double> neuron_div[] = {
            {"neuron_exc.C_m", d.exc.C_m},         {"neuron_exc.Delta_T", d.exc.Delta_T},
            {"neuron_exc.tau_w", d.exc.tau_w},     {"neuron_inh.C_m", d.inh.C_m},
            {"neuron_inh.Delta_T", d.inh.Delta_T}, {"neuron_inh.tau_w", d.inh.tau_w}};
        const std::pair<const char*, double> astro_div[] = {
            {"astrocyte.ratio_ER_cyt", d.astro.ratio_ER_cyt},
            {"astrocyte.tau_IP3", d.tau_IP3 == nullptr ? d.tau_IP3_u : 1.0}};
        for (const auto& dv : neuron_div)
            if (N > 0 && !divisor_ok(dv.second))
                return fail(ASG_ERR_UNSUPPORTED, "%s = %g outside [2^-46, 2^63]", dv.first,
                            dv.second);
        for (const auto& dv : astro_div)
            if (NA > 0 && !divisor_ok(dv.second))
                return fail(ASG_ERR_UNSUPPORTED, "%s = %g outside [2^-46, 2^63]", dv.first,
                            dv.second);
        if (d.stp.enabled && !divisor_ok(d.stp.tau_rec))
            return fail(ASG_ERR_UNSUPPORTED, "stp.tau_rec = %g outside [2^-46, 2^63]",
                        d.stp.tau_rec);
        if (d.stp.enabled && d.stp.tau_fac >= 1e-10 && !divisor_ok(d.stp.tau_fac))
            return fail(ASG_ERR_UNSUPPORTED, "stp.tau_fac = %g outside [2^-46, 2^63]",
                        d.stp.tau_fac);
        if (d.tau_IP3 != nullptr)
            for (std::uint32_t a = 0; a < NA; ++a)
                if (!divisor_ok(d.tau_IP3[a]))
                    return fail(ASG_ERR_UNSUPPORTED, "tau_IP3[%u] = %g outside [2^-46, 2^63]", a,
                                d.tau_IP3[a]);
        // Minuends of the astrocyte's divided differences (div_diff_by).
        auto diff_check = [NA](const char* name, const double* arr, double u) {
            if (NA == 0) return ASG_OK;
            if (arr == nullptr)
                return diff_param_ok(u) ? ASG_OK
                                        : fail(ASG_ERR_UNSUPPORTED, "%s = %g: magnitude must be "
                                               "in [2^-906, 2^976]", name, u);
            for (std::uint32_t a = 0; a < NA; ++a)
                if (!diff_param_ok(arr[a]))
                    return fail(ASG_ERR_UNSUPPORTED, "%s[%u] = %g: magnitude must be in "
                                "[2^-906, 2^976]", name, a, arr[a]);
            return ASG_OK;
        };
        ASG_TRY(diff_check("Ca_tot", d.Ca_tot, d.Ca_tot_u));
        ASG_TRY(diff_check("IP3_0", d.IP3_0, d.IP3_0_u));
    }

    auto inst = std::make_unique<Instance>();
    Instance& I = *inst;
    InstDev& D = I.dev;
    std::memset(&D, 0, sizeof D);
    D.N = N;
    D.NE = NE;
    D.NA = NA;
    D.d_e = d.d_e_steps;
    D.d_i = d.d_i_steps;
    D.d_a2n = d.d_a2n_steps;
    D.slots = std::max({1, D.d_e, D.d_i, D.d_a2n}) + 1;
    D.sic_interval = d.sic_interval;
    static const std::uint32_t zero_rs[1] = {0};
    auto rs_of = [](const asg_csr& c) { return c.n_sources ? c.row_start : zero_rs; };
    // SIC form.  A one-step delay needs the fused form.  In auto mode a
    // large network (N >= 2^16, or an instance of a batch of 2^16+ neurons
    // in all: the step's blocks fill the GPU more than twice, so it is
    // throughput-bound) with short SIC lists also sums each target's SIC in
    // its neuron thread, which saves the SIC role's blocks (a third of the
    // step's); a smaller network keeps the SIC role, which runs beside the
    // neuron role (lower latency).
    const std::uint32_t sic_mx =
        NA > 0 ? sic_max_edges(NA, rs_of(d.astro_neuron), d.astro_neuron.target, N) : 0;
    const bool fuse_auto =
        D.d_a2n < 2 || ((N >= (1u << 16) || cfg.large_total) && sic_mx <= kSicEdgesPerPart);
    D.fused_sic = cfg.sic_mode == 1 ? 1 : cfg.sic_mode == 2 ? (D.d_a2n >= 2 ? 0 : 1)
                                                            : (fuse_auto ? 1 : 0);
    D.stp_on = d.stp.enabled != 0;
    // Deferred push needs both spike delays >= 2 steps (the push of step s
    // runs in step s+1 and must land before step s+d reads it).
    D.deferred_push = (cfg.push_mode != 1 && d.d_e_steps >= 2 && d.d_i_steps >= 2) ? 1 : 0;
    // One push block per kPushCells neurons, at most two per SM: the grid
    // of a step (push, SIC parts, neurons, astrocytes) should fit the GPU in
    // one wave; a burst is spread over the blocks' threads by striding.
    D.push_blocks = static_cast<std::int32_t>(std::min<std::uint32_t>(
        2u * static_cast<std::uint32_t>(sms),
        std::max<std::uint32_t>(1, (N + kPushCells - 1) / kPushCells)));
    D.seed = d.seed;
    D.dt = d.dt;
    const double h = d.dt / static_cast<double>(d.substeps);
    D.pe = make_neuron_k(d.exc, d.input_exc, d.dt, h);
    D.pi = make_neuron_k(d.inh, d.input_inh, d.dt, h);
    D.ak = make_astro_k(d.astro, h, d.substeps);
    D.a_rate = d.input_astro.poiss_rate;
    D.a_weight = d.input_astro.poiss_weight;
    D.a_lambda = d.input_astro.poiss_rate * d.dt * 1e-3;
    D.a_limit = std::exp(-D.a_lambda);
    D.a_std = d.input_astro.gauss_noise_std;
    D.a_indep = d.input_astro.independent_noise != 0;
    D.a_steps_per_noise =
        std::max(1, static_cast<int>(std::llround(d.input_astro.noise_dt / d.dt)));
    D.SIC_scale = d.astro.SIC_scale;
    D.SIC_th = d.astro.SIC_th;
    D.w_e = d.w_e;
    D.w_i = d.w_i;
    D.w_n2a = d.w_n2a;
    D.w_a2n = d.w_a2n;
    D.U = d.stp.U;
    D.tau_rec = d.stp.tau_rec;
    D.tau_fac = d.stp.tau_fac;
    D.inv_tau_rec = 1.0 / d.stp.tau_rec;
    D.inv_tau_fac = d.stp.tau_fac > 0.0 ? 1.0 / d.stp.tau_fac : 0.0;

    // Per-cell astrocyte parameters collapse to scalars when all equal.
    const double* pa[4] = {d.Ca_tot, d.IP3_0, d.tau_IP3, d.delta_IP3};
    const double pu[4] = {d.Ca_tot_u, d.IP3_0_u, d.tau_IP3_u, d.delta_IP3_u};
    bool uniform = true;
    double uval[4];
    for (int k = 0; k < 4; ++k) {
        if (pa[k] == nullptr) {
            uval[k] = pu[k];
        } else if (NA > 0 && all_equal(pa[k], NA)) {
            uval[k] = pa[k][0];
        } else if (NA > 0) {
            uniform = false;
            uval[k] = 0.0;
        } else {
            uval[k] = pu[k];
        }
    }
    D.astro_uniform = uniform ? 1 : 0;
    D.astro_fp32 = cfg.astro_fp32 ? 1 : 0;
    D.Ca_tot_u = uval[0];
    D.IP3_0_u = uval[1];
    D.tau_u = uval[2];
    D.delta_u = uval[3];
    D.inv_tau_u = 1.0 / uval[2];

    // Host preprocessing of the tables.
    InRingDev rex, rin, ras;
    ASG_TRY(build_in_ring(NE, rs_of(d.exc_primary), d.exc_primary.target, N, upload, rex));
    ASG_TRY(build_in_ring(NI, rs_of(d.inh_primary), d.inh_primary.target, N, upload, rin));
    ASG_TRY(build_in_ring(NE, rs_of(d.neuron_astro), d.neuron_astro.target, NA, upload, ras));
    // SIC parts: about kSicEdgesPerPart edges each, at most d_a2n - 1 (the
    // first part of arrival step A runs at step A - P and reads the factors
    // of step A - d_a2n, written by an earlier launch).
    D.sic_npad = (N + 31) / 32 * 32;
    D.sic_parts = 1;
    // Side-stream SIC batches need a delay that leaves a few steps between
    // a batch and its first reader (lead >= 4); sic_mode 2 keeps the
    // in-kernel parts.
    D.sic_side = (!D.fused_sic && cfg.sic_mode != 2 && NA > 0 &&
                  D.d_a2n >= kSicBatchSteps + 4) ? 1 : 0;
    D.sic_lead = D.sic_side ? std::min(D.d_a2n - kSicBatchSteps, kSicRing - kSicBatchSteps - 8) : 0;
    D.sic_ring = D.sic_side ? kSicRing : 2;
    if (!D.fused_sic && !D.sic_side) {
        const int want = static_cast<int>((sic_mx + kSicEdgesPerPart - 1) / kSicEdgesPerPart);
        D.sic_parts = std::max(1, std::min({want, kMaxSicParts, D.d_a2n - 1}));
    }
    SicHost sic = make_sic(NA, rs_of(d.astro_neuron), d.astro_neuron.target, N,
                           static_cast<std::uint32_t>(D.sic_parts), D.sic_npad);

    // Initial state (reference defaults where not given).
    std::vector<double> V0, Ca0, IP30, h0, stp_x(N, 1.0), stp_u(N, d.stp.U), stp_t(N, -1e12);
    if (d.V == nullptr) {
        V0.resize(N);
        for (std::uint32_t i = 0; i < N; ++i) V0[i] = i < NE ? d.V_m_init_exc : d.V_m_init_inh;
    }
    if (d.Ca == nullptr) Ca0.assign(NA, d.Ca_init);
    if (d.IP3 == nullptr) IP30.assign(NA, d.IP3_init);
    if (d.h == nullptr) h0.assign(NA, d.h_init);
    // Per-source STP from the first edge of each row, if the caller gave state.
    auto take_stp = [&](const asg_csr& c, std::uint32_t n_src, std::uint32_t off) {
        if (!d.stp.enabled || n_src == 0) return;
        for (std::uint32_t s = 0; s < n_src; ++s) {
            const std::uint32_t e = c.row_start[s];
            if (e == c.row_start[s + 1]) continue;
            if (c.stp_x) stp_x[off + s] = c.stp_x[e];
            if (c.stp_u) stp_u[off + s] = c.stp_u[e];
            if (c.stp_t_last) stp_t[off + s] = c.stp_t_last[e];
        }
    };
    take_stp(d.neuron_astro, NE, 0);
    take_stp(d.exc_primary, NE, 0);
    take_stp(d.inh_primary, NI, NE);

    const std::size_t S = static_cast<std::size_t>(D.slots);
    const std::size_t n8 = static_cast<std::size_t>(N) * 8, a8 = static_cast<std::size_t>(NA) * 8;
    std::vector<Seg> segs;
    auto add_seg = [&](auto*& dst, std::size_t bytes, const void* src) {
        segs.push_back(Seg{static_cast<void*>(&dst), bytes, src});
    };
    add_seg(D.V, n8, d.V ? d.V : V0.data());
    add_seg(D.w, n8, d.w);
    add_seg(D.gex, n8, d.g_ex);
    add_seg(D.dgex, n8, d.dg_ex);
    add_seg(D.gin, n8, d.g_in);
    add_seg(D.dgin, n8, d.dg_in);
    add_seg(D.Isic, n8, d.I_sic);
    add_seg(D.refr, static_cast<std::size_t>(N) * 4, d.refractory);
    add_seg(D.V_reset, n8, d.V_reset);
    add_seg(D.b, n8, d.b);
    add_seg(D.Ca, a8, d.Ca ? d.Ca : Ca0.data());
    add_seg(D.IP3, a8, d.IP3 ? d.IP3 : IP30.data());
    add_seg(D.h, a8, d.h ? d.h : h0.data());
    std::vector<double> inv_tau;
    if (!uniform) {
        inv_tau.resize(NA);
        for (std::uint32_t i = 0; i < NA; ++i) inv_tau[i] = 1.0 / d.tau_IP3[i];
        add_seg(D.Ca_tot, a8, d.Ca_tot);
        add_seg(D.IP3_0, a8, d.IP3_0);
        add_seg(D.tau, a8, d.tau_IP3);
        add_seg(D.inv_tau, a8, inv_tau.data());
        add_seg(D.delta, a8, d.delta_IP3);
    }
    add_seg(D.stp_x, n8, stp_x.data());
    add_seg(D.stp_u, n8, stp_u.data());
    add_seg(D.stp_t, n8, stp_t.data());
    add_seg(D.exc_rs, (NE + 1) * 4, d.exc_primary.n_sources ? d.exc_primary.row_start : zero_rs);
    add_seg(D.inh_rs, (NI + 1) * 4, d.inh_primary.n_sources ? d.inh_primary.row_start : zero_rs);
    add_seg(D.n2a_rs, (NE + 1) * 4, d.neuron_astro.n_sources ? d.neuron_astro.row_start : zero_rs);
    auto ring_segs = [&](InRing& R, InRingDev& H, std::uint32_t n_t) {
        const std::size_t W = std::max<std::uint32_t>(H.words, 1);
        add_seg(R.wbase, (static_cast<std::size_t>(n_t) + 1) * 4, H.wbase.p);  // device copies
        add_seg(R.edge, static_cast<std::size_t>(H.m) * 8, H.edge.p);
        const std::size_t T = std::max<std::uint32_t>(n_t, 1);
        add_seg(R.cnt, S * T * 4, nullptr);
        add_seg(R.lbit, S * T * kListCap * 4, nullptr);
        add_seg(R.lval, S * T * kListCap * 8, nullptr);
        add_seg(R.bits, S * W * 4, nullptr);
        add_seg(R.sum, S * std::max<std::uint32_t>(n_t, 1) * 8, nullptr);
        add_seg(R.vals, S * W * 32 * 8, nullptr);
        R.words = H.words;
        R.n_targets = n_t;
    };
    ring_segs(D.ring_ex, rex, N);
    ring_segs(D.ring_in, rin, N);
    ring_segs(D.ring_as, ras, NA);

    add_seg(D.spk_packed, 3 * kHeaderStride * 8, nullptr);
    add_seg(D.spk_meta, 3 * std::max<std::size_t>(N, 1) * 16, nullptr);
    add_seg(D.spk_val, 3 * std::max<std::size_t>(N, 1) * 16, nullptr);
    add_seg(D.sic_soff, sic.soff.size() * 4, sic.soff.data());
    add_seg(D.sic_ent, sic.ent.size() * 4, sic.ent.data());
    add_seg(D.fac, S * std::max<std::size_t>(a8, 8), nullptr);
    add_seg(D.fac_any, (S + 1) * 4, nullptr);
    add_seg(D.noise_n, n8, nullptr);
    add_seg(D.noise_a, a8, nullptr);
    add_seg(D.sic_part,
            2 * static_cast<std::size_t>(std::max(D.sic_parts - 1, 1)) * D.sic_npad * 8, nullptr);
    add_seg(D.sic_val, static_cast<std::size_t>(D.sic_ring) * std::max<std::size_t>(n8, 8), nullptr);

    std::size_t total = 0;
    for (const Seg& s : segs) total += align256(std::max<std::size_t>(s.bytes, 1));
    if (check_budget && resident_bytes + total > cfg.mem_budget)
        return fail(ASG_ERR_OOM, "instance needs %zu device bytes; %llu of %llu in use", total,
                    static_cast<unsigned long long>(resident_bytes),
                    static_cast<unsigned long long>(cfg.mem_budget));
    ASG_TRY(I.arena.alloc(total, false));
    I.arena_bytes = total;
    {
        char* base = I.arena.as<char>();
        std::size_t off = 0;
        std::vector<char> zeros;
        for (const Seg& s : segs) {
            *static_cast<void**>(s.dst) = base + off;
            if (s.bytes > 0) {
                if (s.src != nullptr) {
                    // host tables and the device-built rings alike (unified addressing)
                    ASG_CUDA(cudaMemcpyAsync(base + off, s.src, s.bytes, cudaMemcpyDefault,
                                             upload));
                } else {
                    ASG_CUDA(cudaMemsetAsync(base + off, 0, s.bytes, upload));
                }
            }
            off += align256(std::max<std::size_t>(s.bytes, 1));
        }
        ASG_CUDA(cudaStreamSynchronize(upload));  // host sources go out of scope
    }

    // Recording and spike-log buffers (mapped host memory, two parities).
    asg_record_opts ro{};
    if (rec) ro = *rec;
    if (ro.record_every < 1) ro.record_every = 1;
    D.rec_spikes = ro.spikes ? 1 : 0;
    D.rec_from = ro.record_from_step;
    D.rec_every = ro.record_every;
    D.rec_astro_max = std::min(ro.astro_max, NA);
    D.rec_neuron_max = std::min(ro.neuron_max, N);
    I.rec_rows = static_cast<std::uint32_t>(cfg.chunk_steps / ro.record_every + 2);
    D.rec_rows = I.rec_rows;
    const std::uint64_t full = static_cast<std::uint64_t>(N) * cfg.chunk_steps;
    I.log_cap = static_cast<std::uint32_t>(
        std::max<std::uint64_t>(1, std::min<std::uint64_t>(full, std::max<std::uint64_t>(
                                                                     65536, full / 8))));
    I.keep_spikes = keep_spikes;
    I.max_chunk = cfg.chunk_steps;
    const std::size_t rec_doubles =
        static_cast<std::size_t>(I.rec_rows) * (2 * D.rec_astro_max + 2 * D.rec_neuron_max) + 1;
    for (int p = 0; p < 2; ++p) {
        if (D.rec_spikes) {
            ASG_CUDA(cudaHostAlloc(&I.log_h[p], static_cast<std::size_t>(I.log_cap) * 8,
                                   cudaHostAllocMapped));
            ASG_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&I.log_d[p]), I.log_h[p], 0));
        }
        ASG_CUDA(cudaHostAlloc(&I.rec_h[p], rec_doubles * 8, cudaHostAllocMapped));
        ASG_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&I.rec_d[p]), I.rec_h[p], 0));
    }
    D.spike_log_cap = D.rec_spikes ? I.log_cap : 0;
    D.noise_from = first;  // the noise-term caches hold nothing yet
    I.step = first;
    I.end = end;
    *out = std::move(inst);
    return ASG_OK;
}

int Engine::remove(int id) {
    ASG_TRY(finish_pending());  // pending statistics are indexed by position
    for (std::size_t i = 0; i < insts.size(); ++i) {
        if (insts[i]->id == id) {
            ASG_CUDA(cudaStreamSynchronize(stream));
            resident_bytes -= insts[i]->arena_bytes;
            insts.erase(insts.begin() + static_cast<std::ptrdiff_t>(i));
            dirty = true;
            return ASG_OK;
        }
    }
    return fail(ASG_ERR_NOT_FOUND, "no instance %d", id);
}

int Engine::set_block(int block) {
    if (block < 32 || block > 512 || block % 32)
        return fail(ASG_ERR_ARG, "block size %d must be a multiple of 32 in [32, 512]", block);
    cfg.block = block;
    dirty = true;
    return ASG_OK;
}

int Engine::set_mode(int use_graphs) {
    if (use_graphs != -1 && use_graphs != 0 && use_graphs != 1 && use_graphs != 2)
        return fail(ASG_ERR_ARG, "launch mode %d is not -1, 0, 1 or 2", use_graphs);
    cfg.use_graphs = use_graphs;
    dirty = true;
    return ASG_OK;
}

int Engine::set_chunk(int chunk) {
    if (chunk < 1) return fail(ASG_ERR_ARG, "chunk must be >= 1");
    // Output buffers were sized for the chunk in force when each instance
    // was added; a longer chunk could overrun them.
    for (auto& p : insts)
        if (chunk > p->max_chunk)
            return fail(ASG_ERR_ARG, "chunk %d exceeds %d, the chunk instance %d was sized for",
                        chunk, p->max_chunk, p->id);
    cfg.chunk_steps = chunk;
    dirty = true;
    return ASG_OK;
}

int Engine::rebuild() {
    ASG_TRY(finish_pending());
    ASG_CUDA(cudaStreamSynchronize(stream));
    drop_graphs();
    const int B = cfg.block;
    work.clear();
    order.clear();
    // Push and SIC blocks first (longest dependent chains), then neurons, then
    // astrocytes.  A PUSH item's `first` is its index among the instance's
    // push blocks.
    std::vector<std::uint32_t> helpers(insts.size(), 0);
    for (int role = 0; role < 4; ++role) {
        for (std::size_t s = 0; s < insts.size(); ++s) {
            const InstDev& D = insts[s]->dev;
            const std::uint16_t r = role == 0   ? kRolePush
                                    : role == 1 ? kRoleSic
                                    : role == 2 ? kRoleNeuron
                                                : kRoleAstro;
            if (r == kRoleSic && (D.fused_sic || (D.sic_side && cfg.use_graphs != 2))) continue;
            if (r == kRolePush) {
                if (!D.deferred_push) continue;
                for (int pb = 0; pb < D.push_blocks; ++pb)
                    work.push_back(Work{static_cast<std::uint32_t>(s), r, kNoHelper,
                                        static_cast<std::uint32_t>(pb), 0});
                continue;
            }
            const std::uint32_t n = r == kRoleAstro ? D.NA
                                    : r == kRoleSic ? static_cast<std::uint32_t>(D.sic_parts) * D.sic_npad
                                                    : D.N;
            for (std::uint32_t f = 0; f < n; f += B) {
                const std::uint16_t h = D.deferred_push && helpers[s] < kNoHelper
                                            ? static_cast<std::uint16_t>(helpers[s]++)
                                            : kNoHelper;
                work.push_back(Work{static_cast<std::uint32_t>(s), r, h, f,
                                    std::min<std::uint32_t>(B, n - f)});
            }
        }
    }
    for (std::size_t s = 0; s < insts.size(); ++s)
        insts[s]->dev.push_helpers = static_cast<std::int32_t>(helpers[s]);
    // Side-stream SIC batches (graph and plain launches; the persistent
    // kernel computes the single-part sums in its SIC role instead).
    side_work.clear();
    side_lead = 0;
    side_lead_max = 0;
    side_prime = true;
    if (cfg.use_graphs != 2) {
        for (std::size_t s = 0; s < insts.size(); ++s) {
            const InstDev& D = insts[s]->dev;
            if (!D.sic_side) continue;
            side_lead = side_lead == 0 ? D.sic_lead : std::min(side_lead, D.sic_lead);
            side_lead_max = std::max(side_lead_max, static_cast<int>(D.sic_lead));
            for (std::uint32_t f = 0; f < D.N; f += B)
                side_work.push_back(Work{static_cast<std::uint32_t>(s), kRoleSic, kNoHelper, f,
                                         std::min<std::uint32_t>(B, D.N - f)});
        }
    }
    if (insts.size() > cap_insts || work.size() * sizeof(Work) > d_work.bytes()) {
        const std::size_t cap = std::max<std::size_t>(insts.size(), 1);
        if (cap > cap_insts) {
            const std::size_t c2 = std::max(cap, cap_insts * 2);
            ASG_TRY(d_insts.alloc(c2 * sizeof(InstDev)));
            ASG_TRY(d_stats.alloc(c2 * 8 * sizeof(unsigned long long)));
            for (int p = 0; p < 2; ++p) {
                if (h_insts[p]) cudaFreeHost(h_insts[p]);
                if (h_stats[p]) cudaFreeHost(h_stats[p]);
                h_insts[p] = nullptr;
                h_stats[p] = nullptr;
                ASG_CUDA(cudaHostAlloc(&h_insts[p], c2 * sizeof(InstDev), cudaHostAllocDefault));
                ASG_CUDA(cudaHostAlloc(&h_stats[p], c2 * 8 * sizeof(unsigned long long),
                                       cudaHostAllocDefault));
            }
            cap_insts = c2;
        }
        if (work.size() * sizeof(Work) > d_work.bytes())
            ASG_TRY(d_work.alloc(std::max<std::size_t>(work.size(), 64) * 2 * sizeof(Work)));
    }
    if (!work.empty())
        ASG_CUDA(cudaMemcpyAsync(d_work.get(), work.data(), work.size() * sizeof(Work),
                                 cudaMemcpyHostToDevice, stream));
    if (side_work.size() * sizeof(Work) > d_side_work.bytes())
        ASG_TRY(d_side_work.alloc(side_work.size() * 2 * sizeof(Work)));
    if (!side_work.empty())
        ASG_CUDA(cudaMemcpyAsync(d_side_work.get(), side_work.data(),
                                 side_work.size() * sizeof(Work), cudaMemcpyHostToDevice, stream));
    ASG_CUDA(cudaMemsetAsync(d_stats.get(), 0, cap_insts * 8 * sizeof(unsigned long long), stream));
    ASG_CUDA(cudaStreamSynchronize(stream));
    // Step kernel form: a step of more than two waves of the latency form
    // (4 blocks of 128 threads per SM) is throughput-bound, and the
    // high-occupancy form (6 blocks per SM, some spilled registers) runs it
    // faster; a smaller step is bound by its dependent round trips, which
    // the latency form keeps fewest.
    wide = cfg.block == 128 &&
           (cfg.occupancy == 2 ||
            (cfg.occupancy == 0 && work.size() > static_cast<std::size_t>(2 * 4 * sms)));
    // The high-occupancy form runs as one wave of resident blocks, each
    // taking several work items (no per-item block launch or descriptor
    // staging after its first).
    wide_grid = 0;
    if (wide && cfg.item_loop) {
        const int nb = step_wide_blocks_per_sm();
        if (nb > 0) wide_grid = nb * sms;
    }
    persistent_grid = 0;
    if (cfg.use_graphs == 2 && !work.empty()) {
        const int cap = persistent_blocks(B);
        if (cap <= 0) return fail(ASG_ERR_CUDA, "persistent kernel: no co-resident blocks");
        persistent_grid = std::min<int>(cap, static_cast<int>(work.size()));
    }
    dirty = false;
    if (graph_mode() && !work.empty()) ASG_TRY(capture_graph(cfg.chunk_steps));
    return ASG_OK;
}

void Engine::drop_graphs() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    graphs.clear();
}

cudaGraphExec_t Engine::find_graph(int steps) {
    for (std::size_t i = 0; i < graphs.size(); ++i) {
        if (graphs[i].first != steps) continue;
        std::rotate(graphs.begin(), graphs.begin() + static_cast<std::ptrdiff_t>(i),
                    graphs.begin() + static_cast<std::ptrdiff_t>(i) + 1);
        return graphs.front().second;
    }
    return nullptr;
}

// The graph of a chunk of `steps` steps, captured unless cached.  Capturing
// waits for the chunks in flight, so the streams it records on are idle.
int Engine::capture_graph(int steps) {
    if (find_graph(steps) != nullptr) return ASG_OK;
    ASG_TRY(finish_pending());
    ASG_CUDA(cudaStreamSynchronize(stream));
    if (side) ASG_CUDA(cudaStreamSynchronize(side));
    cudaGraph_t g = nullptr;
    ASG_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    const cudaError_t le = issue_steps(steps);
    const cudaError_t ce = cudaStreamEndCapture(stream, &g);
    if (le != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return cuda_fail(le, "step launch (capture)", __FILE__, __LINE__);
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "graph capture", __FILE__, __LINE__);
    cudaGraphExec_t x = nullptr;
    const cudaError_t ci = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (ci != cudaSuccess) return cuda_fail(ci, "graph instantiate", __FILE__, __LINE__);
    if (graphs.size() == kMaxGraphs) {
        cudaGraphExecDestroy(graphs.back().second);
        graphs.pop_back();
    }
    graphs.insert(graphs.begin(), {steps, x});
    return ASG_OK;
}

// The launches of `steps` steps on the engine stream, with the side-stream
// SIC batches: before step k (k a multiple of kSicBatchSteps) the side stream
// waits for the steps before k and runs the batch for the arrival steps
// step0+k+lead..; the step k+lead (the first reader, lead the smallest over
// the instances) waits for that batch.  The side stream joins the engine
// stream at the end, so nothing of a chunk outlives it.  The first step of a
// chunk follows the descriptor copy: no early (programmatic) launch for it.
cudaError_t Engine::issue_steps(int steps) {
    NvtxRange nvtx("step chain: arrival application, background input, update astrocytes, "
                   "update neurons, spike delivery, SIC gather+deliver");
    const bool side_on = !side_work.empty();
    const int G = kSicBatchSteps;
    cudaError_t e = cudaSuccess;
    if (side_on) {
        e = cudaEventRecord(ev_side_fork, stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(side, ev_side_fork, 0);
    }
    for (int k = 0; k < steps && e == cudaSuccess; ++k) {
        if (side_on && k % G == 0) {
            cudaEvent_t before = ev_side_pre[(k / G) % kSideEvents];
            cudaEvent_t done = ev_side_done[(k / G) % kSideEvents];
            e = cudaEventRecord(before, stream);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(side, before, 0);
            if (e == cudaSuccess)
                e = launch_sic_batch(d_insts.as<InstDev>(), d_side_work.as<Work>(),
                                     static_cast<int>(side_work.size()), cfg.block, k, side);
            if (e == cudaSuccess) e = cudaEventRecord(done, side);
        }
        // (A step that waits for a batch still launches early: it reads the
        // SIC values after griddepcontrol.wait, and the batch is a completed
        // prerequisite by then whichever way the wait is honoured.)
        if (side_on && k >= side_lead && (k - side_lead) % G == 0 && e == cudaSuccess)
            e = cudaStreamWaitEvent(stream, ev_side_done[((k - side_lead) / G) % kSideEvents], 0);
        if (e == cudaSuccess)
            e = launch_step(d_insts.as<InstDev>(), d_work.as<Work>(), static_cast<int>(work.size()),
                            cfg.block, k, cfg.pdl && k > 0, wide, wide_grid, cfg.astro_fp32,
                            stream);
    }
    if (side_on && e == cudaSuccess) {
        e = cudaEventRecord(ev_side_join, side);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, ev_side_join, 0);
    }
    return e;
}

// SIC values of the arrival steps step0 .. step0+lead-1 of every side
// instance, before the chunk's own batches take over (batches with k < 0;
// arrivals before step0 are skipped in the kernel).
cudaError_t Engine::prime_side() {
    const int G = kSicBatchSteps;
    cudaError_t e = cudaEventRecord(ev_side_fork, stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(side, ev_side_fork, 0);
    const int first = -((side_lead_max + G - 1) / G) * G;
    for (int k = first; k < 0 && e == cudaSuccess; k += G)
        e = launch_sic_batch(d_insts.as<InstDev>(), d_side_work.as<Work>(),
                             static_cast<int>(side_work.size()), cfg.block, k, side);
    if (e == cudaSuccess) e = cudaEventRecord(ev_side_join, side);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, ev_side_join, 0);
    return e;
}

int Engine::launch_chunk(int parity, int steps) {
    // Stage the descriptors: step window of this chunk, output pointers.
    InstDev* hi = h_insts[parity];
    for (std::size_t s = 0; s < insts.size(); ++s) {
        Instance& I = *insts[s];
        InstDev D = I.dev;
        D.step0 = I.step;
        D.end_step = std::min<std::int64_t>(I.end, I.step + steps);
        unsigned long long* st = d_stats.as<unsigned long long>() + s * 8;
        D.spike_log_n = st;
        D.counters = st + 1;
        D.spike_log = I.log_d[parity];
        double* r = I.rec_d[parity];
        const std::size_t R = I.rec_rows;
        D.rec_Ca = r;
        D.rec_IP3 = r + R * D.rec_astro_max;
        D.rec_V = r + 2 * R * D.rec_astro_max;
        D.rec_Isic = r + 2 * R * D.rec_astro_max + R * D.rec_neuron_max;
        hi[s] = D;
        I.chunk_first[parity] = I.step;
        I.chunk_last[parity] = D.end_step;
    }
    ASG_CUDA(cudaEventRecord(ev_chunk0[parity], stream));
    ASG_CUDA(cudaMemcpyAsync(d_insts.get(), hi, insts.size() * sizeof(InstDev),
                             cudaMemcpyHostToDevice, stream));
    if (side_prime) {
        if (!side_work.empty()) ASG_CUDA(prime_side());
        side_prime = false;
    }
    if (persistent_grid > 0) {
        ASG_CUDA(cudaMemsetAsync(d_barrier.get(), 0, sizeof(GridBarrier), stream));
        ASG_CUDA(launch_chunk_persistent(d_insts.as<InstDev>(), d_work.as<Work>(),
                                         static_cast<int>(work.size()), cfg.block,
                                         persistent_grid, steps, d_barrier.as<GridBarrier>(),
                                         cfg.astro_fp32, stream));
        ASG_CUDA(cudaMemcpyAsync(h_barrier_err[parity], &d_barrier.as<GridBarrier>()->error,
                                 sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    } else if (cudaGraphExec_t g = graph_mode() ? find_graph(steps) : nullptr) {
        ASG_CUDA(cudaGraphLaunch(g, stream));
    } else {
        ASG_CUDA(issue_steps(steps));
    }
    const int launched = persistent_grid > 0 ? 1 : steps;
    last_kernels += launched;
    launched_kernels += launched;
    ASG_CUDA(cudaMemcpyAsync(h_stats[parity], d_stats.get(),
                             insts.size() * 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             stream));
    ASG_CUDA(cudaMemsetAsync(d_stats.get(), 0, insts.size() * 8 * sizeof(unsigned long long),
                             stream));
    ASG_CUDA(cudaEventRecord(ev_chunk[parity], stream));
    pending[parity] = true;
    launched_insts[parity] = insts.size();
    for (auto& p : insts) p->step = std::min<std::int64_t>(p->end, p->step + steps);
    return ASG_OK;
}

int Engine::collect(int parity) {
    NvtxRange nvtx("collect: spikes and recorded rows to the recorder");
    if (!pending[parity]) return ASG_OK;
    ASG_CUDA(cudaEventSynchronize(ev_chunk[parity]));
    pending[parity] = false;
    float chunk_ms = 0.0f;
    if (cudaEventElapsedTime(&chunk_ms, ev_chunk0[parity], ev_chunk[parity]) == cudaSuccess)
        chunk_device_ms += chunk_ms;
    if (*h_barrier_err[parity] != 0) {
        *h_barrier_err[parity] = 0;
        return fail(ASG_ERR_TIMEOUT,
                    "persistent step kernel: a grid barrier wait gave up; the chunk's results "
                    "are invalid");
    }
    const unsigned long long* st = h_stats[parity];
    const std::size_t n_launched = std::min(insts.size(), launched_insts[parity]);
    for (std::size_t s = 0; s < n_launched; ++s) {
        Instance& I = *insts[s];
        const InstDev& D = I.dev;
        const unsigned long long* c = st + s * 8;
        if (c[4] != 0)
            return fail(ASG_ERR_OVERFLOW,
                        "instance %d: %llu spikes did not fit the %u-entry chunk log; use a "
                        "smaller chunk_steps",
                        I.id, c[4], I.log_cap);
        I.spike_edges += static_cast<std::int64_t>(c[1]);
        I.sic_edges += static_cast<std::int64_t>(c[2]);
        I.n_spikes += static_cast<std::int64_t>(c[3]);
        if (D.rec_spikes && I.keep_spikes) {
            const std::uint64_t n = std::min<std::uint64_t>(c[0], I.log_cap);
            const unsigned long long* lg = I.log_h[parity];
            const std::size_t base = I.spikes.size();
            I.spikes.resize(base + n);
            for (std::uint64_t q = 0; q < n; ++q)
                I.spikes[base + q] = SpikeRec{static_cast<std::int64_t>(lg[q] >> 32),
                                              static_cast<std::uint32_t>(lg[q] & 0xFFFFFFFFu)};
            std::sort(I.spikes.begin() + static_cast<std::ptrdiff_t>(base), I.spikes.end(),
                      [](const SpikeRec& a, const SpikeRec& b) {
                          return a.step != b.step ? a.step < b.step : a.source < b.source;
                      });
        }
        // Record rows written in this chunk.
        const std::int64_t f = I.chunk_first[parity], l = I.chunk_last[parity];
        if ((D.rec_astro_max || D.rec_neuron_max) && l > f) {
            const std::size_t R = I.rec_rows;
            const double* r = I.rec_h[parity];
            for (std::int64_t s2 = std::max<std::int64_t>(f, D.rec_from); s2 < l; ++s2) {
                if ((s2 - D.rec_from) % D.rec_every != 0) continue;
                const std::size_t row = static_cast<std::size_t>(((s2 - D.rec_from) / D.rec_every) % R);
                if (D.rec_astro_max) {
                    I.astro_rec_steps.push_back(s2);
                    const double* ca = r + row * D.rec_astro_max;
                    const double* ip = r + R * D.rec_astro_max + row * D.rec_astro_max;
                    I.rec_Ca.insert(I.rec_Ca.end(), ca, ca + D.rec_astro_max);
                    I.rec_IP3.insert(I.rec_IP3.end(), ip, ip + D.rec_astro_max);
                }
                if (D.rec_neuron_max) {
                    I.neuron_rec_steps.push_back(s2);
                    const double* v = r + 2 * R * D.rec_astro_max + row * D.rec_neuron_max;
                    const double* is = r + 2 * R * D.rec_astro_max + R * D.rec_neuron_max +
                                       row * D.rec_neuron_max;
                    I.rec_V.insert(I.rec_V.end(), v, v + D.rec_neuron_max);
                    I.rec_Isic.insert(I.rec_Isic.end(), is, is + D.rec_neuron_max);
                }
            }
        }
    }
    return ASG_OK;
}

int Engine::finish_pending() {
    for (int k = 0; k < 2; ++k) ASG_TRY(collect((next_parity + k) & 1));
    return ASG_OK;
}

int Engine::run_chunk(std::int64_t max_steps) {
    if (dirty) ASG_TRY(rebuild());
    std::int64_t steps = 0;
    for (auto& p : insts) steps = std::max<std::int64_t>(steps, p->end - p->step);
    steps = std::min<std::int64_t>({steps, max_steps, cfg.chunk_steps});
    if (steps <= 0 || work.empty()) return ASG_OK;
    // Two chunks in flight: the host collects one while the next runs.
    const int p = next_parity;
    ASG_TRY(collect(p));
    ASG_TRY(launch_chunk(p, static_cast<int>(steps)));
    next_parity ^= 1;
    ++chunks;
    return ASG_OK;
}

int Engine::run(std::int64_t n_steps) {
    NvtxRange nvtx("Network::run (engine)");
    if (n_steps < 0) return fail(ASG_ERR_ARG, "negative step count");
    if (dirty) ASG_TRY(rebuild());
    last_kernels = 0;
    std::vector<std::int64_t> target(insts.size());
    for (std::size_t s = 0; s < insts.size(); ++s)
        target[s] = std::min<std::int64_t>(insts[s]->end, insts[s]->step + n_steps);
    // Restrict every instance to this call's window.
    std::vector<std::int64_t> saved_end(insts.size());
    for (std::size_t s = 0; s < insts.size(); ++s) {
        saved_end[s] = insts[s]->end;
        insts[s]->end = target[s];
    }
    // Equal chunks: the l steps left run as ceil(l / chunk_steps) chunks of
    // ceil(l / c) or ceil(l / c) - 1 steps.  Their graphs (at most two
    // lengths) are captured before the timed region; on a failure every
    // instance's window is restored before returning.
    auto left = [&]() {
        std::int64_t m = 0;
        for (auto& p : insts) m = std::max<std::int64_t>(m, p->end - p->step);
        return m;
    };
    auto next_chunk = [&](std::int64_t l) {
        const std::int64_t c = (l + cfg.chunk_steps - 1) / cfg.chunk_steps;
        return (l + c - 1) / c;
    };
    int st = ASG_OK;
    if (graph_mode() && !work.empty()) {
        for (std::int64_t l = left(), prev = 0; l > 0 && st == ASG_OK; l -= prev) {
            const std::int64_t a = next_chunk(l);
            if (a != prev) st = capture_graph(static_cast<int>(a));
            prev = a;
        }
    }
    if (st == ASG_OK) {
        const cudaError_t e = cudaEventRecord(ev_start, stream);
        if (e != cudaSuccess) st = cuda_fail(e, "event record", __FILE__, __LINE__);
    }
    for (; st == ASG_OK;) {
        const std::int64_t l = left();
        if (l <= 0) break;
        st = run_chunk(next_chunk(l));
        if (st == ASG_OK && left() == l) break;  // nothing to launch (no work items)
    }
    if (st == ASG_OK) st = finish_pending();
    for (std::size_t s = 0; s < insts.size(); ++s) insts[s]->end = saved_end[s];
    ASG_TRY(st);
    ASG_CUDA(cudaEventRecord(ev_end, stream));
    ASG_CUDA(cudaEventSynchronize(ev_end));
    float ms = 0.0f;
    ASG_CUDA(cudaEventElapsedTime(&ms, ev_start, ev_end));
    last_ms = ms;
    total_ms += ms;
    total_kernels += last_kernels;
    return ASG_OK;
}

int Engine::pull_state(int id, asg_state* out) {
    Instance* I = find(id);
    if (I == nullptr) return fail(ASG_ERR_NOT_FOUND, "no instance %d", id);
    ASG_TRY(finish_pending());
    const InstDev& D = I->dev;
    const std::size_t n8 = static_cast<std::size_t>(D.N) * 8, a8 = static_cast<std::size_t>(D.NA) * 8;
    struct {
        void* dst;
        const void* src;
        std::size_t bytes;
    } cp[] = {{out->V, D.V, n8},       {out->w, D.w, n8},         {out->g_ex, D.gex, n8},
              {out->dg_ex, D.dgex, n8}, {out->g_in, D.gin, n8},    {out->dg_in, D.dgin, n8},
              {out->I_sic, D.Isic, n8}, {out->refractory, D.refr, static_cast<std::size_t>(D.N) * 4},
              {out->Ca, D.Ca, a8},      {out->IP3, D.IP3, a8},     {out->h, D.h, a8}};
    for (auto& c : cp)
        if (c.dst && c.bytes)
            ASG_CUDA(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, stream));
    ASG_CUDA(cudaStreamSynchronize(stream));
    return ASG_OK;
}

int Engine::pull_stp(int id, double* x, double* u, double* t) {
    Instance* I = find(id);
    if (I == nullptr) return fail(ASG_ERR_NOT_FOUND, "no instance %d", id);
    ASG_TRY(finish_pending());
    const std::size_t n8 = static_cast<std::size_t>(I->dev.N) * 8;
    if (n8 == 0) return ASG_OK;
    if (x) ASG_CUDA(cudaMemcpyAsync(x, I->dev.stp_x, n8, cudaMemcpyDeviceToHost, stream));
    if (u) ASG_CUDA(cudaMemcpyAsync(u, I->dev.stp_u, n8, cudaMemcpyDeviceToHost, stream));
    if (t) ASG_CUDA(cudaMemcpyAsync(t, I->dev.stp_t, n8, cudaMemcpyDeviceToHost, stream));
    ASG_CUDA(cudaStreamSynchronize(stream));
    return ASG_OK;
}

}  // namespace asg
