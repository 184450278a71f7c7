// Device form of the counter-based fixed-in-degree generator (the host form
// and the rule itself are in asg_model.cpp).  Every edge is a pure function
// of (seed, target, k), so the device and the host produce the same tables:
//   1. one thread per (target, k) draws the source and the recruited
//      astrocyte (or none);
//   2. a stable radix sort by source (by astrocyte for the SIC set) of the
//      edge ids puts every row in (target, k) order, the order the host
//      emits; row starts come from the sorted keys.
// A one-time build step: the per-step path never runs it.

#include <cub/cub.cuh>

#include <vector>

#include "asg_common.hpp"
#include "asg_device.cuh"
#include "asg_model.hpp"

namespace asg {

namespace {

constexpr std::uint64_t kGenSalt = 0x6A09E667F3BCC909ULL;
constexpr std::uint32_t kNone = 0xFFFFFFFFu;

__global__ void draw_edges(std::uint32_t N, std::uint32_t NE, std::uint32_t NA,
                           std::uint32_t k_in, std::uint64_t gseed, double p_third, int psz,
                           int pool_random, std::uint32_t* src, std::uint32_t* ast) {
    const std::uint64_t e = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<std::uint64_t>(N) * k_in) return;
    const std::uint32_t t = static_cast<std::uint32_t>(e / k_in);
    const std::uint32_t k = static_cast<std::uint32_t>(e % k_in);
    const double u = uniform_at(gseed, t, 3ull * k);
    std::uint32_t s = static_cast<std::uint32_t>(u * static_cast<double>(N - 1));
    if (s >= N - 1) s = N - 2;
    if (s >= t) ++s;
    src[e] = s;
    std::uint32_t a = kNone;
    if (s < NE && NA > 0 && uniform_at(gseed, t, 3ull * k + 1) < p_third) {
        const double v = uniform_at(gseed, t, 3ull * k + 2);
        std::uint32_t pick = static_cast<std::uint32_t>(v * psz);
        if (pick > static_cast<std::uint32_t>(psz - 1)) pick = psz - 1;
        if (!pool_random) {
            const std::uint32_t start =
                static_cast<std::uint32_t>((static_cast<std::uint64_t>(t) * NA) / N);
            a = (start + pick) % NA;
        } else {
            a = static_cast<std::uint32_t>(uniform_at(gseed, static_cast<std::uint64_t>(N) + t, pick) * NA);
            if (a >= NA) a = NA - 1;
        }
    }
    ast[e] = a;
}

// Keys for one set: exc (src < NE), inh (src >= NE, key src-NE), n2a
// (recruited, key src), a2n (recruited, key astro).  Edges outside the set
// get key `none` and sort to the end.
__global__ void make_keys(std::uint64_t m, int which, std::uint32_t NE, const std::uint32_t* src,
                          const std::uint32_t* ast, std::uint32_t* key, std::uint32_t* val,
                          std::uint32_t none) {
    const std::uint64_t e = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const std::uint32_t s = src[e], a = ast[e];
    std::uint32_t k = none;
    if (which == 0 && s < NE) k = s;
    if (which == 1 && s >= NE) k = s - NE;
    if (which == 2 && s < NE && a != kNone) k = s;
    if (which == 3 && a != kNone) k = a;
    key[e] = k;
    val[e] = static_cast<std::uint32_t>(e);
}

int sort_set(std::uint64_t m, int which, std::uint32_t NE, std::uint32_t n_rows, std::uint32_t k_in,
             const std::uint32_t* d_src, const std::uint32_t* d_ast, HostCsr& out,
             cudaStream_t st) {
    DevBuf key, val, key2, val2, tmp;
    ASG_TRY(key.alloc(m * 4, false));
    ASG_TRY(val.alloc(m * 4, false));
    ASG_TRY(key2.alloc(m * 4, false));
    ASG_TRY(val2.alloc(m * 4, false));
    const std::uint32_t none = n_rows;
    const int B = 256;
    make_keys<<<static_cast<unsigned>((m + B - 1) / B), B, 0, st>>>(
        m, which, NE, d_src, d_ast, key.as<std::uint32_t>(), val.as<std::uint32_t>(), none);
    ASG_CUDA(cudaGetLastError());
    int bits = 1;
    while ((1ull << bits) <= none) ++bits;
    std::size_t tb = 0;
    ASG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.as<std::uint32_t>(),
                                             key2.as<std::uint32_t>(), val.as<std::uint32_t>(),
                                             val2.as<std::uint32_t>(), static_cast<int>(m), 0,
                                             bits, st));
    ASG_TRY(tmp.alloc(std::max<std::size_t>(tb, 1), false));
    ASG_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, key.as<std::uint32_t>(),
                                             key2.as<std::uint32_t>(), val.as<std::uint32_t>(),
                                             val2.as<std::uint32_t>(), static_cast<int>(m), 0,
                                             bits, st));
    std::vector<std::uint32_t> k(m), v(m);
    ASG_CUDA(cudaMemcpyAsync(k.data(), key2.get(), m * 4, cudaMemcpyDeviceToHost, st));
    ASG_CUDA(cudaMemcpyAsync(v.data(), val2.get(), m * 4, cudaMemcpyDeviceToHost, st));
    ASG_CUDA(cudaStreamSynchronize(st));
    out.row_start.assign(n_rows + 1, 0);
    std::size_t cnt = 0;
    while (cnt < m && k[cnt] != none) {
        out.row_start[k[cnt] + 1]++;
        ++cnt;
    }
    for (std::uint32_t r = 0; r < n_rows; ++r) out.row_start[r + 1] += out.row_start[r];
    out.target.resize(cnt);
    std::vector<std::uint32_t> ast_h;
    if (which == 2) {
        ast_h.resize(m);
        ASG_CUDA(cudaMemcpy(ast_h.data(), d_ast, m * 4, cudaMemcpyDeviceToHost));
    }
    for (std::size_t q = 0; q < cnt; ++q) {
        const std::uint32_t e = v[q];
        out.target[q] = which == 2 ? ast_h[e] : e / k_in;  // n2a rows hold astrocytes
    }
    return ASG_OK;
}

}  // namespace

int build_fixed_indegree_device(Model& m, std::uint32_t k_in, int device) {
    const ModelConfig& c = m.cfg;
    ASG_CUDA(cudaSetDevice(device));
    // Per-cell parameters come from the same sequential stream as the
    // reference builder, on the host.
    build_fixed_indegree_host_cells(m);
    const std::uint32_t NE = c.N_E, NI = c.N_I, N = NE + NI, NA = c.N_A;
    const std::uint64_t M = static_cast<std::uint64_t>(N) * k_in;
    if (M >= (1ull << 32)) return fail(ASG_ERR_UNSUPPORTED, "more than 2^32 edges");
    cudaStream_t st;
    ASG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    DevBuf src, ast;
    int rc = src.alloc(M * 4, false);
    if (rc == ASG_OK) rc = ast.alloc(M * 4, false);
    if (rc == ASG_OK && M > 0) {
        const int B = 256;
        const int psz = NA == 0 ? 0 : std::min<int>(c.pool_size, static_cast<int>(NA));
        draw_edges<<<static_cast<unsigned>((M + B - 1) / B), B, 0, st>>>(
            N, NE, NA, k_in, c.seed ^ kGenSalt, c.p_third, psz, c.pool_random ? 1 : 0,
            src.as<std::uint32_t>(), ast.as<std::uint32_t>());
        const cudaError_t ce = cudaGetLastError();
        if (ce != cudaSuccess) rc = cuda_fail(ce, "draw_edges", __FILE__, __LINE__);
    }
    if (rc == ASG_OK) rc = sort_set(M, 0, NE, NE, k_in, src.as<std::uint32_t>(), ast.as<std::uint32_t>(), m.exc, st);
    if (rc == ASG_OK) rc = sort_set(M, 1, NE, NI, k_in, src.as<std::uint32_t>(), ast.as<std::uint32_t>(), m.inh, st);
    if (rc == ASG_OK) rc = sort_set(M, 2, NE, NE, k_in, src.as<std::uint32_t>(), ast.as<std::uint32_t>(), m.n2a, st);
    if (rc == ASG_OK) rc = sort_set(M, 3, NE, NA, k_in, src.as<std::uint32_t>(), ast.as<std::uint32_t>(), m.a2n, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (rc == ASG_OK) m.built = true;
    return rc;
}

}  // namespace asg
