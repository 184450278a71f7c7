// The fused per-timestep kernel of the network engine (layout and design in
// asg_engine.cuh).  Compiled with -fmad=false: every floating-point
// expression is evaluated as separate IEEE operations in the reference's
// order (neuron.cpp:101-250, astrocyte.cpp:233-329, network.cpp:230-355).
//
// Latency, not bandwidth, bounds a step of a network of this size: each
// role is a short chain of dependent memory round trips and FP64 operations,
// and a step ends with its slowest thread.  So every role (1) reads what the
// previous step cannot have changed (per-cell constants, CSR rows, SIC lists)
// BEFORE waiting on the previous step's grid, (2) then issues every load of
// the step's inputs at once, (3) reads its arrivals with one more batch of
// loads in the common case of a few arrivals per target, and (4) keeps rare
// paths (noise, the large-lambda Poisson branch, many-arrival merges, the
// in-block push, the fused SIC) out of line so the instruction stream of the
// common path stays small.  The per-step slot and modulo arithmetic is done
// once per block, also before the wait.

#include <cuda_runtime.h>

#include "asg_engine.cuh"

namespace asg {

namespace {

constexpr int kMaxBlock = 512;
constexpr std::uint32_t kNoBit = 0xFFFFFFFFu;
constexpr int kSicBatch = 8;  // SIC list entries loaded per batch

__device__ __forceinline__ void grid_dep_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ Work load_work(const Work* p) {
    static_assert(sizeof(Work) == 16, "Work is one 16-byte load");
    const uint4 v = __ldcg(reinterpret_cast<const uint4*>(p));
    Work w;
    w.inst = v.x;
    w.role = static_cast<std::uint16_t>(v.y & 0xFFFFu);
    w.helper = static_cast<std::uint16_t>(v.y >> 16);
    w.first = v.z;
    w.count = v.w;
    return w;
}

// Everything about the current step that is the same for a whole block.
struct StepInfo {
    std::int64_t step;
    std::uint32_t slot;        // ring slot read this step: step % slots
    std::uint32_t fslot;       // factor slot of the SIC arriving now (fused SIC)
    // SIC role: part p works on arrival step+P-p; bit p of sic_due says
    // that arrival takes SIC, sic_slot[p] is its factor slot
    std::uint32_t sic_due;
    std::uint32_t sic_slot[kMaxSicParts];
    std::uint32_t push_e, push_i;          // deferred push of step-1's spikes
    std::uint32_t now_e, now_i;            // in-block push of this step's spikes
    std::uint32_t ls, ls_prev, ls_next;    // spike-list slots of step, step-1, step+1
    std::uint32_t rec_row;
    std::uint64_t noise_e, noise_i, noise_a;  // noise draw indices
    std::int32_t sic_now, fac_now, rec_now;
    // noise terms drawn this step (else read from the cache): exc, inh, astro
    std::int32_t fresh_e, fresh_i, fresh_a;
    // fac_any indices: this step's emission, the next step's (cleared now),
    // and the emission the fused SIC of this step reads (-1: none yet)
    std::int32_t fany_now, fany_next, fany_read;
};

// Computed by warp 0 of the block: each lane forms one quotient and
// remainder (of a step offset by a period), so the whole set costs the
// latency of one 64-bit division instead of some twenty in a row.
__device__ void make_step_info(const InstDev& I, std::int64_t step, StepInfo& S) {
    __shared__ long long s_q[32], s_r[32];
    const int lane = static_cast<int>(threadIdx.x);
    const int P = I.sic_parts;
    std::int64_t n = step, d = I.slots;  // lane 0: ring slot
    if (lane == 1) { n = step - I.d_a2n; d = I.sic_interval; }
    if (lane == 2) { n = step - I.d_a2n; }
    if (lane == 3) { n = step - 1 + I.d_e; }
    if (lane == 4) { n = step - 1 + I.d_i; }
    if (lane == 5) { n = step + I.d_e; }
    if (lane == 6) { n = step + I.d_i; }
    if (lane == 7) { d = 3; }
    if (lane == 8) { d = I.sic_interval; }
    if (lane == 9) { n = step - I.rec_from; d = I.rec_every; }
    if (lane == 10) { d = I.pe.steps_per_noise; }
    if (lane == 11) { d = I.pi.steps_per_noise; }
    if (lane == 12) { d = I.a_steps_per_noise; }
    if (lane >= 13 && lane < 13 + P) { n = step + P - (lane - 13) - I.d_a2n; d = I.sic_interval; }
    if (lane >= 13 + P && lane < 13 + 2 * P) { n = step + P - (lane - 13 - P) - I.d_a2n; }
    if (lane == 29) { d = I.slots + 1; }
    if (lane == 30) { n = step + 1; d = I.slots + 1; }
    if (lane == 31) { n = step - I.d_a2n; d = I.slots + 1; }
    std::int64_t q = -1, r = -1;  // -1: negative numerator (not yet due)
    if (n >= 0) {
        const auto un = static_cast<unsigned long long>(n), ud = static_cast<unsigned long long>(d);
        q = static_cast<std::int64_t>(un / ud);
        r = static_cast<std::int64_t>(un - static_cast<unsigned long long>(q) * ud);
    }
    s_q[lane] = q;
    s_r[lane] = r;
    __syncwarp();
    if (lane == 0) {
        S.step = step;
        S.slot = static_cast<std::uint32_t>(s_r[0]);
        S.sic_now = s_r[1] == 0;
        S.fslot = s_r[2] >= 0 ? static_cast<std::uint32_t>(s_r[2]) : 0u;
        S.sic_due = 0;
        for (int p = 0; p < P; ++p) {
            const bool due = s_r[13 + p] == 0;
            S.sic_due |= due ? (1u << p) : 0u;
            S.sic_slot[p] = due ? static_cast<std::uint32_t>(s_r[13 + P + p]) : 0u;
        }
        S.push_e = static_cast<std::uint32_t>(s_r[3]);
        S.push_i = static_cast<std::uint32_t>(s_r[4]);
        S.now_e = static_cast<std::uint32_t>(s_r[5]);
        S.now_i = static_cast<std::uint32_t>(s_r[6]);
        S.ls = static_cast<std::uint32_t>(s_r[7]);
        S.ls_prev = (S.ls + 2) % 3;
        S.ls_next = (S.ls + 1) % 3;
        S.fac_now = s_r[8] == 0;
        S.rec_now = s_r[9] == 0;
        S.rec_row = S.rec_now ? static_cast<std::uint32_t>(
                                    static_cast<unsigned long long>(s_q[9]) % I.rec_rows)
                              : 0u;
        S.noise_e = static_cast<std::uint64_t>(s_q[10]);
        S.noise_i = static_cast<std::uint64_t>(s_q[11]);
        S.noise_a = static_cast<std::uint64_t>(s_q[12]);
        const bool restart = step == I.noise_from;
        S.fresh_e = s_r[10] == 0 || restart;
        S.fresh_i = s_r[11] == 0 || restart;
        S.fresh_a = s_r[12] == 0 || restart;
        S.fany_now = static_cast<std::int32_t>(s_r[29]);
        S.fany_next = static_cast<std::int32_t>(s_r[30]);
        S.fany_read = static_cast<std::int32_t>(s_r[31]);
    }
}

// Routes one arrival the way NeuronPopulation::add_synaptic_input does
// (neuron.cpp:77-83): positive weights to the excitatory input, negative
// ones (as magnitudes) to the inhibitory input.
__device__ __forceinline__ void add_syn(double v, double& exc_in, double& inh_in) {
    if (v > 0.0) {
        exc_in += v;
    } else if (v < 0.0) {
        inh_in -= v;
    }
}

// ------------------------------------------------------------- arrivals

// One batch of loads: the (bit, value) pairs of the first kListCap arrivals
// of (slot, target) `ts`.
struct ShortList {
    uint4 bit;
    double2 v01, v23;
};

__device__ __forceinline__ ShortList load_list(const InRing& R, std::size_t ts) {
    ShortList l;
    l.bit = __ldcg(reinterpret_cast<const uint4*>(R.lbit) + ts);
    l.v01 = __ldcg(reinterpret_cast<const double2*>(R.lval) + 2 * ts);
    l.v23 = __ldcg(reinterpret_cast<const double2*>(R.lval) + 2 * ts + 1);
    return l;
}

__device__ __forceinline__ void order2(std::uint32_t& ba, double& va, std::uint32_t& bb,
                                       double& vb) {
    const bool swap = bb < ba;
    const std::uint32_t b = swap ? bb : ba;
    const double v = swap ? vb : va;
    bb = swap ? ba : bb;
    vb = swap ? va : vb;
    ba = b;
    va = v;
}

__device__ __forceinline__ double accumulate(double acc, double v, bool sub) {
    return sub ? acc - v : acc + v;
}

// merge_overflow for a target of at most 32 bitmap words (in-degree <= 1024):
// every word in one batch of loads (its pushes keep no summary), then the set bits in
// ascending order in passes of 8 value loads.  The words sit in a local
// array (the walk indexes it at run time); the pass's value loads are issued
// at the same point of the code by all lanes, as in merge_overflow.  (Passes
// of 12 or 16 loads measured slower: the larger register footprint of this
// out-of-line call costs the step kernel spills on its common path.)
__device__ __forceinline__ double merge_dense(std::uint32_t* bits, const double* vals,
                                              std::uint32_t w0,
                                              std::uint32_t nw, bool sub, std::uint32_t l0,
                                              std::uint32_t l1, std::uint32_t l2,
                                              std::uint32_t l3, double v0, double v1, double v2,
                                              double v3) {
    std::uint32_t wv[32];
#pragma unroll
    for (int k = 0; k < 32; ++k)
        wv[k] = static_cast<std::uint32_t>(k) < nw ? __ldcg(bits + w0 + k) : 0u;
    std::uint32_t live = 0;  // words with bits not yet taken
#pragma unroll
    for (int k = 0; k < 32; ++k) {
        if (wv[k] != 0) {
            live |= 1u << k;
            bits[w0 + k] = 0;
        }
    }
    double acc = 0.0;
    std::uint32_t cw = 0, ck = 0;  // bits left in the current word, its index
    for (;;) {
        std::uint32_t idx[8];
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            if (cw == 0 && live != 0) {
                ck = static_cast<std::uint32_t>(__ffs(live) - 1);
                live &= live - 1;
                cw = wv[ck];
            }
            if (cw != 0) {
                idx[s] = (w0 + ck) * 32 + static_cast<std::uint32_t>(__ffs(cw) - 1);
                cw &= cw - 1;
            } else {
                idx[s] = kNoBit;
            }
        }
        if (idx[0] == kNoBit) break;
        double v[8];
#pragma unroll
        for (int s = 0; s < 8; ++s) v[s] = idx[s] != kNoBit ? __ldcg(vals + idx[s]) : 0.0;
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            if (idx[s] == kNoBit) break;
            while (l0 < idx[s]) {  // list entries that precede this bit
                acc = accumulate(acc, v0, sub);
                l0 = l1;
                v0 = v1;
                l1 = l2;
                v1 = v2;
                l2 = l3;
                v2 = v3;
                l3 = kNoBit;
            }
            acc = accumulate(acc, v[s], sub);
        }
    }
    while (l0 != kNoBit) {
        acc = accumulate(acc, v0, sub);
        l0 = l1;
        v0 = v1;
        l1 = l2;
        v1 = v2;
        l2 = l3;
        v2 = v3;
        l3 = kNoBit;
    }
    return acc;
}

// More than kListCap arrivals: the first kListCap (sorted, l0 < l1 < l2 <
// l3) are merged in bit order with the later ones, which sit in the
// target's bitmap words (visited through the summary).  Loads go out in
// batches -- up to 8 words, then up to 8 values -- and every batch is issued
// at the same point of the code by all lanes of a warp: lanes with more
// arrivals run more passes, but no lane's loads wait behind another lane's
// (a per-lane "flush when 8 are collected" would serialize the warp's round
// trips lane by lane).  All arrays are indexed by unrolled constants.
// Clears the summary and the words.
__device__ __noinline__ double merge_overflow(const InRing& R, std::uint32_t slot,
                                              std::uint32_t t, bool sub, std::uint32_t l0,
                                              std::uint32_t l1, std::uint32_t l2,
                                              std::uint32_t l3, double v0, double v1, double v2,
                                              double v3) {
    unsigned long long* sp = R.sum + static_cast<std::size_t>(slot) * R.n_targets + t;
    std::uint32_t* bits = R.bits + static_cast<std::size_t>(slot) * R.words;
    const double* vals = R.vals + static_cast<std::size_t>(slot) * R.words * 32;
    const std::uint32_t w0 = R.wbase[t], nw = R.wbase[t + 1] - w0;
    if (nw <= 32)
        return merge_dense(bits, vals, w0, nw, sub, l0, l1, l2, l3, v0, v1, v2, v3);
    unsigned long long groups = __ldcg(sp);
    *sp = 0;
    const std::uint32_t G = (nw + 63) >> 6;  // words per summary bit
    double acc = 0.0;
    std::uint32_t q[8], wv[8];
    std::uint32_t cur = 0, cur_end = 0;  // words [cur, cur_end) of the open group
    bool open = false;
    for (;;) {
        int nq = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (!open && groups != 0) {
                const std::uint32_t g = __ffsll(groups) - 1;
                groups &= groups - 1;
                cur = w0 + g * G;
                cur_end = min(cur + G, w0 + nw);
                open = cur < cur_end;
            }
            q[k] = cur;
            if (open) {
                nq = k + 1;
                if (++cur >= cur_end) open = false;
            }
        }
        if (nq == 0) break;
#pragma unroll
        for (int k = 0; k < 8; ++k) wv[k] = k < nq ? __ldcg(bits + q[k]) : 0u;
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (wv[k] != 0) bits[q[k]] = 0;
        // Passes of up to 8 set bits, in ascending order over the words.
        for (;;) {
            std::uint32_t any = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) any |= wv[k];
            if (any == 0) break;
            std::uint32_t idx[8];
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                std::uint32_t w = 0, base = 0;
                bool found = false;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const bool take = !found && wv[k] != 0;
                    w = take ? wv[k] : w;
                    base = take ? q[k] * 32 : base;
                    if (take) wv[k] &= wv[k] - 1;
                    found = found || take;
                }
                idx[s] = found ? base + static_cast<std::uint32_t>(__ffs(w) - 1) : kNoBit;
            }
            double v[8];
#pragma unroll
            for (int s = 0; s < 8; ++s) v[s] = idx[s] != kNoBit ? __ldcg(vals + idx[s]) : 0.0;
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                if (idx[s] == kNoBit) break;
                while (l0 < idx[s]) {  // list entries that precede this bit
                    acc = accumulate(acc, v0, sub);
                    l0 = l1;
                    v0 = v1;
                    l1 = l2;
                    v1 = v2;
                    l2 = l3;
                    v2 = v3;
                    l3 = kNoBit;
                }
                acc = accumulate(acc, v[s], sub);
            }
        }
    }
    while (l0 != kNoBit) {
        acc = accumulate(acc, v0, sub);
        l0 = l1;
        v0 = v1;
        l1 = l2;
        v1 = v2;
        l2 = l3;
        v2 = v3;
        l3 = kNoBit;
    }
    return acc;
}

// Ordered sum of the `n` (>= 1) arrivals of target t in `slot`, given its
// short list.  kSubtract selects ring_inh's `-=` accumulation
// (network.cpp:271-275).
template <bool kSubtract>
__device__ __forceinline__ double sum_arrivals(const InRing& R, std::uint32_t slot,
                                               std::uint32_t t, std::uint32_t n,
                                               const ShortList& l) {
    std::uint32_t b0 = l.bit.x, b1 = n > 1 ? l.bit.y : kNoBit, b2 = n > 2 ? l.bit.z : kNoBit,
                  b3 = n > 3 ? l.bit.w : kNoBit;
    double v0 = l.v01.x, v1 = l.v01.y, v2 = l.v23.x, v3 = l.v23.y;
    order2(b0, v0, b1, v1);
    order2(b2, v2, b3, v3);
    order2(b0, v0, b2, v2);
    order2(b1, v1, b3, v3);
    order2(b1, v1, b2, v2);
    if (n > static_cast<std::uint32_t>(kListCap))
        return merge_overflow(R, slot, t, kSubtract, b0, b1, b2, b3, v0, v1, v2, v3);
    double acc = accumulate(0.0, v0, kSubtract);
    if (n > 1) acc = accumulate(acc, v1, kSubtract);
    if (n > 2) acc = accumulate(acc, v2, kSubtract);
    if (n > 3) acc = accumulate(acc, v3, kSubtract);
    return acc;
}

// One arrival on the edge with packed word `pe` (bit | target << 32 | dense
// << 57 | summary bit << 58): a ticket from the target's counter decides
// between the short list and the bitmap; the summary is kept only for
// targets of more than 32 words.
__device__ __forceinline__ void push_edge(const InRing& R, std::uint32_t slot,
                                          unsigned long long pe, double value) {
    const std::uint32_t b = static_cast<std::uint32_t>(pe);
    const std::uint32_t t = static_cast<std::uint32_t>(pe >> 32) & 0x1FFFFFFu;
    const std::size_t ts = static_cast<std::size_t>(slot) * R.n_targets + t;
    const std::uint32_t k = atomicAdd(R.cnt + ts, 1u);
    if (k < static_cast<std::uint32_t>(kListCap)) {
        R.lbit[ts * kListCap + k] = b;
        R.lval[ts * kListCap + k] = value;
    } else {
        const std::uint32_t g = static_cast<std::uint32_t>(pe >> 58);
        R.vals[static_cast<std::size_t>(slot) * R.words * 32 + b] = value;
        atomicOr(R.bits + static_cast<std::size_t>(slot) * R.words + (b >> 5), 1u << (b & 31));
        if (((pe >> 57) & 1ull) == 0) atomicOr(R.sum + ts, 1ull << g);
    }
}

// Writes `value` at every out-edge of `row` (in-block push, used when a
// spike delay is a single step).
__device__ __noinline__ void push_row(const std::uint32_t* rs, const InRing& R, std::uint32_t row,
                                      std::uint32_t slot, double value) {
    const std::uint32_t e1 = rs[row + 1];
#pragma unroll 4
    for (std::uint32_t e = rs[row] + threadIdx.x; e < e1; e += blockDim.x)
        push_edge(R, slot, __ldg(R.edge + e), value);
}

// ---------------------------------------------------------------- SIC

// Sequential SIC sum from the factors of emission slot fslot, continuing
// `acc` (network.cpp:281-299 order: ascending astrocyte, one add of
// w_a2n * factor per edge).  `e` holds the first kSicBatch list entries
// (loaded by the caller); the factors of a batch are fetched with
// independent loads before its additions.
__device__ __forceinline__ double sic_sum(const InstDev& I, std::uint32_t o0, std::uint32_t len,
                                          std::uint32_t (&e)[kSicBatch], std::uint32_t fslot,
                                          double acc, unsigned long long& edges) {
    const double* fac = I.fac + static_cast<std::size_t>(fslot) * I.NA;
    for (std::uint32_t b0 = 0;; b0 += kSicBatch) {
        double f[kSicBatch];
#pragma unroll
        for (int k = 0; k < kSicBatch; ++k) f[k] = (e[k] & 0xFFu) ? __ldcg(fac + (e[k] >> 8)) : 0.0;
        bool done = false;
#pragma unroll
        for (int k = 0; k < kSicBatch; ++k) {
            const std::uint32_t m = e[k] & 0xFFu;
            if (m == 0) {
                done = true;  // padding ends the list
                break;
            }
            if (f[k] == 0.0) continue;
            const double c = I.w_a2n * f[k];
            for (std::uint32_t r = 0; r < m; ++r) acc += c;
            edges += m;
        }
        if (done || b0 + kSicBatch >= len) break;
#pragma unroll
        for (int k = 0; k < kSicBatch; ++k) {
            const std::uint32_t j = b0 + kSicBatch + k;
            e[k] = j < len ? __ldg(I.sic_ent + o0 + j * 32) : 0u;
        }
    }
    return acc;
}

// First batch of a target's SIC list entries (static data).  o0 is the
// target's first entry; entries of one target are 32 apart (sliced ELL).
__device__ __forceinline__ void sic_prefetch(const InstDev& I, std::uint32_t t, std::uint32_t& o0,
                                             std::uint32_t& len,
                                             std::uint32_t (&e)[kSicBatch]) {
    const std::uint32_t slice = t >> 5;
    const std::uint32_t s0 = I.sic_soff[slice], s1 = I.sic_soff[slice + 1];
    o0 = s0 + (t & 31);
    len = (s1 - s0) >> 5;
#pragma unroll
    for (int k = 0; k < kSicBatch; ++k)
        e[k] = static_cast<std::uint32_t>(k) < len ? __ldg(I.sic_ent + o0 + k * 32) : 0u;
}

// SIC of a neuron summed by its own thread (fused mode, SIC delay of one step).
__device__ __noinline__ double fused_sic(const InstDev& I, std::uint32_t c, std::uint32_t fslot) {
    std::uint32_t o0, len, e[kSicBatch];
    sic_prefetch(I, c, o0, len, e);
    unsigned long long edges = 0;
    const double v = sic_sum(I, o0, len, e, fslot, 0.0, edges);
    if (edges) atomicAdd(I.counters + 1, edges);
    return v;
}

// ---------------------------------------------------------------- noise

// Box-Muller draws, out of line (log, sqrt and cos are sizeable code and
// most configurations run without noise).
__device__ __noinline__ double normal_first_at(std::uint64_t seed, std::uint64_t stream) {
    Draws r(seed, stream);
    return r.normal_first();
}

__device__ __noinline__ double normal_clamped_at(std::uint64_t seed, std::uint64_t stream) {
    return normal_clamped(seed, stream);
}

// apply_arrivals (network.cpp:301-338) for one target: both short lists in
// one batch, the counters cleared for the slot's next use, the excitatory
// sum then the inhibitory one routed as add_synaptic_input does.
__device__ __forceinline__ void apply_arrivals(const InstDev& I, std::uint32_t slot,
                                               std::uint32_t c, std::size_t ts_ex,
                                               std::size_t ts_in, std::uint32_t n_ex,
                                               std::uint32_t n_in, double v0_ex, double& exc_in,
                                               double& inh_in) {
    ShortList lex{}, lin{};
    if (n_ex > 1) lex = load_list(I.ring_ex, ts_ex);
    if (n_in) lin = load_list(I.ring_in, ts_in);
    if (n_ex) {
        I.ring_ex.cnt[ts_ex] = 0;
        // one arrival: 0.0 + v, the sum sum_arrivals forms for n = 1
        const double ex =
            n_ex == 1 ? 0.0 + v0_ex : sum_arrivals<false>(I.ring_ex, slot, c, n_ex, lex);
        if (ex != 0.0) add_syn(ex, exc_in, inh_in);
    }
    if (n_in) {
        I.ring_in.cnt[ts_in] = 0;
        const double in = sum_arrivals<true>(I.ring_in, slot, c, n_in, lin);
        if (in != 0.0) add_syn(-in, exc_in, inh_in);
    }
}

struct SynIn {
    double exc, inh;
};

__device__ __noinline__ SynIn arrivals_out_of_line(const InstDev& I, std::uint32_t slot,
                                                   std::uint32_t c, std::size_t ts_ex,
                                                   std::size_t ts_in, std::uint32_t n_ex,
                                                   std::uint32_t n_in, double v0_ex) {
    SynIn r{0.0, 0.0};
    apply_arrivals(I, slot, c, ts_ex, ts_in, n_ex, n_in, v0_ex, r.exc, r.inh);
    return r;
}

// --------------------------------------------------------------- roles

// kWide, the form for large steps: a warp's spikes take one atomic per warp
// (ballot and prefix sums), which pays off when a step has many spiking
// warps, and targets with several arrivals are summed out of line.
// Otherwise each spiking thread appends itself, the shortest chain for the
// few spikes of a small network's step, and the arrival lists stay inline.
// Either order of the spike records gives the same rings (the arrivals are
// summed in bit order).
template <bool kPdl, bool kWide>
__device__ void neuron_role(const InstDev& I, const StepInfo& S, const Work& wk) {
    __shared__ std::uint32_t s_spk[kMaxBlock];
    __shared__ double s_val[2 * kMaxBlock];
    __shared__ int s_nspk;
    if (threadIdx.x == 0) s_nspk = 0;

    const std::uint32_t c = wk.first + threadIdx.x;
    const bool active = threadIdx.x < wk.count;
    const bool exc = c < I.NE;
    // Written before the chunk started: read before waiting on the
    // previous step.
    double Vr = 0.0, bc = 0.0;
    std::uint32_t r0 = 0, len0 = 0, len1 = 0;  // out-edge rows (the wide form: on a spike)
    if (active) {
        if (!kWide) {  // the wide form reads these where a reset needs them
            Vr = I.V_reset[c];
            bc = I.b[c];
            if (exc) {
                r0 = I.exc_rs[c];
                len0 = I.exc_rs[c + 1] - r0;
                len1 = I.n2a_rs[c + 1] - I.n2a_rs[c];
            } else {
                r0 = I.inh_rs[c - I.NE];
                len0 = I.inh_rs[c - I.NE + 1] - r0;
            }
        }
    }
    if (kPdl) grid_dep_wait();
    __syncthreads();
    const std::int64_t step = S.step;
    if (step >= I.end_step) return;

    if (active) {
        const NeuronK& P = exc ? I.pe : I.pi;
        const std::uint32_t slot = S.slot;

        // Every input of the step in one batch of independent loads.
        const std::size_t ts_ex = static_cast<std::size_t>(slot) * I.ring_ex.n_targets + c;
        const std::size_t ts_in = static_cast<std::size_t>(slot) * I.ring_in.n_targets + c;
        const std::uint32_t n_ex = __ldcg(I.ring_ex.cnt + ts_ex);
        const std::uint32_t n_in = __ldcg(I.ring_in.cnt + ts_in);
        // The first excitatory list value, loaded before the count is known:
        // with a single arrival (the common case) the sum needs no second
        // round trip.
        const double v0_ex = __ldcg(I.ring_ex.lval + ts_ex * kListCap);
        const bool sic_due = S.sic_now != 0;
        double Isic = (sic_due && !I.fused_sic)
                          ? __ldcg(I.sic_val +
                                   static_cast<std::size_t>(step & (I.sic_ring - 1)) * I.N + c)
                          : I.Isic[c];
        double V = I.V[c], w = I.w[c], gex = I.gex[c], gin = I.gin[c];
        double dgex = I.dgex[c], dgin = I.dgin[c];
        int refr = I.refr[c];
        // The source's STP state: prefetched with the state in the latency
        // form; in the wide form read by a spiking thread only (one more
        // round trip for a rare event, three fewer values live through the
        // RK4).
        double sx = 1.0, su = 1.0, st = 0.0;
        if (!kWide && I.stp_on) {
            sx = I.stp_x[c];
            su = I.stp_u[c];
            st = I.stp_t[c];
        }

        // Draws need no memory: they overlap the loads above.
        int ev = 0;
        if (P.poiss_rate > 0.0) {
            Draws r(I.seed ^ kSaltNeuronPoisson,
                    static_cast<std::uint64_t>(step) * kStreamStride + c);
            ev = r.poisson(P.lambda, P.knuth_limit);
        }
        // Noise term noise_std * z (neuron.cpp:243-248), z drawn once per
        // noise interval.
        double zterm = 0.0;
        if (P.noise_std > 0.0) {
            if (exc ? S.fresh_e : S.fresh_i) {
                const std::uint64_t idx = exc ? S.noise_e : S.noise_i;
                const double z =
                    P.independent_noise
                        ? normal_first_at(I.seed ^ kSaltNeuronNoise, idx * kNoiseStride + c)
                        : normal_first_at(I.seed ^ (exc ? kSaltSharedExc : kSaltSharedInh), idx);
                zterm = P.noise_std * z;
                I.noise_n[c] = zterm;
            } else {
                zterm = I.noise_n[c];
            }
        }

        double exc_in = 0.0, inh_in = 0.0;
        if constexpr (kWide) {
            // Most targets of a large network see no arrival or a single
            // excitatory one in a step; the rest go out of line, so the list
            // registers are not live on the common path.
            if (n_ex > 1 || n_in != 0u) {
                const SynIn a = arrivals_out_of_line(I, slot, c, ts_ex, ts_in, n_ex, n_in, v0_ex);
                exc_in = a.exc;
                inh_in = a.inh;
            } else if (n_ex) {
                I.ring_ex.cnt[ts_ex] = 0;
                const double ex = 0.0 + v0_ex;
                if (ex != 0.0) add_syn(ex, exc_in, inh_in);
            }
        } else {
            apply_arrivals(I, slot, c, ts_ex, ts_in, n_ex, n_in, v0_ex, exc_in, inh_in);
        }
        if (sic_due) {
            if (I.fused_sic)
                Isic = (S.fany_read >= 0 && __ldcg(I.fac_any + S.fany_read) != 0u)
                           ? fused_sic(I, c, S.fslot)
                           : 0.0;  // no emitting astrocyte: the sum of no terms
            I.Isic[c] = Isic;
        }

        // Poisson drive and noise (neuron.cpp:228-248)
        if (ev > 0) exc_in += P.poiss_weight * static_cast<double>(ev);
        double Iext = Isic;
        if (P.noise_std > 0.0) Iext += 0.0 + zterm;

        if (exc_in != 0.0) dgex += exc_in * P.psc_ex;
        if (inh_in != 0.0) dgin += inh_in * P.psc_in;

        const double h = I.ak.h;  // h_step is shared by both models
        const double half_h = I.ak.half_h, h6 = I.ak.h6;
        bool spiked = false;
        for (int s = 0; s < I.ak.substeps; ++s) {
            const double gex1 = P.decay_ex * (gex + h * dgex);
            const double dgex1 = P.decay_ex * dgex;
            const double gin1 = P.decay_in * (gin + h * dgin);
            const double dgin1 = P.decay_in * dgin;
            if (refr > 0) {
                V = kWide ? I.V_reset[c] : Vr;
                const AdexRates r = adex<false>(P, V, w, gex, gin, Iext);
                w += h * r.w;
            } else {
                // RK4 with the conductances at the start, midpoint and end of
                // the substep (neuron.cpp:285-298), the four stages unrolled
                // (no stage selects at run time); the stage sum
                // k1 + 2 k2 + 2 k3 + k4 accumulates left to right.
                const double gexm = 0.5 * (gex + gex1), ginm = 0.5 * (gin + gin1);
                double sV = 0.0, sw = 0.0, xV = V, xw = w;
#pragma unroll
                for (int stg = 0; stg < 4; ++stg) {
                    const double ge = stg == 0 ? gex : (stg < 3 ? gexm : gex1);
                    const double gi = stg == 0 ? gin : (stg < 3 ? ginm : gin1);
                    const AdexRates r = adex<true>(P, xV, xw, ge, gi, Iext);
                    if (stg == 0) {
                        sV = r.V;
                        sw = r.w;
                    } else if (stg < 3) {
                        sV = fma(2.0, r.V, sV);  // = sV + 2.0 * r.V: 2r is exact
                        sw = fma(2.0, r.w, sw);
                    } else {
                        sV = sV + r.V;
                        sw = sw + r.w;
                    }
                    const double stp = stg < 2 ? half_h : h;
                    xV = V + stp * r.V;
                    xw = w + stp * r.w;
                }
                V += h6 * sV;
                w += h6 * sw;
            }
            gex = gex1;
            dgex = dgex1;
            gin = gin1;
            dgin = dgin1;
            if (refr > 0) {
                --refr;
            } else if (V >= P.V_peak) {
                V = kWide ? I.V_reset[c] : Vr;
                w += kWide ? I.b[c] : bc;
                refr = P.ref_steps;
                spiked = true;
            }
        }
        I.V[c] = V;
        I.w[c] = w;
        I.gex[c] = gex;
        I.dgex[c] = dgex;
        I.gin[c] = gin;
        I.dgin[c] = dgin;
        I.refr[c] = refr;

        double v0 = 0.0, v1 = 0.0;  // the values a spike's edges deliver
        std::uint32_t r1 = 0;
        if (spiked) {
            if (kWide) {
                if (I.stp_on) {
                    sx = I.stp_x[c];
                    su = I.stp_u[c];
                    st = I.stp_t[c];
                }
                if (exc) {
                    r0 = I.exc_rs[c];
                    len0 = I.exc_rs[c + 1] - r0;
                    len1 = I.n2a_rs[c + 1] - I.n2a_rs[c];
                } else {
                    r0 = I.inh_rs[c - I.NE];
                    len0 = I.inh_rs[c - I.NE + 1] - r0;
                }
            }
            // Tsodyks-Markram update of this source (network.cpp:230-247); the
            // value its edges deliver is w*x*u per set.
            double x = 1.0, u = 1.0;
            if (I.stp_on) {
                const double t_now = static_cast<double>(step) * I.dt;
                const double d = t_now - st;
                const double xd = exp(div_by(-d, I.tau_rec, I.inv_tau_rec));
                const double ud =
                    I.tau_fac < 1e-10 ? 0.0 : exp(div_by(-d, I.tau_fac, I.inv_tau_fac));
                x = 1.0 + (sx - sx * su - 1.0) * xd;
                u = I.U + su * (1.0 - I.U) * ud;
                I.stp_x[c] = x;
                I.stp_u[c] = u;
                I.stp_t[c] = t_now;
            }
            v0 = exc ? (I.stp_on ? I.w_e * x * u : I.w_e) : (I.stp_on ? I.w_i * x * u : I.w_i);
            v1 = exc ? (I.stp_on ? I.w_n2a * x * u : I.w_n2a) : 0.0;
            // n2a row start of an excitatory source (~0: inhibitory), loaded
            // while the warp's append is formed
            if (I.deferred_push) r1 = exc ? __ldg(I.n2a_rs + c) : kNoBit;
            if (!I.deferred_push) {
                s_val[threadIdx.x * 2 + 0] = v0;
                s_val[threadIdx.x * 2 + 1] = v1;
                const int pos = atomicAdd(&s_nspk, 1);
                s_spk[pos] = threadIdx.x;
            }
        }

        if constexpr (!kWide) {
            if (spiked) {
                // One atomic reserves this spike's record and edge range.
                if (I.deferred_push) {
                    const unsigned long long old = atomicAdd(
                        I.spk_packed + S.ls * kHeaderStride,
                        (1ull << 40) | static_cast<unsigned long long>(len0 + len1));
                    const std::size_t o = static_cast<std::size_t>(S.ls) * I.N + (old >> 40);
                    *reinterpret_cast<uint4*>(I.spk_meta + 4 * o) = make_uint4(
                        r1, static_cast<std::uint32_t>(old & 0xFFFFFFFFFFull), r0, len0);
                    *reinterpret_cast<double2*>(I.spk_val + 2 * o) = make_double2(v0, v1);
                }
                if (I.rec_spikes && step >= I.rec_from) {
                    const unsigned long long li = atomicAdd(I.spike_log_n, 1ULL);
                    if (li < I.spike_log_cap) {
                        I.spike_log[li] = (static_cast<unsigned long long>(step) << 32) | c;
                    } else {
                        atomicAdd(I.counters + 3, 1ULL);
                    }
                }
                atomicAdd(I.counters + 0, static_cast<unsigned long long>(len0 + len1));
                atomicAdd(I.counters + 2, 1ULL);
            }
        }
        // The warp's spikes are compacted with a ballot and prefix sums: one
        // atomic per warp reserves the spike records and edge range of the
        // deferred push, one the spike-log entries, one each counter; every
        // spiking lane writes at its rank among the warp's spiking lanes
        // (ascending source) and at its exclusive prefix of edge counts.
        // The active lanes of a warp are a prefix of it (threadIdx.x <
        // wk.count), all of which reach this point.
        const unsigned lane = threadIdx.x & 31u;
        const unsigned wbase = threadIdx.x & ~31u;
        const unsigned left = wk.count - wbase;  // > 0 for an active lane
        const unsigned act = left >= 32u ? 0xFFFFFFFFu : ((1u << left) - 1u);
        const unsigned smask = kWide ? __ballot_sync(act, spiked) : 0u;  // syncs act
        if (kWide && smask != 0u) {
            const unsigned rank = __popc(smask & ((1u << lane) - 1u));
            const int leader = __ffs(smask) - 1;
            const unsigned nspk = __popc(smask);
            const unsigned long long edges =
                spiked ? static_cast<unsigned long long>(len0 + len1) : 0ull;
            unsigned long long incl = edges;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const unsigned long long t = __shfl_up_sync(act, incl, d);
                if (lane >= static_cast<unsigned>(d)) incl += t;
            }
            const int last = 31 - __clz(act);
            const unsigned long long total = __shfl_sync(act, incl, last);
            unsigned long long base_spk = 0, base_log = 0;
            const bool logging = I.rec_spikes && step >= I.rec_from;
            if (lane == static_cast<unsigned>(leader)) {
                if (I.deferred_push)
                    base_spk = atomicAdd(I.spk_packed + S.ls * kHeaderStride,
                                         (static_cast<unsigned long long>(nspk) << 40) | total);
                if (logging) base_log = atomicAdd(I.spike_log_n, static_cast<unsigned long long>(nspk));
                atomicAdd(I.counters + 0, total);
                atomicAdd(I.counters + 2, static_cast<unsigned long long>(nspk));
            }
            base_spk = __shfl_sync(act, base_spk, leader);
            base_log = __shfl_sync(act, base_log, leader);
            if (spiked) {
                if (I.deferred_push) {
                    const std::size_t o = static_cast<std::size_t>(S.ls) * I.N + (base_spk >> 40) + rank;
                    const unsigned long long eoff = (base_spk & 0xFFFFFFFFFFull) + (incl - edges);
                    *reinterpret_cast<uint4*>(I.spk_meta + 4 * o) =
                        make_uint4(r1, static_cast<std::uint32_t>(eoff), r0, len0);
                    *reinterpret_cast<double2*>(I.spk_val + 2 * o) = make_double2(v0, v1);
                }
                if (logging) {
                    const unsigned long long li = base_log + rank;
                    if (li < I.spike_log_cap) {
                        I.spike_log[li] = (static_cast<unsigned long long>(step) << 32) | c;
                    } else {
                        atomicAdd(I.counters + 3, 1ULL);
                    }
                }
            }
        }

        if (I.rec_neuron_max > 0 && c < I.rec_neuron_max && S.rec_now) {
            const std::size_t row = S.rec_row;
            I.rec_V[row * I.rec_neuron_max + c] = V;
            I.rec_Isic[row * I.rec_neuron_max + c] = Isic;
        }
    }

    // Push the out-edges of this block's spiking sources into the rings of
    // their arrival steps (deliver_spikes, network.cpp:249-279) when the
    // push is not deferred to the next step.
    if (I.deferred_push) return;
    __syncthreads();
    const int nspk = s_nspk;
    for (int q = 0; q < nspk; ++q) {
        const std::uint32_t lane = s_spk[q];
        const std::uint32_t j = wk.first + lane;
        if (j < I.NE) {
            push_row(I.exc_rs, I.ring_ex, j, S.now_e, s_val[2 * lane]);
            push_row(I.n2a_rs, I.ring_as, j, S.now_e, s_val[2 * lane + 1]);
        } else {
            push_row(I.inh_rs, I.ring_in, j - I.NE, S.now_i, s_val[2 * lane]);
        }
    }
}

// Deferred push of the spikes of step-1.  The participating blocks stride
// over the flat edge space of that step (edge x belongs to the spike whose
// range holds it, found by binary search in shared memory), so the work is
// split evenly whatever the number of spikes.
constexpr int kPushBatch = 256;

// The deferred push of the spikes of step-1 by participant `rank` of
// `nranks` (each a block).  The spike list is cut into batches of
// kPushBatch spikes.  kDealt (the wide form, whose bursts have ~10^4 helper
// blocks and up to ~60 batches): the participants are dealt over the
// batches -- with at least as many participants as batches, the Q
// participants of batch b (ranks b, b + nbatch, ...) stage that batch once
// and share its edges, edge x going to thread (x - first edge) %
// (Q * blockDim.x) of them; with fewer, participant r pushes batches r,
// r + nranks, ... alone -- so a participant stages only the batches it
// pushes.  Otherwise (the latency form: tens of participants, one or two
// batches) every participant stages every batch and edge x of the flat edge
// space goes to thread x % (nranks * blockDim.x); the dealt form measured
// 0.16 us slower per paper-sparse step there.
template <bool kDealt>
__device__ void push_spikes(const InstDev& I, const StepInfo& S, unsigned long long packed,
                            std::uint32_t rank, std::uint32_t nranks) {
    __shared__ std::uint32_t s_off[kPushBatch + 1], s_r0[kPushBatch], s_len0[kPushBatch],
        s_r1[kPushBatch];
    __shared__ double s_v[2 * kPushBatch];
    const std::uint32_t n = static_cast<std::uint32_t>(packed >> 40);
    const std::uint32_t total = static_cast<std::uint32_t>(packed & 0xFFFFFFFFFFull);
    if (n == 0) return;  // block-uniform
    const std::uint32_t nbatch = (n + kPushBatch - 1) / kPushBatch;
    const std::uint32_t as_e = S.push_e, as_i = S.push_i;
    const std::size_t base = static_cast<std::size_t>(S.ls_prev) * I.N;
    // first batch, rank among the batch's participants, their number (no
    // division in the common single-batch case)
    std::uint32_t first = rank, q = 0, share = 1;
    if (!kDealt) {  // every batch, all participants
        first = 0;
        q = rank;
        share = nranks;
    } else if (nbatch == 1) {
        first = 0;
        q = rank;
        share = nranks;
    } else if (nranks > nbatch) {
        first = rank % nbatch;
        q = rank / nbatch;
        share = (nranks - 1 - first) / nbatch + 1;
    }
    const std::uint32_t stride = blockDim.x * share;
    const std::uint32_t gtid = q * blockDim.x + threadIdx.x;
    for (std::uint32_t bi = first; bi < nbatch; bi += kDealt ? nranks : 1u) {
        const std::uint32_t b0 = bi * kPushBatch;
        const std::uint32_t nb = min(static_cast<std::uint32_t>(kPushBatch), n - b0);
        __syncthreads();
        for (std::uint32_t i = threadIdx.x; i < nb; i += blockDim.x) {
            const std::size_t o = base + b0 + i;
            const uint4 m = __ldcg(reinterpret_cast<const uint4*>(I.spk_meta + 4 * o));
            const double2 v = __ldcg(reinterpret_cast<const double2*>(I.spk_val + 2 * o));
            s_r1[i] = m.x;  // n2a row start; kNoBit marks an inhibitory source
            s_off[i] = m.y;
            s_r0[i] = m.z;
            s_len0[i] = m.w;
            s_v[2 * i] = v.x;
            s_v[2 * i + 1] = v.y;
        }
        if (threadIdx.x == 0)
            s_off[nb] = b0 + nb < n ? __ldcg(I.spk_meta + 4 * (base + b0 + nb) + 1) : total;
        __syncthreads();
        // The list order is the atomic order, so offsets ascend along it.
        const std::uint32_t x0 = s_off[0], x1 = s_off[nb];
        // Groups of kPushGroup edges per thread: every edge word of the group
        // is loaded before the group's tickets are taken, so a thread waits
        // one round trip for its edges and one for its tickets per group.
        constexpr int kPushGroup = 4;
        for (std::uint32_t xg = x0 + gtid; xg < x1; xg += kPushGroup * stride) {
            unsigned long long pe[kPushGroup];
            double val[kPushGroup];
            int which[kPushGroup];  // 0 inh, 1 exc, 2 astrocyte, -1 none
#pragma unroll
            for (int u = 0; u < kPushGroup; ++u) {
                const std::uint32_t x = xg + static_cast<std::uint32_t>(u) * stride;
                which[u] = -1;
                pe[u] = 0;
                val[u] = 0.0;
                if (x < x1) {
                    std::uint32_t lo = 0, hi = nb;  // last entry with s_off <= x
                    while (hi - lo > 1) {
                        const std::uint32_t mid = (lo + hi) >> 1;
                        if (s_off[mid] <= x) lo = mid; else hi = mid;
                    }
                    const std::uint32_t k = x - s_off[lo];
                    if (s_r1[lo] == kNoBit) {
                        which[u] = 0;
                        pe[u] = __ldg(I.ring_in.edge + s_r0[lo] + k);
                        val[u] = s_v[2 * lo];
                    } else if (k < s_len0[lo]) {
                        which[u] = 1;
                        pe[u] = __ldg(I.ring_ex.edge + s_r0[lo] + k);
                        val[u] = s_v[2 * lo];
                    } else {
                        which[u] = 2;
                        pe[u] = __ldg(I.ring_as.edge + s_r1[lo] + (k - s_len0[lo]));
                        val[u] = s_v[2 * lo + 1];
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kPushGroup; ++u) {
                if (which[u] == 0) push_edge(I.ring_in, as_i, pe[u], val[u]);
                else if (which[u] == 1) push_edge(I.ring_ex, as_e, pe[u], val[u]);
                else if (which[u] == 2) push_edge(I.ring_as, as_e, pe[u], val[u]);
            }
        }
    }
}

// A burst: more than kBurstEdgesPerThread spike edges per push thread.
constexpr std::uint32_t kBurstEdgesPerThread = 4;

__device__ __forceinline__ bool push_burst(const InstDev& I, unsigned long long packed) {
    return (packed & 0xFFFFFFFFFFull) >
           static_cast<unsigned long long>(kBurstEdgesPerThread) * blockDim.x * I.push_blocks;
}

// Deferred push of the spikes of step-1 by the PUSH blocks (joined by every
// other block of the instance in a burst).  One thread also clears the list
// slot the next step appends to.
template <bool kPdl, bool kWide>
__device__ void push_role(const InstDev& I, const StepInfo& S, const Work& wk) {
    if (kPdl) grid_dep_wait();
    const std::int64_t step = S.step;
    if (step >= I.end_step) return;
    if (wk.first == 0 && threadIdx.x == 0) I.spk_packed[S.ls_next * kHeaderStride] = 0;
    if (step == 0) return;
    const unsigned long long packed = __ldcg(I.spk_packed + S.ls_prev * kHeaderStride);
    const std::uint32_t nranks = static_cast<std::uint32_t>(I.push_blocks) +
                                 (push_burst(I, packed) ? I.push_helpers : 0u);
    push_spikes<kWide>(I, S, packed, wk.first, nranks);
}

// A non-push block's share of a burst push, after its own role.
// A non-push block's share of a burst push (its rank among the helpers).
template <bool kWide>
__device__ __noinline__ void help_push_spikes(const InstDev& I, const StepInfo& S,
                                              unsigned long long packed, std::uint32_t helper) {
    push_spikes<kWide>(I, S, packed, static_cast<std::uint32_t>(I.push_blocks) + helper,
                static_cast<std::uint32_t>(I.push_blocks + I.push_helpers));
}

// After its own role, a block joins the push of step-1's spikes when that
// push is a burst.  `burst` carries the answer across the items a block runs
// in one step of one instance (-1: not known yet, else 0 or 1), so the spike
// count is read once per block rather than once per item; the new answer is
// returned.  Only a burst leaves the inline path.
template <bool kWide>
__device__ __forceinline__ int help_push(const InstDev& I, const StepInfo& S, const Work& wk,
                                         int burst) {
    if (burst == 0 || !I.deferred_push || wk.helper == kNoHelper || S.step == 0 ||
        S.step >= I.end_step)
        return burst;
    const unsigned long long packed = __ldcg(I.spk_packed + S.ls_prev * kHeaderStride);
    if (!push_burst(I, packed)) return 0;
    help_push_spikes<kWide>(I, S, packed, wk.helper);
    return 1;
}

// The precision study's astrocyte update (astro_rk4_f32): state, parameters
// and input rounded to float, the update in float, the result held as the
// double of that float.  Out of line: the FP64 path carries none of it.
__device__ __noinline__ void astro_update_f32(const InstDev& I, double ca_tot, double ip3_0,
                                              double tau, double delta, double input,
                                              double noise, double& ca, double& ip3,
                                              double& hh) {
    float c = static_cast<float>(ca), i3 = static_cast<float>(ip3), hv = static_cast<float>(hh);
    astro_rk4_f32(astro_k_f32(I.ak), static_cast<float>(ca_tot), static_cast<float>(ip3_0),
                  static_cast<float>(tau), static_cast<float>(delta), static_cast<float>(input),
                  static_cast<float>(noise), c, i3, hv);
    ca = c;
    ip3 = i3;
    hh = hv;
}

template <bool kPdl, bool kF32>
__device__ void astro_role(const InstDev& I, const StepInfo& S, const Work& wk) {
    const std::uint32_t a = wk.first + threadIdx.x;
    const bool active = threadIdx.x < wk.count;
    double ca_tot = I.Ca_tot_u, ip3_0 = I.IP3_0_u, tau = I.tau_u, inv_tau = I.inv_tau_u,
           delta = I.delta_u;
    if (active && !I.astro_uniform) {
        ca_tot = I.Ca_tot[a];
        ip3_0 = I.IP3_0[a];
        tau = I.tau[a];
        inv_tau = I.inv_tau[a];
        delta = I.delta[a];
    }
    if (kPdl) grid_dep_wait();
    const std::int64_t step = S.step;
    // The next step's emission flag starts clear (nothing reads or writes
    // that entry during this step: see InstDev::fac_any).
    if (wk.first == 0 && threadIdx.x == 0 && step < I.end_step) I.fac_any[S.fany_next] = 0u;
    if (!active || step >= I.end_step) return;
    const std::uint32_t slot = S.slot;
    const std::size_t ts = static_cast<std::size_t>(slot) * I.ring_as.n_targets + a;
    const std::uint32_t n = __ldcg(I.ring_as.cnt + ts);
    double ca = I.Ca[a], ip3 = I.IP3[a], hh = I.h[a];
    // drive_astrocytes (network.cpp:340-355) and the noise draw
    // (astrocyte.cpp:307-329): no memory, overlapping the loads.
    int ev = 0;
    if (I.a_rate > 0.0) {
        Draws r(I.seed ^ kSaltAstroPoisson, static_cast<std::uint64_t>(step) * kStreamStride + a);
        ev = r.poisson(I.a_lambda, I.a_limit);
    }
    double noise = 0.0;  // a_std * z, z drawn once per noise interval
    if (I.a_std > 0.0) {
        if (S.fresh_a) {
            const std::uint64_t nseed = I.seed ^ kSaltAstroNoise;
            noise = I.a_std * normal_clamped_at(nseed, I.a_indep ? S.noise_a * kStreamStride + a
                                                                 : S.noise_a);
            I.noise_a[a] = noise;
        } else {
            noise = I.noise_a[a];
        }
    }
    double ip3_in = 0.0;
    if (n) {
        const ShortList l = load_list(I.ring_as, ts);
        I.ring_as.cnt[ts] = 0;
        const double v = sum_arrivals<false>(I.ring_as, slot, a, n, l);
        if (v != 0.0) ip3_in += v;
    }
    if (ev > 0) ip3_in += I.a_weight * static_cast<double>(ev);
    // AstrocytePopulation::update (astrocyte.cpp:307-329)
    // (the precision study's FP32 form is a separate instantiation: the FP64
    // kernels carry none of its code)
    if constexpr (kF32)
        astro_update_f32(I, ca_tot, ip3_0, tau, delta, ip3_in, noise, ca, ip3, hh);
    else
        astro_rk4<false>(I.ak, ca_tot, ip3_0, tau, inv_tau, delta, ip3_in, noise, ca, ip3, hh);
    I.Ca[a] = ca;
    I.IP3[a] = ip3;
    I.h[a] = hh;
    // SIC factor of this step (astrocyte.cpp:331-339), read by the SIC sums
    // of the arrival step.
    if (S.fac_now) {
        const double y = (ca - I.SIC_th) * 1000.0;
        const double f = y <= 1.0 ? 0.0 : I.SIC_scale * log(y);
        I.fac[static_cast<std::size_t>(slot) * I.NA + a] = f;
        if (f != 0.0) I.fac_any[S.fany_now] = 1u;  // every writer stores the same 1
    }
    if (I.rec_astro_max > 0 && a < I.rec_astro_max && S.rec_now) {
        const std::size_t row = S.rec_row;
        I.rec_Ca[row * I.rec_astro_max + a] = ca;
        I.rec_IP3[row * I.rec_astro_max + a] = ip3;
    }
}

// Part p of the SIC sum of arrival step A = step+P-p (valid when d_a2n > P:
// its factors were written by a launch that has completed).  Part 0 starts
// from zero, part p > 0 continues the partial sum part p-1 left at step-1,
// the last part writes the SIC current of A = step+1.  The list entries are
// static and are read before the wait; after it, the partial sum and one
// batch of factor loads.  Edges are counted by the step that adds them,
// also for arrivals past the end of the chunk (the next chunk uses them).
template <bool kPdl>
__device__ void sic_role(const InstDev& I, const StepInfo& S, const Work& wk) {
    const std::uint32_t v = wk.first + threadIdx.x;  // part * sic_npad + target
    const std::uint32_t p = v / I.sic_npad, t = v - p * I.sic_npad;
    const std::uint32_t P = static_cast<std::uint32_t>(I.sic_parts);
    const bool on = threadIdx.x < wk.count && t < I.N && ((S.sic_due >> p) & 1u);
    std::uint32_t o0 = 0, len = 0, e[kSicBatch];
    if (on) {
        sic_prefetch(I, v, o0, len, e);
    } else {
#pragma unroll
        for (int k = 0; k < kSicBatch; ++k) e[k] = 0u;
    }
    if (kPdl) grid_dep_wait();
    if (S.step >= I.end_step) return;
    unsigned long long edges = 0;
    if (on) {
        const std::size_t part_n = static_cast<std::size_t>(P - 1) * I.sic_npad;
        const double acc0 =
            p == 0 ? 0.0
                   : __ldcg(I.sic_part + static_cast<std::size_t>((S.step + 1) & 1) * part_n +
                            static_cast<std::size_t>(p - 1) * I.sic_npad + t);
        const double acc = sic_sum(I, o0, len, e, S.sic_slot[p], acc0, edges);
        if (p + 1 == P) {
            I.sic_val[static_cast<std::size_t>((S.step + 1) & (I.sic_ring - 1)) * I.N + t] = acc;
        } else {
            I.sic_part[static_cast<std::size_t>(S.step & 1) * part_n +
                       static_cast<std::size_t>(p) * I.sic_npad + t] = acc;
        }
    }
    // one atomic per warp
    for (int o = 16; o > 0; o >>= 1) edges += __shfl_down_sync(0xFFFFFFFFu, edges, o);
    if ((threadIdx.x & 31) == 0 && edges) atomicAdd(I.counters + 1, edges);
}

template <bool kPdl, bool kF32, bool kWide>
__device__ __forceinline__ int run_role(const InstDev& I, const StepInfo& S, const Work& wk,
                                        int burst) {
    if (wk.role == kRolePush) {
        push_role<kPdl, kWide>(I, S, wk);
        return burst;
    }
    if (wk.role == kRoleNeuron) {
        neuron_role<kPdl, kWide>(I, S, wk);
    } else if (wk.role == kRoleAstro) {
        astro_role<kPdl, kF32>(I, S, wk);
    } else {
        sic_role<kPdl>(I, S, wk);
    }
    return help_push<kWide>(I, S, wk, burst);
}

// One step of every resident instance (the body of both kernel forms below).
// kLoop: block b runs work items b, b + gridDim.x, ... -- several when the
// grid is one wave of resident blocks (a large step), which saves the
// per-block staging and scheduling of the items after the first.  Without
// kLoop the grid covers the work table and block b runs item b alone (a step
// of a few waves: no loop structure on its path).  No item waits on another
// within a launch, so any assignment of items to blocks is valid.
template <bool kF32, bool kLoop>
__device__ __forceinline__ void step_body(const InstDev* __restrict__ insts,
                                          const Work* __restrict__ work, int k, int n_work) {
    // Stage the item's instance descriptor and step arithmetic in shared
    // memory (again only when the instance changes).  Both depend only on
    // data written before the chunk started, so this overlaps the tail of
    // the previous step's grid.
    __shared__ __align__(16) unsigned char s_raw[sizeof(InstDev)];
    __shared__ StepInfo s_info;
    const InstDev& I = *reinterpret_cast<const InstDev*>(s_raw);
    if constexpr (!kLoop) {
        const Work wk = load_work(work + blockIdx.x);  // gridDim.x == n_work
        const auto* src = reinterpret_cast<const std::uint32_t*>(insts + wk.inst);
        auto* dst = reinterpret_cast<std::uint32_t*>(s_raw);
        for (unsigned i = threadIdx.x; i < sizeof(InstDev) / 4; i += blockDim.x)
            dst[i] = __ldcg(src + i);
        __syncthreads();
        if (threadIdx.x < 32) make_step_info(I, I.step0 + k, s_info);
        __syncthreads();
        asm volatile("griddepcontrol.launch_dependents;");  // see below
        run_role<true, kF32, false>(I, s_info, wk, -1);
        (void)n_work;
        return;
    }
    std::uint32_t staged = 0xFFFFFFFFu;
    int burst = -1;  // help_push's answer for this step of the staged instance
    for (int wi = blockIdx.x; wi < n_work; wi += gridDim.x) {
        // Through L2 (never a cached line of an earlier chunk or engine):
        // the descriptors are rewritten by a host copy before every chunk.
        const Work wk = load_work(work + wi);
        if (wk.inst != staged) {  // block-uniform
            __syncthreads();      // the previous item is done with s_raw / s_info
            const auto* src = reinterpret_cast<const std::uint32_t*>(insts + wk.inst);
            auto* dst = reinterpret_cast<std::uint32_t*>(s_raw);
            for (unsigned i = threadIdx.x; i < sizeof(InstDev) / 4; i += blockDim.x)
                dst[i] = __ldcg(src + i);
            __syncthreads();
            if (threadIdx.x < 32) make_step_info(I, I.step0 + k, s_info);
            __syncthreads();
            if (staged == 0xFFFFFFFFu) {
                // Programmatic dependent launch: let the next step's grid be
                // scheduled now.  Each role waits (griddepcontrol.wait) for
                // this launch's predecessor to complete before touching
                // state it writes.
                asm volatile("griddepcontrol.launch_dependents;");
            }
            staged = wk.inst;
            burst = -1;
        }
        burst = run_role<true, kF32, true>(I, s_info, wk, burst);
        __syncthreads();  // the role's shared arrays are free for the next item
    }
}

// Two forms of the step kernel, same arithmetic: step_kernel allows blocks of
// up to kMaxBlock threads and 128 registers per thread (4 blocks of 128
// threads per SM; the fewest dependent round trips, for steps of a few
// waves); step_kernel_wide is for 128-thread blocks at 6 per SM (80
// registers, some spilled: more warps to hide latency when a step is many
// waves of blocks).
template <bool kF32>
__global__ void __launch_bounds__(kMaxBlock) step_kernel(const InstDev* __restrict__ insts,
                                                         const Work* __restrict__ work, int k,
                                                         int n_work) {
    step_body<kF32, false>(insts, work, k, n_work);
}

template <bool kF32>
__global__ void __launch_bounds__(128, 6) step_kernel_wide(const InstDev* __restrict__ insts,
                                                           const Work* __restrict__ work, int k,
                                                           int n_work) {
    step_body<kF32, true>(insts, work, k, n_work);
}

// Grid-wide barrier of the persistent chunk kernel (all blocks co-resident
// by cooperative launch).  Sense by generation count; every wait is bounded:
// a block still waiting after kBarrierWaitNs (or kBarrierPolls polls) sets the error word
// and the whole grid stops at its next barrier, so a fault can only end the
// launch early, never hang it.
// The wait is bounded by time: 1 s on the GPU's global timer (ns).  A poll
// count bounds it as well, as a backstop that does not depend on the timer
// (each poll sleeps ~64 ns and makes an acquire load: well above 1 s).
constexpr unsigned long long kBarrierWaitNs = 1000000000ull;
constexpr unsigned kBarrierPolls = 1u << 26;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ bool grid_sync(GridBarrier* gb, unsigned nblocks) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned gen = ld_acquire(&gb->gen);
        __threadfence();
        int ok = 1;
        if (atomicAdd(&gb->count, 1u) == nblocks - 1) {
            atomicExch(&gb->count, 0u);
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        } else {
            unsigned polls = 0;
            const unsigned long long t0 = global_ns();
            while (ld_acquire(&gb->gen) == gen) {
                if (++polls > kBarrierPolls || ld_acquire(&gb->error) != 0 ||
                    global_ns() - t0 > kBarrierWaitNs) {
                    atomicExch(&gb->error, 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (ld_acquire(&gb->error) != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// All `steps` steps of a chunk in one cooperative launch: each block takes
// work items blockIdx.x, blockIdx.x + gridDim.x, ... of every step, with a
// grid barrier between steps.  Data other blocks wrote in earlier steps is
// read through L2 (__ldcg in the roles), never a stale L1 line.
template <bool kF32>
__global__ void __launch_bounds__(kMaxBlock) chunk_kernel(const InstDev* __restrict__ insts,
                                                          const Work* __restrict__ work,
                                                          int n_work, int steps,
                                                          GridBarrier* gb) {
    __shared__ __align__(16) unsigned char s_raw[sizeof(InstDev)];
    __shared__ StepInfo s_info;
    __shared__ unsigned s_inst;
    if (threadIdx.x == 0) s_inst = 0xFFFFFFFFu;
    const InstDev& I = *reinterpret_cast<const InstDev*>(s_raw);
    for (int k = 0; k < steps; ++k) {
        for (int wi = blockIdx.x; wi < n_work; wi += gridDim.x) {
            const Work wk = load_work(work + wi);
            __syncthreads();
            if (s_inst != wk.inst) {
                const auto* src = reinterpret_cast<const std::uint32_t*>(insts + wk.inst);
                auto* dst = reinterpret_cast<std::uint32_t*>(s_raw);
                for (unsigned i = threadIdx.x; i < sizeof(InstDev) / 4; i += blockDim.x)
                    dst[i] = __ldcg(src + i);
                __syncthreads();
                if (threadIdx.x == 0) s_inst = wk.inst;
            }
            if (threadIdx.x < 32) make_step_info(I, I.step0 + k, s_info);
            __syncthreads();
            if (s_info.step < I.end_step) run_role<false, kF32, false>(I, s_info, wk, -1);
        }
        if (k + 1 < steps && !grid_sync(gb, gridDim.x)) return;
    }
}

// Side-stream SIC batch: thread per target, its whole list (P = 1), and the
// sums of all kSicBatchSteps arrival steps of the batch at once: for each
// list entry the factors of the astrocyte at the arrivals' emission steps
// are loaded together, and the m additions of the entry advance the
// kSicBatchSteps sums side by side -- independent chains, each the SIC
// role's sequential sum (a zero factor adds +0.0, exact since a sum that
// starts at +0.0 and adds nonzero values is never -0.0).  One block per
// work item, so the batch leaves the SMs to the step kernels beside it.
// Launched when the step before step0+k has completed (the factors it
// needs are older still), and waited for before the first step that reads it.
__global__ void __launch_bounds__(kMaxBlock) sic_batch_kernel(const InstDev* __restrict__ insts,
                                                              const Work* __restrict__ work,
                                                              int k) {
    constexpr int G = kSicBatchSteps;
    const Work wk = load_work(work + blockIdx.x);
    const InstDev& I = insts[wk.inst];
    unsigned long long edges = 0;
    if (threadIdx.x < wk.count) {
        const std::uint32_t t = wk.first + threadIdx.x;
        std::uint32_t o0 = 0, len = 0, e[kSicBatch];
        sic_prefetch(I, t, o0, len, e);
        const double* fac[G];
        bool due[G];
        double acc[G];
#pragma unroll
        for (int j = 0; j < G; ++j) {
            const std::int64_t a = I.step0 + k + I.sic_lead + j;
            const std::int64_t se = a - I.d_a2n;
            due[j] = a >= I.step0 && se >= 0 && se % I.sic_interval == 0;
            fac[j] = I.fac + static_cast<std::size_t>(due[j] ? se % I.slots : 0) * I.NA;
            acc[j] = 0.0;
        }
        for (std::uint32_t b0 = 0;; b0 += kSicBatch) {
            bool done = false;
            for (int q = 0; q < kSicBatch; ++q) {
                const std::uint32_t m = e[q] & 0xFFu;
                if (m == 0) {
                    done = true;  // padding ends the list
                    break;
                }
                const std::uint32_t as = e[q] >> 8;
                double c[G];
#pragma unroll
                for (int j = 0; j < G; ++j) {
                    const double f = __ldcg(fac[j] + as);
                    c[j] = I.w_a2n * f;
                    if (due[j] && f != 0.0) edges += m;
                    if (f == 0.0) c[j] = 0.0;
                }
                for (std::uint32_t r = 0; r < m; ++r) {
#pragma unroll
                    for (int j = 0; j < G; ++j) acc[j] += c[j];
                }
            }
            if (done || b0 + kSicBatch >= len) break;
#pragma unroll
            for (int q = 0; q < kSicBatch; ++q) {
                const std::uint32_t jj = b0 + kSicBatch + q;
                e[q] = jj < len ? __ldg(I.sic_ent + o0 + jj * 32) : 0u;
            }
        }
#pragma unroll
        for (int j = 0; j < G; ++j) {
            const std::int64_t a = I.step0 + k + I.sic_lead + j;
            if (due[j]) I.sic_val[static_cast<std::size_t>(a & (I.sic_ring - 1)) * I.N + t] = acc[j];
        }
    }
    for (int o = 16; o > 0; o >>= 1) edges += __shfl_down_sync(0xFFFFFFFFu, edges, o);
    if ((threadIdx.x & 31) == 0 && edges) atomicAdd(I.counters + 1, edges);
}

// Failure-detection check of the bounded barrier: block 0 never arrives, so
// every other block's wait must run out, set the error word and return.
__global__ void barrier_selftest_kernel(GridBarrier* gb) {
    if (blockIdx.x == 0) return;
    grid_sync(gb, gridDim.x);
}

}  // namespace

cudaError_t launch_sic_batch(const InstDev* insts, const Work* work, int n_work, int block, int k,
                             cudaStream_t stream) {
    sic_batch_kernel<<<static_cast<unsigned>(n_work), block, 0, stream>>>(insts, work, k);
    return cudaGetLastError();
}

cudaError_t barrier_selftest(GridBarrier* gb, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(4);
    cfg.blockDim = dim3(32);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, barrier_selftest_kernel, gb);
}

int persistent_blocks(int block) {
    int per_sm = 0, dev = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, chunk_kernel<false>, block, 0) !=
        cudaSuccess)
        return 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return per_sm * sms;
}

cudaError_t launch_chunk_persistent(const InstDev* insts, const Work* work, int n_work,
                                    int block, int grid, int steps, GridBarrier* gb, bool f32,
                                    cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(static_cast<unsigned>(block));
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (f32) return cudaLaunchKernelEx(&cfg, chunk_kernel<true>, insts, work, n_work, steps, gb);
    return cudaLaunchKernelEx(&cfg, chunk_kernel<false>, insts, work, n_work, steps, gb);
}

int step_wide_blocks_per_sm() {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, step_kernel_wide<false>, 128, 0) !=
        cudaSuccess)
        return 0;
    return nb;
}

cudaError_t launch_step(const InstDev* insts, const Work* work, int n_work, int block, int k,
                        bool pdl, bool wide, int max_grid, bool f32, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(max_grid > 0 ? std::min(n_work, max_grid) : n_work));
    cfg.blockDim = dim3(static_cast<unsigned>(block));
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = pdl ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (wide && block == 128)
        return f32 ? cudaLaunchKernelEx(&cfg, step_kernel_wide<true>, insts, work, k, n_work)
                   : cudaLaunchKernelEx(&cfg, step_kernel_wide<false>, insts, work, k, n_work);
    return f32 ? cudaLaunchKernelEx(&cfg, step_kernel<true>, insts, work, k, n_work)
               : cudaLaunchKernelEx(&cfg, step_kernel<false>, insts, work, k, n_work);
}

}  // namespace asg
