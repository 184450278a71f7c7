// Device data layout of the network engine (one descriptor per instance) and
// the fused per-timestep kernel.
//
// One kernel launch advances every resident instance by one step.  Its
// blocks are typed by a work table built on the host:
//   NEURON  arrivals (exc/inh rings, SIC), Poisson drive, noise, AdEx RK4,
//           spike test, STP update of the spiking source and the push of its
//           out-edges into the arrival rings of later steps;
//   ASTRO   arrivals (neuron->astrocyte ring), Poisson drive, noise, Li-Rinzel
//           RK4, SIC factor of the step;
//   SIC     (only when the SIC delay is >= 2 steps) the SIC current arriving
//           at the NEXT step, summed from the factors of its emission step.
// No role waits on another inside a launch: every cross-cell read is of data
// written by an earlier launch (delays are >= 1 step), so one launch per step
// is the only synchronisation, and K steps are one captured CUDA graph.
//
// Exact, reproducible arrivals without floating-point atomics
// ----------------------------------------------------------
// The reference sums each ring entry sequentially in ascending source order
// (network.cpp:249-279).  Here every target numbers its incoming edges in
// (source, position in the source's row) order; an arrival is identified by
// that number (its "bit").  A push takes a ticket from the target's per-slot
// arrival counter (integer atomicAdd).  Tickets 0..kListCap-1 store (bit,
// value) in the target's short list for the slot; later tickets store the
// value at the bit's position, set the bit in the target's bitmap words
// (integer atomicOr, no return value) and set the target's summary bit for
// the word group holding it (64-bit summary per target and slot).  The
// target, when the slot arrives, reads its counter; for up to kListCap
// arrivals it loads the list in one batch and sorts it by bit; beyond that it
// also walks the set bits of its bitmap words in ascending order, merging
// them with the sorted list (a target of at most 32 words loads all of them
// in one batch; a larger one visits the non-empty words its summary names).
// Either way the
// values are added left to right in ascending bit order: the reference's
// IEEE operations in the reference's order, hence bitwise equal, for any
// number of coincident spikes and any interleaving of the pushes.  Reading
// clears the counter, the summary and the words it used.
//
// STP: the reference keeps x, u, t_last per edge, but all edges of a source
// start equal (network.cpp:43-52) and are updated together on each spike of
// that source, so they stay equal: one state per source is exact.  The
// spiking thread updates it and forms w*x*u once per set.
//
// SIC: the reference adds w_a2n*factor(a) once per astrocyte->neuron edge, in
// ascending astrocyte order (network.cpp:281-299).  A target's edges from one
// astrocyte all add the same value, so its list is stored compressed as
// (astrocyte, multiplicity) pairs in ascending astrocyte order and summed
// sequentially -- same operations, far fewer bytes.  The sum is one chain
// of dependent additions (hundreds per target), so when the SIC delay
// allows it the chain is cut into P consecutive parts of about equal edge
// count, computed on P consecutive steps by P threads: the part-p thread of
// step s continues, for the arrival step s+P-p, the partial sum the
// part-(p-1) thread left at step s-1.  Every addition is the reference's, in
// its order; a step's longest chain is 1/P of a target's.  Layout: sliced ELL with
// slices of 32 targets (one warp), entries packed as astro << 8 | mult.
#pragma once

#include <cstdint>

#include "asg_device.cuh"

namespace asg {

enum Role : std::uint16_t { kRoleNeuron = 0, kRoleAstro = 1, kRoleSic = 2, kRolePush = 3 };

struct Work {
    std::uint32_t inst;
    std::uint16_t role;
    std::uint16_t helper;  // rank among the instance's push helpers (kNoHelper: none)
    std::uint32_t first;
    std::uint32_t count;
};

constexpr std::uint16_t kNoHelper = 0xFFFFu;

// Incoming-edge structure of one arrival ring (transpose of a source CSR).
constexpr int kListCap = 4;      // arrivals per (slot, target) held in the short list
constexpr int kMaxSicParts = 8;  // most parts a target's SIC chain is cut into
constexpr int kHeaderStride = 16;  // u64 words between spike-list headers (128 bytes)
constexpr int kSicBatchSteps = 8;  // arrival steps per side-stream SIC batch
constexpr int kSicRing = 32;       // SIC value slots of an instance with side batches

struct InRing {
    const std::uint32_t* wbase;   // [n_targets+1] first bitmap word of each target
    // [E] per OUT-edge (source CSR order): bit index | target << 32 | dense
    // << 57 (target of at most 32 words: no summary) | summary bit << 58 --
    // one 8-byte load gives everything a push needs.
    const unsigned long long* edge;
    std::uint32_t* cnt;           // [slots][n_targets] arrivals pushed into the slot
    std::uint32_t* lbit;          // [slots][n_targets][kListCap] bits of the first arrivals
    double* lval;                 // [slots][n_targets][kListCap] their values
    std::uint32_t* bits;          // [slots][words] bitmaps of the later arrivals
    unsigned long long* sum;      // [slots][n_targets] non-empty word groups (targets of > 32 words)
    double* vals;                 // [slots][words*32] value at each set bit
    std::uint32_t words;          // total bitmap words of one slot
    std::uint32_t n_targets;
};

struct InstDev {
    // sizes and time
    std::uint32_t N, NE, NA;
    std::int32_t slots, d_e, d_i, d_a2n, sic_interval;
    std::int32_t fused_sic;  // 1: neuron thread sums its own SIC
    std::int32_t stp_on;
    std::int64_t step0;      // step of kernel index 0 in the current chunk
    std::int64_t end_step;   // first step this instance does not run
    std::uint64_t seed;
    double dt;
    // neuron populations
    NeuronK pe, pi;
    double sh_std_e, sh_std_i;  // shared-noise std (0 unless shared noise is on)
    // astrocytes
    AstroK ak;
    std::int32_t astro_uniform;
    std::int32_t astro_fp32;  // precision study: the astrocyte update in FP32
    double Ca_tot_u, IP3_0_u, tau_u, delta_u, inv_tau_u;
    double a_rate, a_weight, a_lambda, a_limit, a_std;
    std::int32_t a_indep, a_steps_per_noise;
    // Noise terms of the current noise interval: a draw index changes every
    // steps_per_noise steps, and between changes the term is read back here
    // instead of drawn again (the same bits: the draw depends only on seed,
    // index and cell).  Drawn afresh at each interval's first step and at
    // noise_from, the first step after the instance was created or restored.
    double* noise_n;  // [N]  noise_std * z of each neuron
    double* noise_a;  // [NA] a_std * z of each astrocyte
    std::int64_t noise_from;
    double SIC_scale, SIC_th;
    // synapses
    double w_e, w_i, w_n2a, w_a2n, U, tau_rec, tau_fac;
    // neuron state
    double *V, *w, *gex, *dgex, *gin, *dgin, *Isic;
    std::int32_t* refr;
    const double *V_reset, *b;
    // astrocyte state / params
    double *Ca, *IP3, *h;
    const double *Ca_tot, *IP3_0, *tau, *inv_tau, *delta;
    double inv_tau_rec, inv_tau_fac;  // correctly rounded reciprocals (div_by)
    // STP per source
    double *stp_x, *stp_u, *stp_t;
    // row starts of the three spike-carrying sets (source CSR order); the
    // edges themselves are the rings' packed `edge` words
    const std::uint32_t *exc_rs, *inh_rs, *n2a_rs;
    InRing ring_ex, ring_in, ring_as;
    // Deferred push (both spike delays >= 2 steps): each spike of step s
    // reserves a contiguous range of that step's flat edge space (one 64-bit
    // atomic: list index in the high bits, edge offset in the low 40) and is
    // pushed in step s+1 by the PUSH blocks, whose threads stride over the
    // flat space -- every edge of every spike gets one thread, whatever the
    // spike count.  Three list slots rotate: append (s), push (s-1), reset (s+1).
    std::int32_t deferred_push;
    std::int32_t push_blocks;          // PUSH work items of this instance
    // In a burst (many more spike edges than push threads) every other work
    // item of the instance joins the push after its own role: push_helpers
    // of them, ranks push_blocks.. in the flat edge space.
    std::int32_t push_helpers;
    // [3][kHeaderStride]: count << 40 | edges, one 128-byte line per slot --
    // the slot being appended to (atomics) and the slot being read by every
    // block must not share an L2 sector, or the reads queue behind the atomics.
    unsigned long long* spk_packed;
    std::uint32_t* spk_meta;           // [3][N][4]: n2a row start (~0: inhibitory source),
                                       // edge offset, row0 start, row0 length
    double* spk_val;                   // [3][N][2]: exc or inh set value, n2a value
    // SIC: sliced ELL over virtual targets v = part * sic_npad + target,
    // factors per emission slot, partial sums between parts, final values.
    // With sic_side the currents are computed off the step kernels, by
    // side-stream batches: the batch launched before step s (s a multiple of
    // kSicBatchSteps in the chunk) covers the arrival steps s+sic_lead ..
    // s+sic_lead+kSicBatchSteps-1, one whole chain per thread (P = 1).
    std::int32_t sic_side;
    std::int32_t sic_lead;
    std::int32_t sic_ring;          // slots of sic_val, a power of two
    std::int32_t sic_parts;         // P (1 when the delay is too short to split)
    std::uint32_t sic_npad;         // N rounded up to a multiple of 32
    const std::uint32_t* sic_soff;  // [P*sic_npad/32+1] entry offset of each 32-target slice
    const std::uint32_t* sic_ent;   // astro << 8 | mult
    double* fac;                    // [slots][NA]
    // fac_any[e % (slots + 1)] != 0: some factor of emission step e is
    // non-zero.  Set by the astrocyte role, cleared one step ahead by the
    // instance's first astrocyte block; a fused SIC sum of an arrival whose
    // emission had none is the +0.0 it would add up to, without its loads.
    std::uint32_t* fac_any;         // [slots + 1]
    double* sic_part;               // [2][P-1][sic_npad] partial sums, by step parity
    double* sic_val;                // [sic_ring][N], slot = arrival step % sic_ring
    // outputs (host-mapped memory)
    unsigned long long* spike_log;  // (step << 32) | source
    unsigned long long* spike_log_n;
    std::uint32_t spike_log_cap;
    std::int32_t rec_spikes;
    std::int64_t rec_from;
    std::int32_t rec_every;
    std::uint32_t rec_astro_max, rec_neuron_max, rec_rows;  // rows held in the ring below
    double *rec_Ca, *rec_IP3, *rec_V, *rec_Isic;             // [rec_rows][max]
    unsigned long long* counters;  // spike_edges, sic_edges, spikes, overflow
};

// Barrier words of the persistent chunk kernel (device memory, zeroed).
struct GridBarrier {
    unsigned count, gen, error, pad;
};

// Launches 4 blocks of which one never reaches the barrier (self-test of the
// bounded wait: the others must give up and set gb->error).
cudaError_t barrier_selftest(GridBarrier* gb, cudaStream_t stream);

// Co-resident blocks of the persistent chunk kernel at this block size.
int persistent_blocks(int block);
// All `steps` steps of a chunk in one cooperative launch of `grid` blocks.
cudaError_t launch_chunk_persistent(const InstDev* insts, const Work* work, int n_work,
                                    int block, int grid, int steps, GridBarrier* gb, bool f32,
                                    cudaStream_t stream);

// One side-stream SIC batch (instances with sic_side): the arrival steps
// step0+k+sic_lead .. +kSicBatchSteps-1 of every work item's targets.
cudaError_t launch_sic_batch(const InstDev* insts, const Work* work, int n_work, int block, int k,
                             cudaStream_t stream);

// One step launch; with `pdl` the launch may start while the previous kernel
// of the stream is still running (the kernel waits for it before any access
// to instance state).
// `wide`: the high-occupancy form (block 128 only; same arithmetic).
// One step launch over the work table.  max_grid > 0 caps the grid (blocks
// then run several work items each); 0 launches one block per item.
cudaError_t launch_step(const InstDev* insts, const Work* work, int n_work, int block, int k,
                        bool pdl, bool wide, int max_grid, bool f32, cudaStream_t stream);
// Resident blocks per SM of the high-occupancy step kernel form (128 threads).
int step_wide_blocks_per_sm();

}  // namespace asg
