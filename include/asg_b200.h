/*
 * asg_b200.h -- C ABI of the B200-native per-timestep engine for the
 * astrosimgpu neuron-astrocyte network (AdEx RK4 neurons, Li-Rinzel
 * astrocytes, CSR spike delivery with Tsodyks-Markram STP into per-delay
 * rings, astrocytic SIC return current).  FP64 throughout, one GPU.
 *
 * Plain C: pointers, sizes and status codes.  No CUDA or C++ types cross
 * this boundary.  Every entry point returns an int status (ASG_OK == 0);
 * asg_last_error() gives the text of the most recent failure on the calling
 * thread.  Nothing aborts the process.
 *
 * Threading: one handle per host thread.  Calls on one handle are
 * serialised by the caller; each handle owns its own CUDA stream.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   - the per-step loop body of Network::run          src/network.cpp:385-431
 *     (apply_arrivals, drive_astrocytes, AstrocytePopulation::update,
 *      NeuronPopulation::update, deliver_spikes, deliver_sic)
 *   - the native CUDA astrocyte backend               include/astrosimgpu/astrocyte_cuda.hpp:15-27
 *   - Network(ModelConfig) + build()                  include/astrosimgpu/network.hpp:58-67
 *   - load_config(path)                               include/astrosimgpu/parameters.hpp:202
 */
#ifndef ASG_B200_H
#define ASG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define ASG_OK 0
#define ASG_ERR_ARG 1          /* invalid argument or size                     */
#define ASG_ERR_OOM 2          /* device or host allocation failed / over budget */
#define ASG_ERR_CUDA 3         /* CUDA runtime error (text in asg_last_error)  */
#define ASG_ERR_UNSUPPORTED 4  /* input outside what the engine implements    */
#define ASG_ERR_TIMEOUT 5      /* a bounded device wait gave up               */
#define ASG_ERR_OVERFLOW 6     /* an output buffer was too small              */
#define ASG_ERR_CONFIG 7       /* malformed configuration / unknown key       */
#define ASG_ERR_STATE 8        /* call not valid in the handle's state        */
#define ASG_ERR_CANCELLED 9    /* serving request was cancelled               */
#define ASG_ERR_NO_DEVICE 10   /* no CUDA device visible                      */
#define ASG_ERR_NOT_FOUND 11   /* unknown instance / request id               */

/* Text of the last error raised on this thread ("" if none). */
const char* asg_last_error(void);
/* Library version string. */
const char* asg_version(void);

/* ------------------------------------------------------- model parameters
 * Field meanings and units follow the reference's parameters.hpp:14-198.   */

/* NeuronParams (parameters.hpp:44-62) minus the per-cell V_reset and b,
 * which the reference randomises per cell (neuron.cpp:150-153). */
typedef struct asg_neuron_params {
    double C_m, g_L, E_L, V_th, Delta_T, a, tau_w, V_peak, t_ref, E_ex, E_in, tau_syn_ex,
        tau_syn_in, I_e;
} asg_neuron_params;

/* AstroConstants (astrocyte_kernel.hpp:29-40) + SIC_scale, SIC_th. */
typedef struct asg_astro_params {
    double Kd_IP3_1, Kd_IP3_2, Kd_act, Kd_inh, Km_SERCA, k_IP3R, rate_IP3R, rate_L, rate_SERCA,
        ratio_ER_cyt, SIC_scale, SIC_th;
} asg_astro_params;

/* InputParams (parameters.hpp:134-140); noise_dt already resolved (> 0). */
typedef struct asg_input {
    double poiss_rate, poiss_weight, gauss_noise_std, noise_dt;
    int32_t independent_noise;
} asg_input;

/* StpParams (parameters.hpp:65-70). */
typedef struct asg_stp {
    int32_t enabled;
    double U, tau_rec, tau_fac;
} asg_stp;

/* One ConnectionSet (network.hpp:14-27), CSR grouped by source, exactly as
 * Network::build_primary_connections leaves it (network.cpp:206-227).
 * weight/delay_steps are per edge but must be uniform within the set (the
 * reference assigns one value per set); STP arrays may be NULL (fresh
 * state x=1, u=U, t_last=-1e12) and must be identical along each row. */
typedef struct asg_csr {
    uint32_t n_sources;
    const uint32_t* row_start; /* n_sources + 1 */
    const uint32_t* target;    /* row_start[n_sources] */
    const double* weight;      /* may be NULL: uses the set weight below */
    const int32_t* delay_steps;/* may be NULL: uses the set delay below  */
    const double* stp_x;
    const double* stp_u;
    const double* stp_t_last;
} asg_csr;

/* Everything Network::run needs after build(): sizes, time grid, populations,
 * the four connection sets, per-cell parameters and the initial state.
 * All arrays are host memory and are copied by asg_create; NULL state arrays
 * take the reference's initial values (neuron.cpp:117-131, astrocyte.cpp:
 * 108-111 with V_m_init / Ca_init / IP3_init / h_init below). */
typedef struct asg_network_desc {
    uint32_t n_exc, n_inh, n_astro;
    double dt;
    int32_t substeps;
    uint64_t seed;
    int32_t sic_interval;
    int32_t d_e_steps, d_i_steps, d_a2n_steps; /* delay_to_steps of d_e, d_i, d_a2n */
    double w_e, w_i, w_n2a, w_a2n;              /* set weights */
    asg_neuron_params exc, inh;
    asg_astro_params astro;
    asg_input input_exc, input_inh, input_astro;
    asg_stp stp;
    asg_csr exc_primary, inh_primary, neuron_astro, astro_neuron;
    /* per-cell parameters */
    const double* V_reset; /* n_neurons */
    const double* b;       /* n_neurons */
    const double* Ca_tot;  /* n_astro; NULL = uniform value below */
    const double* IP3_0;
    const double* tau_IP3;
    const double* delta_IP3;
    double Ca_tot_u, IP3_0_u, tau_IP3_u, delta_IP3_u; /* used when the arrays are NULL */
    /* initial state (NULL = defaults) */
    double V_m_init_exc, V_m_init_inh, Ca_init, IP3_init, h_init;
    const double *V, *w, *g_ex, *dg_ex, *g_in, *dg_in, *I_sic;
    const int32_t* refractory;
    const double *Ca, *IP3, *h;
} asg_network_desc;

/* Recording, as Network::run does it (network.cpp:443-462): from
 * `record_from_step` on, spikes every step and every `record_every` steps the
 * first astro_max astrocytes' Ca, IP3 and the first neuron_max neurons'
 * V, I_sic. */
typedef struct asg_record_opts {
    int64_t record_from_step;
    int32_t record_every;
    int32_t spikes;
    uint32_t astro_max;
    uint32_t neuron_max;
} asg_record_opts;

/* Host-side copy of the dynamic state (pull/push). */
typedef struct asg_state {
    double *V, *w, *g_ex, *dg_ex, *g_in, *dg_in, *I_sic; /* n_neurons each */
    int32_t* refractory;                                 /* n_neurons */
    double *Ca, *IP3, *h;                                /* n_astro each */
} asg_state;

/* Engine options.  Zero-initialised fields take the defaults. */
typedef struct asg_engine_opts {
    int32_t device;         /* CUDA device ordinal (default 0)                    */
    int32_t chunk_steps;    /* steps per captured CUDA graph (default: asg_create
                               ~2^23 / neurons as a power of two in [32, 512];
                               batches and servers 32 and 64)                  */
    int32_t block;          /* threads per block of the step kernel (default 128)  */
    int32_t use_graphs;     /* 0/1 = a CUDA graph of per-step launches (default),
                               -1 = plain launches, 2 = persistent: one cooperative
                               launch per chunk, bounded grid barrier per step    */
    int32_t sic_mode;       /* 0 auto, 1 fused into the neuron role, 2 own role.
                               Auto fuses for a one-step SIC delay and, with
                               <= 160 SIC edges per target, for a network (or a
                               batch) of >= 2^16 neurons; otherwise side-stream
                               batches when the delay is >= 12 steps, else the
                               own role.                                        */
    int32_t pdl;            /* 0 = programmatic dependent launch (default), -1 off */
    int32_t push_mode;      /* 0 = spikes pushed one step later by load-balanced
                               push blocks when both spike delays are >= 2 steps
                               (default), 1 = pushed by the spiking block      */
    uint64_t mem_budget;    /* device bytes the engine may hold (0 = 90% free)     */
    int32_t occupancy;      /* step kernel form: 0 auto (by the number of blocks
                               a step launches), 1 latency form (fewest round
                               trips, 128 registers), 2 high-occupancy form
                               (6 blocks of 128 threads per SM; block 128 only).
                               Both forms give the same bits.                  */
    int32_t astro_precision;/* 0 or 64: FP64 (the product); 32: the astrocyte
                               update in FP32 -- the reference's precision
                               study (docs/experiments.md), opt-in, not
                               bitwise to anything                             */
} asg_engine_opts;

/* ------------------------------------------------------ single network
 * The plain path: one network, one handle.  Steps are numbered as in
 * Network::run (0 .. pre_steps+sim_steps-1); RNG streams are keyed by them. */
typedef struct asg_network asg_network;

int asg_create(const asg_network_desc* desc, const asg_record_opts* rec,
               const asg_engine_opts* opts, asg_network** out);
/* Advance n_steps from the handle's current step. */
int asg_step(asg_network* net, int64_t n_steps);
int asg_current_step(asg_network* net, int64_t* step);
/* Time launch shapes (chunk length, block size, graph vs persistent launch)
 * for `steps` steps on a snapshot of the network (restored after each trial:
 * the simulation does not advance) and keep the fastest; *chosen (may be NULL)
 * receives it.  The batched form has asg_batch_autotune. */
int asg_autotune(asg_network* net, int32_t steps, asg_engine_opts* chosen);
/* Spikes emitted since the last fetch, sorted by (step, source).  *count is
 * the number available; ASG_ERR_OVERFLOW (nothing consumed) if > cap. */
int asg_fetch_spikes(asg_network* net, int64_t* steps, uint32_t* sources, int64_t cap,
                     int64_t* count);
/* Recorded rows since the last fetch: astro rows of astro_max (Ca, IP3),
 * neuron rows of neuron_max (V, I_sic), with their step numbers. */
int asg_fetch_record(asg_network* net, int64_t* astro_steps, double* Ca, double* IP3,
                     int64_t astro_cap_rows, int64_t* astro_rows, int64_t* neuron_steps,
                     double* V, double* I_sic, int64_t neuron_cap_rows, int64_t* neuron_rows);
int asg_pull_state(asg_network* net, asg_state* out);
/* Per-source STP state (x, u, t_last) of every neuron (n_neurons each). */
int asg_pull_stp(asg_network* net, double* x, double* u, double* t_last);
/* Counters since creation: delivered spike edges, SIC edges summed, spikes. */
int asg_counters(asg_network* net, int64_t* spike_edges, int64_t* sic_edges, int64_t* spikes);
/* Device milliseconds of the last asg_step call (CUDA events on the handle's
 * stream) and the number of kernels it launched. */
int asg_last_timing(asg_network* net, double* device_ms, int64_t* kernels);
/* Snapshot and restore the complete device state (bitwise resume). */
int asg_checkpoint_size(asg_network* net, uint64_t* bytes);
int asg_checkpoint(asg_network* net, void* host_buf, uint64_t bytes);
int asg_restore(asg_network* net, const void* host_buf, uint64_t bytes);
int asg_destroy(asg_network* net);

/* ------------------------------------------------------ batched sweep
 * Many instances of uneven size packed into one device arena and advanced
 * together by one fused kernel per step, captured in CUDA graphs. */
typedef struct asg_batch asg_batch;

int asg_batch_create(int32_t n, const asg_network_desc* const* descs,
                     const asg_record_opts* rec, const asg_engine_opts* opts, asg_batch** out);
/* Advance every instance by n_steps. */
int asg_batch_step(asg_batch* b, int64_t n_steps);
int asg_batch_fetch_spikes(asg_batch* b, int32_t inst, int64_t* steps, uint32_t* sources,
                           int64_t cap, int64_t* count);
int asg_batch_fetch_record(asg_batch* b, int32_t inst, int64_t* astro_steps, double* Ca,
                           double* IP3, int64_t astro_cap_rows, int64_t* astro_rows,
                           int64_t* neuron_steps, double* V, double* I_sic,
                           int64_t neuron_cap_rows, int64_t* neuron_rows);
int asg_batch_pull_state(asg_batch* b, int32_t inst, asg_state* out);
int asg_batch_counters(asg_batch* b, int32_t inst, int64_t* spike_edges, int64_t* sic_edges,
                       int64_t* spikes);
int asg_batch_last_timing(asg_batch* b, double* device_ms, int64_t* kernels);
/* Time candidate launch shapes on a snapshot of the batch (state restored
 * afterwards) and keep the fastest.  `steps` per candidate.  Writes the
 * chosen block sizes / chunk / sic mode into *chosen (may be NULL). */
int asg_batch_autotune(asg_batch* b, int32_t steps, asg_engine_opts* chosen);
int asg_batch_destroy(asg_batch* b);

/* ------------------------------------------------------ serving
 * Continuous batching: requests of different sizes and durations are
 * admitted by device footprint, join the running batch at a step boundary,
 * and leave it when done.  A host thread drives the engine. */
typedef struct asg_server asg_server;

typedef struct asg_serve_opts {
    asg_engine_opts engine;
    uint64_t mem_budget;    /* device bytes for resident requests (0 = 80% free) */
    int32_t max_instances;  /* resident requests at most (default 256)          */
} asg_serve_opts;

typedef struct asg_request_result {
    int32_t status;         /* ASG_OK, ASG_ERR_CANCELLED, ...                   */
    int64_t n_spikes;
    int64_t spike_edges, sic_edges;
    double submit_to_admit_ms, submit_to_done_ms;
    double mean_rate_hz;
} asg_request_result;

int asg_serve_create(const asg_serve_opts* opts, asg_server** out);
/* The descriptor is copied.  n_steps = simulated steps from step 0.
 * Returns ASG_ERR_OOM at once when the request alone exceeds the budget. */
int asg_serve_submit(asg_server* s, const asg_network_desc* desc, int64_t n_steps,
                     int32_t keep_spikes, int64_t* request_id);
/* Non-blocking: ASG_OK with *done=1 and the result once finished. */
int asg_serve_poll(asg_server* s, int64_t request_id, int32_t* done, asg_request_result* res);
/* Blocks until the request finished (timeout_ms < 0: no limit). */
int asg_serve_wait(asg_server* s, int64_t request_id, double timeout_ms,
                   asg_request_result* res);
int asg_serve_fetch_spikes(asg_server* s, int64_t request_id, int64_t* steps,
                           uint32_t* sources, int64_t cap, int64_t* count);
int asg_serve_cancel(asg_server* s, int64_t request_id);
/* Aggregate: steps run, kernels, device ms, resident requests (now / peak). */
int asg_serve_stats(asg_server* s, int64_t* chunks, int64_t* kernels, double* device_ms,
                    int32_t* resident, int32_t* peak_resident);
int asg_serve_destroy(asg_server* s);

/* -------------------------------------- astrocyte backend (drop-in)
 * Same four movement points as the reference's native CUDA backend
 * (astrocyte_cuda.hpp:15-27): create with resident state, push the step's
 * input, update, pull calcium, destroy with the state copied back.
 * As in the reference, an update consumes the pushed input: an update with
 * no push since the previous one sees zero input.  Per-cell parameter
 * arrays whose entries are all equal are held as scalars. */
typedef struct asg_astro asg_astro;

int asg_astro_create(uint32_t n, const double* Ca, const double* IP3, const double* h,
                     const double* Ca_tot, const double* IP3_0, const double* tau_IP3,
                     const double* delta_IP3, asg_astro** out);
int asg_astro_destroy(asg_astro* s, double* Ca, double* IP3, double* h);
int asg_astro_push_input(asg_astro* s, const double* ip3_input);
int asg_astro_pull_calcium(asg_astro* s, double* Ca);
/* consts: Kd_IP3_1, Kd_IP3_2, Kd_act, Kd_inh, Km_SERCA, k_IP3R, rate_IP3R,
 * rate_L, rate_SERCA, ratio_ER_cyt (AstroConstants order). */
int asg_astro_update(asg_astro* s, const double* consts, double h_step, int32_t substeps,
                     double noise_std, int32_t independent_noise, double shared_noise,
                     uint64_t noise_seed, uint64_t noise_index);
/* The astrocyte kernel-scaling workload: steps [first, first+count) with the
 * input generated on the device: an event of `weight` whenever
 * rng_uniform(seed, cell, 1000+step) < p (rng.hpp:36-39), noise off.
 * Uniform parameters are taken from the scalars; per-cell arrays given at
 * create are used when uniform == 0. */
int asg_astro_run_bernoulli(asg_astro* s, const double* consts, double h_step, int32_t substeps,
                            uint64_t seed, double p, double weight, int64_t first, int64_t count,
                            int32_t uniform, double Ca_tot, double IP3_0, double tau_IP3,
                            double delta_IP3);
/* Precision study (the reference's docs/experiments.md, "Single or double
 * precision": is FP32 enough for the Li-Rinzel dynamics?).  The same
 * workload with uniform parameters, the state rounded to float on entry (or
 * kept in float from the previous call of this entry point) and advanced in
 * FP32 arithmetic; the handle's FP64 state receives the widened result.
 * Device time of the steps alone in asg_astro_last_timing.  No counterpart
 * in the reference's GPU backend (the reference runs the study by rebuilding
 * with `real = float`); not bitwise to anything. */
int asg_astro_run_bernoulli_f32(asg_astro* s, const double* consts, double h_step,
                                int32_t substeps, uint64_t seed, double p, double weight,
                                int64_t first, int64_t count, double Ca_tot, double IP3_0,
                                double tau_IP3, double delta_IP3);
/* Read the state without destroying the handle. */
int asg_astro_pull_state(asg_astro* s, double* Ca, double* IP3, double* h);
/* Time the kernel's launch shapes (cells per thread, block size, register
 * budget) for `steps` steps of the Bernoulli workload on a scratch copy of
 * the state, keep the fastest for this handle (state unchanged) and return
 * its index and per-step microseconds (may be NULL). */
int asg_astro_autotune(asg_astro* s, const double* consts, double h_step, int32_t substeps,
                       int32_t steps, int32_t* chosen, double* us_per_step);
/* Use launch shape `shape` (an index asg_astro_autotune may return) for this
 * handle; ASG_ERR_ARG names the valid range.  Every shape gives the same
 * bits.  No counterpart in the reference (a tuning knob, like autotune). */
int asg_astro_set_shape(asg_astro* s, int32_t shape);
/* Device ms and kernels launched of the last asg_astro_run_bernoulli call,
 * or of all asg_astro_update calls since the previous timing read (waits for
 * them to finish). */
int asg_astro_last_timing(asg_astro* s, double* device_ms, int64_t* kernels);

/* Allocation-free astrocyte update.  No counterpart in the reference: it
 * exists for callers that cannot call cudaMalloc -- e.g. an OpenMP
 * target-offload build whose device arrays belong to the OpenMP runtime, or a
 * framework whose memory pool owns all device memory.  All array arguments
 * are DEVICE pointers owned by the caller (8-byte aligned) and are updated in
 * place exactly like asg_astro_update updates its resident copies (ip3_input
 * is consumed and zeroed).  `stream` is a cudaStream_t (NULL: the default
 * stream); the call is asynchronous on it.  The only scratch, one double per
 * cell, lives in a static device array of at most 1,048,576 cells: larger n
 * is rejected with ASG_ERR_ARG.  The call allocates nothing itself.  The
 * 8 MiB array is reserved together with the library's device code when CUDA
 * loads that module: at context creation under eager module loading, or, under
 * CUDA's default lazy loading, during the first call on a device; if device
 * memory is already exhausted then, that call returns ASG_ERR_OOM.  The first
 * call on a device (and the first after that device's context was re-created,
 * e.g. by cudaDeviceReset) looks up the array's device address, so make it
 * before any stream capture.  The call refuses to launch (ASG_ERR_CUDA) while
 * an earlier CUDA error is pending on the calling thread.  Every call shares
 * the array: calls that overlap on the GPU race and must be ordered by the
 * caller. */
int asg_astro_update_noalloc(uint32_t n, double* Ca, double* IP3, double* h, double* ip3_input,
                             const double* Ca_tot, const double* IP3_0, const double* tau_IP3,
                             const double* delta_IP3, const double* consts, double h_step,
                             int32_t substeps, double noise_std, int32_t independent_noise,
                             double shared_noise, uint64_t noise_seed, uint64_t noise_index,
                             void* stream);

/* Failure-detection self-test of the bounded device waits: launches a grid in
 * which one block never reaches the grid barrier; the others must give up
 * within about a second, set the error word and return.  *timed_out = 1 when
 * they did; *wait_ms is the launch's device time.  The context stays usable. */
int asg_selftest_barrier_timeout(int32_t* timed_out, double* wait_ms);

/* ------------------------------------------ host side: config + builder
 * The reference's JSON schema (parameters.cpp:85-205): '//' comments, key
 * aliases (V_m, IP3, gauss_noise_var), noise_dt default 10*dt, validation,
 * and unknown keys rejected.  The builder reproduces Network::build
 * (network.cpp:56-228, astrocyte.cpp:28-53, neuron.cpp:23-75) bit for bit. */
typedef struct asg_model asg_model;

/* Parse JSON text.  Overrides < 0 keep the file's value (main.cpp:216-233). */
int asg_model_from_json(const char* json_text, int64_t seed, double sim_time, double pre_time,
                        int64_t n_astro, asg_model** out);
int asg_model_from_file(const char* path, int64_t seed, double sim_time, double pre_time,
                        int64_t n_astro, asg_model** out);
/* Build connectivity and per-cell parameters (deterministic for the seed). */
int asg_model_build(asg_model* m);
/* Replace the reference builder by the counter-based fixed-in-degree
 * generator (in-degree k_in per neuron; each excitatory synapse recruits an
 * astrocyte of the target's pool with p_third_if_primary), built on the
 * device (device >= 0) or on the host (device < 0); both give identical
 * tables. */
int asg_model_build_fixed_indegree(asg_model* m, uint32_t k_in, int32_t device);
/* Descriptor view of the built model (valid while the model lives). */
int asg_model_desc(asg_model* m, asg_network_desc* out);
int asg_model_record_opts(asg_model* m, asg_record_opts* out);
/* Resolved scalars: dt, substeps, seed, pre_steps, sim_steps, record_every,
 * pre_sim_time, sim_time, analysis threshold, merge_gap, hist_window,
 * hist_shift (12 doubles). */
int asg_model_scalars(asg_model* m, double* out12);
/* Edge counts: n_primary_exc, n_primary_inh, n_n2a, n_a2n, ring_slots. */
int asg_model_stats(asg_model* m, int64_t* out5);
int asg_model_free(asg_model* m);

/* Calcium analysis of recorded traces (analysis.cpp:10-166 semantics):
 * n_cells traces of n_samples (times row-major like ca).  out: active cells,
 * transients, mean duration, pairs correlated, mean pairwise correlation. */
int asg_calcium_analysis(const double* times, const double* ca, int32_t n_cells,
                         int32_t n_samples, double threshold, double merge_gap, double win_start,
                         double win_end, double width, double shift, double* out5);

#ifdef __cplusplus
}
#endif

#endif /* ASG_B200_H */
