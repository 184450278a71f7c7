/*
 * asg_oracle.h -- CPU restatement of the astrosimgpu per-timestep algorithm,
 * in plain C, used ONLY as a checker by tests/ (and as the "port" CPU
 * baseline).  It is test infrastructure: the product never links it.
 *
 * Each function cites the reference file:line it restates.  The restatement
 * is pinned against the reference itself (oracle/_ref, compiled from the
 * reference sources) by tests/test_oracle_pin.py: RNG streams, astro_advance,
 * builder tables and full network steps must agree bit for bit.
 */
#ifndef ASG_ORACLE_H
#define ASG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* rng.hpp:26-33 */
uint64_t orc_bits(uint64_t seed, uint64_t stream, uint64_t counter);
/* rng.hpp:36-39 */
double orc_uniform(uint64_t seed, uint64_t stream, uint64_t counter);
/* rng.hpp:42-50 */
double orc_normal(uint64_t seed, uint64_t stream);

/* CounterRng (rng.hpp:53-143). */
typedef struct orc_rng {
    uint64_t seed, stream, counter;
    int has_spare;
    double spare;
} orc_rng;
void orc_rng_init(orc_rng* r, uint64_t seed, uint64_t stream);
double orc_rng_uniform(orc_rng* r);
double orc_rng_normal(orc_rng* r);
double orc_rng_normal_redraw(orc_rng* r, double mean, double sd, double lo, double hi);
int orc_rng_poisson(orc_rng* r, double lambda);

/* astro_advance (astrocyte_kernel.hpp:71-103).  c: AstroConstants order. */
void orc_astro_advance(const double* c, double Ca_tot, double IP3_0, double tau, double delta,
                       double input, double noise, double h_step, int substeps, double* Ca,
                       double* IP3, double* h);

/* The astrocyte kernel-scaling workload (see ScalingWorkload): N cells,
 * uniform params, input weight when orc_uniform(seed, cell, 1000+step) < p,
 * steps [first, first+count).  Serial. */
void orc_astro_scaling(const double* c, double Ca_tot, double IP3_0, double tau, double delta,
                       double h_step, int substeps, uint64_t seed, double p, double weight,
                       int64_t first, int64_t count, int64_t n, double* Ca, double* IP3,
                       double* h);

/* ---------------------------------------------------------- network ----
 * A whole network in the reference's data structures (dense [slot][cell]
 * rings, per-edge STP), built by the restated builder and stepped by the
 * restated phases.  Config values are passed as a flat array of doubles in
 * the order of ORC_CFG_* below. */
enum {
    ORC_N_A, ORC_N_E, ORC_N_I, ORC_DT, ORC_SUBSTEPS, ORC_SEED,
    /* astrocyte (parameters.hpp:14-40) */
    ORC_A_CA_TOT, ORC_A_IP3_0, ORC_A_KD1, ORC_A_KD2, ORC_A_KDACT, ORC_A_KDINH, ORC_A_KM,
    ORC_A_SIC_SCALE, ORC_A_SIC_TH, ORC_A_DELTA, ORC_A_KIP3R, ORC_A_RIP3R, ORC_A_RL,
    ORC_A_RSERCA, ORC_A_RATIO, ORC_A_TAU, ORC_A_CA_INIT, ORC_A_H_INIT, ORC_A_IP3_INIT,
    /* neuron exc (17) then inh (17): C_m g_L E_L V_th Delta_T a b tau_w V_reset V_peak
     * t_ref E_ex E_in tau_syn_ex tau_syn_in I_e V_m_init */
    ORC_NE0, ORC_NI0 = ORC_NE0 + 17,
    /* synapse */
    ORC_W_E = ORC_NI0 + 17, ORC_W_I, ORC_W_N2A, ORC_W_A2N, ORC_D_E, ORC_D_I, ORC_D_A2N,
    ORC_SIC_INTERVAL, ORC_STP_ON, ORC_STP_U, ORC_STP_TREC, ORC_STP_TFAC,
    /* connectivity */
    ORC_P_PRIMARY, ORC_P_THIRD, ORC_POOL_SIZE, ORC_POOL_RANDOM, ORC_AUTAPSES, ORC_UNIQUE3,
    /* inputs astro, exc, inh: rate weight std noise_dt independent */
    ORC_IN_A, ORC_IN_E = ORC_IN_A + 5, ORC_IN_I = ORC_IN_E + 5,
    /* randomize astro, neuron: enabled lower upper var */
    ORC_RND_A = ORC_IN_I + 5, ORC_RND_N = ORC_RND_A + 4,
    ORC_CFG_SIZE = ORC_RND_N + 4
};

typedef struct orc_net orc_net;

orc_net* orc_net_build(const double* cfg);
void orc_net_free(orc_net* n);
/* Edge count of set which (0 exc, 1 inh, 2 n2a, 3 a2n) and CSR copy-out. */
int64_t orc_net_table_size(const orc_net* n, int which);
void orc_net_table(const orc_net* n, int which, uint32_t* row_start, uint32_t* target);
void orc_net_cells(const orc_net* n, double* V_reset, double* b, double* Ca_tot, double* IP3_0,
                   double* tau_IP3, double* delta_IP3);
/* One step of Network::run's body (network.cpp:385-431); returns the number
 * of spikes, their sources (sorted) into `spikes` up to cap. */
int orc_net_step(orc_net* n, int64_t step, uint32_t* spikes, int cap);
/* Neuron state 7 x N (V w g_ex dg_ex g_in dg_in I_sic), refractory, astro 3 x NA. */
void orc_net_state(const orc_net* n, double* neuron7, int32_t* refractory, double* astro3);

#ifdef __cplusplus
}
#endif

#endif
