/*
 * asg_oracle.c -- CPU restatement of the astrosimgpu per-timestep algorithm
 * (TEST INFRASTRUCTURE ONLY; see asg_oracle.h).  Plain C, serial, FP64,
 * written from the model's equations and the reference's documented
 * behaviour; pinned bit for bit against the reference build by
 * tests/test_oracle_pin.py.
 */
#include "asg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- RNG */

uint64_t orc_bits(uint64_t seed, uint64_t stream, uint64_t counter) {
    /* rng.hpp:26-33: splitmix64 finaliser of seed + stream*phi + counter*A */
    uint64_t z = seed + stream * 0x9E3779B97F4A7C15ULL + counter * 0xBF58476D1CE4E5B9ULL;
    z ^= z >> 30;
    z *= 0xBF58476D1CE4E5B9ULL;
    z ^= z >> 27;
    z *= 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

double orc_uniform(uint64_t seed, uint64_t stream, uint64_t counter) {
    /* rng.hpp:36-39 */
    return (double)(orc_bits(seed, stream, counter) >> 11) * (1.0 / 9007199254740992.0);
}

static const double TWO_PI = 6.283185307179586476925286766559;

double orc_normal(uint64_t seed, uint64_t stream) {
    /* rng.hpp:42-50 */
    double u1 = orc_uniform(seed, stream, 0);
    if (u1 <= 1e-300) u1 = 1e-300;
    double u2 = orc_uniform(seed, stream, 1);
    return sqrt(-2.0 * log(u1)) * cos(TWO_PI * u2);
}

void orc_rng_init(orc_rng* r, uint64_t seed, uint64_t stream) {
    r->seed = seed;
    r->stream = stream;
    r->counter = 0;
    r->has_spare = 0;
    r->spare = 0.0;
}

double orc_rng_uniform(orc_rng* r) { return orc_uniform(r->seed, r->stream, r->counter++); }

double orc_rng_normal(orc_rng* r) {
    /* rng.hpp:74-89: Box-Muller, the sine branch kept for the next call */
    if (r->has_spare) {
        r->has_spare = 0;
        return r->spare;
    }
    double u1;
    do {
        u1 = orc_rng_uniform(r);
    } while (u1 <= 1e-300);
    double u2 = orc_rng_uniform(r);
    double rad = sqrt(-2.0 * log(u1));
    double th = TWO_PI * u2;
    r->spare = rad * sin(th);
    r->has_spare = 1;
    return rad * cos(th);
}

double orc_rng_normal_redraw(orc_rng* r, double mean, double sd, double lo, double hi) {
    /* rng.hpp:94-103 (max_tries 1000) */
    for (int i = 0; i < 1000; ++i) {
        double v = mean + sd * orc_rng_normal(r);
        if (v >= lo && v <= hi) return v;
    }
    double m = mean < lo ? lo : mean;
    return hi < m ? hi : m;
}

int orc_rng_poisson(orc_rng* r, double lambda) {
    /* rng.hpp:107-124 */
    if (lambda <= 0.0) return 0;
    if (lambda > 30.0) {
        double v = lambda + sqrt(lambda) * orc_rng_normal(r);
        return v < 0.0 ? 0 : (int)(v + 0.5);
    }
    double limit = exp(-lambda);
    double prod = orc_rng_uniform(r);
    int k = 0;
    while (prod > limit) {
        ++k;
        prod *= orc_rng_uniform(r);
    }
    return k;
}

/* ------------------------------------------------------------ astrocyte */

/* c: Kd_IP3_1 Kd_IP3_2 Kd_act Kd_inh Km_SERCA k_IP3R rate_IP3R rate_L rate_SERCA ratio */
static void astro_rhs(const double* c, double Ca_tot, double IP3_0, double tau, double Ca,
                      double IP3, double h, double noise, double* dCa, double* dIP3, double* dh) {
    /* astrocyte_kernel.hpp:47-68 */
    double er = (Ca_tot - Ca) / c[9];
    double m = IP3 / (IP3 + c[0]);
    double n = Ca / (Ca + c[2]);
    double m3 = m * m * m, n3 = n * n * n, h3 = h * h * h;
    double jc = c[9] * c[6] * m3 * n3 * h3 * (er - Ca);
    double jp = c[8] * Ca * Ca / (c[4] * c[4] + Ca * Ca);
    double jl = c[9] * c[7] * (er - Ca);
    double ah = c[5] * c[3] * (IP3 + c[0]) / (IP3 + c[1]);
    double bh = c[5] * Ca;
    *dCa = jc - jp + jl + noise;
    *dIP3 = (IP3_0 - IP3) / tau;
    *dh = ah * (1.0 - h) - bh * h;
}

void orc_astro_advance(const double* c, double Ca_tot, double IP3_0, double tau, double delta,
                       double input, double noise, double hs, int substeps, double* Ca,
                       double* IP3, double* h) {
    /* astrocyte_kernel.hpp:71-103 */
    if (input != 0.0) *IP3 += delta * input;
    for (int s = 0; s < substeps; ++s) {
        double a1, b1, c1, a2, b2, c2, a3, b3, c3, a4, b4, c4;
        astro_rhs(c, Ca_tot, IP3_0, tau, *Ca, *IP3, *h, noise, &a1, &b1, &c1);
        astro_rhs(c, Ca_tot, IP3_0, tau, *Ca + 0.5 * hs * a1, *IP3 + 0.5 * hs * b1,
                  *h + 0.5 * hs * c1, noise, &a2, &b2, &c2);
        astro_rhs(c, Ca_tot, IP3_0, tau, *Ca + 0.5 * hs * a2, *IP3 + 0.5 * hs * b2,
                  *h + 0.5 * hs * c2, noise, &a3, &b3, &c3);
        astro_rhs(c, Ca_tot, IP3_0, tau, *Ca + hs * a3, *IP3 + hs * b3, *h + hs * c3, noise, &a4,
                  &b4, &c4);
        *Ca += (hs / 6.0) * (a1 + 2.0 * a2 + 2.0 * a3 + a4);
        *IP3 += (hs / 6.0) * (b1 + 2.0 * b2 + 2.0 * b3 + b4);
        *h += (hs / 6.0) * (c1 + 2.0 * c2 + 2.0 * c3 + c4);
        *Ca = *Ca < 0.0 ? 0.0 : (*Ca > Ca_tot ? Ca_tot : *Ca);
        *h = *h < 0.0 ? 0.0 : (*h > 1.0 ? 1.0 : *h);
        *IP3 = *IP3 < 0.0 ? 0.0 : *IP3;
    }
}

void orc_astro_scaling(const double* c, double Ca_tot, double IP3_0, double tau, double delta,
                       double hs, int substeps, uint64_t seed, double p, double weight,
                       int64_t first, int64_t count, int64_t n, double* Ca, double* IP3,
                       double* h) {
    for (int64_t s = first; s < first + count; ++s) {
        for (int64_t i = 0; i < n; ++i) {
            double in = orc_uniform(seed, (uint64_t)i, 1000u + (uint64_t)s) < p ? weight : 0.0;
            orc_astro_advance(c, Ca_tot, IP3_0, tau, delta, in, 0.0, hs, substeps, Ca + i,
                              IP3 + i, h + i);
        }
    }
}

/* -------------------------------------------------------------- network */

typedef struct {
    uint32_t* rs; /* row_start */
    uint32_t* tg; /* target */
    int64_t m;
    uint32_t rows;
    double w;
    int delay;
    double *x, *u, *t; /* per-edge STP (NULL when disabled) */
} orc_set;

typedef struct {
    double C_m, g_L, E_L, V_th, Delta_T, a, b, tau_w, V_reset, V_peak, t_ref, E_ex, E_in,
        tau_syn_ex, tau_syn_in, I_e, V_m_init;
} orc_pop;

typedef struct {
    double rate, weight, std, noise_dt;
    int indep;
} orc_input;

struct orc_net {
    uint32_t NA, NE, NI, N;
    double dt;
    int substeps;
    uint64_t seed;
    double ac[10]; /* AstroConstants */
    double SIC_scale, SIC_th;
    orc_pop pe, pi;
    orc_input in_a, in_e, in_i;
    int stp_on;
    double U, tau_rec, tau_fac;
    int sic_interval;
    orc_set set[4];
    int slots, sic_delay;
    /* cells */
    double *V_reset, *b;
    double *V, *w, *gex, *dgex, *gin, *dgin, *Isic, *exc_in, *inh_in;
    int* refr;
    double *Ca, *IP3, *h, *Ca_tot, *IP3_0, *tau, *delta, *ip3_in;
    /* rings [slot][cell] */
    double *r_ex, *r_in, *r_sic, *r_astro;
    char* pending;
    uint32_t *sic_src, *sinks;
    uint32_t n_sic_src, n_sinks;
};

static int delay_steps(double ms, double dt) {
    /* network.cpp:32-35 */
    int s = (int)(ms / dt + 0.5);
    return s < 1 ? 1 : s;
}

static double draw_scaled(double mean, const double* rnd, orc_rng* r) {
    /* astrocyte.cpp:8-15 / neuron.cpp:14-21 */
    if (!(rnd[0] != 0.0) || rnd[3] <= 0.0) return mean;
    double lo = mean < 0.0 ? mean * rnd[2] : mean * rnd[1];
    double hi = mean < 0.0 ? mean * rnd[1] : mean * rnd[2];
    return orc_rng_normal_redraw(r, mean, rnd[3] * fabs(mean), lo, hi);
}

/* growable u32 list */
typedef struct {
    uint32_t* v;
    uint32_t n, cap;
} u32v;

static void push(u32v* l, uint32_t x) {
    if (l->n == l->cap) {
        l->cap = l->cap ? 2 * l->cap : 8;
        l->v = (uint32_t*)realloc(l->v, (size_t)l->cap * 4);
    }
    l->v[l->n++] = x;
}

static void flatten(u32v* rows, uint32_t nrows, orc_set* s) {
    /* network.cpp:16-30 */
    s->rows = nrows;
    s->rs = (uint32_t*)calloc((size_t)nrows + 1, 4);
    int64_t tot = 0;
    for (uint32_t r = 0; r < nrows; ++r) {
        s->rs[r] = (uint32_t)tot;
        tot += rows[r].n;
    }
    s->rs[nrows] = (uint32_t)tot;
    s->m = tot;
    s->tg = (uint32_t*)malloc((size_t)(tot ? tot : 1) * 4);
    for (uint32_t r = 0; r < nrows; ++r) {
        if (rows[r].n) memcpy(s->tg + s->rs[r], rows[r].v, (size_t)rows[r].n * 4);
        free(rows[r].v);
    }
}

/* open-addressing set of 64-bit keys (unique_third_out) */
typedef struct {
    uint64_t* k;
    size_t cap, n;
} kset;

static int kset_insert(kset* s, uint64_t key) {
    if (2 * (s->n + 1) > s->cap) {
        size_t nc = s->cap ? 2 * s->cap : 1024;
        uint64_t* nk = (uint64_t*)malloc(nc * 8);
        for (size_t i = 0; i < nc; ++i) nk[i] = ~0ULL;
        for (size_t i = 0; i < s->cap; ++i) {
            if (s->k[i] == ~0ULL) continue;
            size_t j = (size_t)(orc_bits(s->k[i], 0, 0) & (nc - 1));
            while (nk[j] != ~0ULL) j = (j + 1) & (nc - 1);
            nk[j] = s->k[i];
        }
        free(s->k);
        s->k = nk;
        s->cap = nc;
    }
    size_t j = (size_t)(orc_bits(key, 0, 0) & (s->cap - 1));
    while (s->k[j] != ~0ULL) {
        if (s->k[j] == key) return 0;
        j = (j + 1) & (s->cap - 1);
    }
    s->k[j] = key;
    s->n++;
    return 1;
}

static void load_pop(orc_pop* p, const double* c) {
    p->C_m = c[0]; p->g_L = c[1]; p->E_L = c[2]; p->V_th = c[3]; p->Delta_T = c[4];
    p->a = c[5]; p->b = c[6]; p->tau_w = c[7]; p->V_reset = c[8]; p->V_peak = c[9];
    p->t_ref = c[10]; p->E_ex = c[11]; p->E_in = c[12]; p->tau_syn_ex = c[13];
    p->tau_syn_in = c[14]; p->I_e = c[15]; p->V_m_init = c[16];
}

static void load_input(orc_input* in, const double* c) {
    in->rate = c[0]; in->weight = c[1]; in->std = c[2]; in->noise_dt = c[3];
    in->indep = c[4] != 0.0;
}

static void finalise(orc_set* s, int stp_on, double U) {
    /* network.cpp:43-52 */
    if (!stp_on) return;
    size_t m = (size_t)(s->m ? s->m : 1);
    s->x = (double*)malloc(m * 8);
    s->u = (double*)malloc(m * 8);
    s->t = (double*)malloc(m * 8);
    for (int64_t k = 0; k < s->m; ++k) {
        s->x[k] = 1.0;
        s->u[k] = U;
        s->t[k] = -1e12;
    }
}

orc_net* orc_net_build(const double* cfg) {
    orc_net* n = (orc_net*)calloc(1, sizeof(orc_net));
    n->NA = (uint32_t)cfg[ORC_N_A];
    n->NE = (uint32_t)cfg[ORC_N_E];
    n->NI = (uint32_t)cfg[ORC_N_I];
    n->N = n->NE + n->NI;
    n->dt = cfg[ORC_DT];
    n->substeps = (int)cfg[ORC_SUBSTEPS];
    n->seed = (uint64_t)cfg[ORC_SEED];
    n->ac[0] = cfg[ORC_A_KD1]; n->ac[1] = cfg[ORC_A_KD2]; n->ac[2] = cfg[ORC_A_KDACT];
    n->ac[3] = cfg[ORC_A_KDINH]; n->ac[4] = cfg[ORC_A_KM]; n->ac[5] = cfg[ORC_A_KIP3R];
    n->ac[6] = cfg[ORC_A_RIP3R]; n->ac[7] = cfg[ORC_A_RL]; n->ac[8] = cfg[ORC_A_RSERCA];
    n->ac[9] = cfg[ORC_A_RATIO];
    n->SIC_scale = cfg[ORC_A_SIC_SCALE];
    n->SIC_th = cfg[ORC_A_SIC_TH];
    load_pop(&n->pe, cfg + ORC_NE0);
    load_pop(&n->pi, cfg + ORC_NI0);
    load_input(&n->in_a, cfg + ORC_IN_A);
    load_input(&n->in_e, cfg + ORC_IN_E);
    load_input(&n->in_i, cfg + ORC_IN_I);
    n->stp_on = cfg[ORC_STP_ON] != 0.0;
    n->U = cfg[ORC_STP_U];
    n->tau_rec = cfg[ORC_STP_TREC];
    n->tau_fac = cfg[ORC_STP_TFAC];
    n->sic_interval = (int)cfg[ORC_SIC_INTERVAL];

    orc_rng rng;
    orc_rng_init(&rng, n->seed, 0x5EED); /* network.cpp:57 */
    const uint32_t NA = n->NA, NE = n->NE, NI = n->NI, N = n->N;
    const size_t na = NA ? NA : 1, nn = N ? N : 1;

    /* astrocytes (astrocyte.cpp:28-53) */
    n->Ca = (double*)malloc(na * 8); n->IP3 = (double*)malloc(na * 8);
    n->h = (double*)malloc(na * 8); n->ip3_in = (double*)calloc(na, 8);
    n->Ca_tot = (double*)malloc(na * 8); n->IP3_0 = (double*)malloc(na * 8);
    n->tau = (double*)malloc(na * 8); n->delta = (double*)malloc(na * 8);
    const double* ra = cfg + ORC_RND_A;
    for (uint32_t i = 0; i < NA; ++i) {
        n->Ca[i] = cfg[ORC_A_CA_INIT];
        n->h[i] = cfg[ORC_A_H_INIT];
        n->Ca_tot[i] = draw_scaled(cfg[ORC_A_CA_TOT], ra, &rng);
        n->IP3_0[i] = draw_scaled(cfg[ORC_A_IP3_0], ra, &rng);
        n->tau[i] = draw_scaled(cfg[ORC_A_TAU], ra, &rng);
        n->delta[i] = draw_scaled(cfg[ORC_A_DELTA], ra, &rng);
        n->IP3[i] = cfg[ORC_A_IP3_INIT];
    }
    /* neurons (neuron.cpp:23-75) */
    n->V_reset = (double*)malloc(nn * 8); n->b = (double*)malloc(nn * 8);
    n->V = (double*)malloc(nn * 8); n->w = (double*)calloc(nn, 8);
    n->gex = (double*)calloc(nn, 8); n->dgex = (double*)calloc(nn, 8);
    n->gin = (double*)calloc(nn, 8); n->dgin = (double*)calloc(nn, 8);
    n->Isic = (double*)calloc(nn, 8); n->exc_in = (double*)calloc(nn, 8);
    n->inh_in = (double*)calloc(nn, 8); n->refr = (int*)calloc(nn, sizeof(int));
    const double* rn = cfg + ORC_RND_N;
    for (uint32_t i = 0; i < N; ++i) {
        const orc_pop* p = i < NE ? &n->pe : &n->pi;
        n->V_reset[i] = draw_scaled(p->V_reset, rn, &rng);
        n->b[i] = draw_scaled(p->b, rn, &rng);
        n->V[i] = p->V_m_init;
    }

    /* connectivity (network.cpp:110-228) */
    const double pp = cfg[ORC_P_PRIMARY], p3 = cfg[ORC_P_THIRD];
    const int pool_size = (int)cfg[ORC_POOL_SIZE];
    const int random_pool = cfg[ORC_POOL_RANDOM] != 0.0;
    const int autapses = cfg[ORC_AUTAPSES] != 0.0;
    const int unique3 = cfg[ORC_UNIQUE3] != 0.0;
    u32v* pool = (u32v*)calloc(nn, sizeof(u32v));
    uint32_t* cand = (uint32_t*)malloc(na * 4);
    for (int blk = 0; blk < 2; ++blk) {
        uint32_t off = blk ? NE : 0, cnt = blk ? NI : NE;
        for (uint32_t l = 0; l < cnt; ++l) {
            uint32_t post = off + l;
            if (!random_pool) {
                uint32_t start =
                    NA == 0 ? 0 : (uint32_t)(((uint64_t)l * NA) / (uint64_t)(cnt ? cnt : 1));
                for (int k = 0; k < pool_size; ++k) push(&pool[post], (start + (uint32_t)k) % NA);
            } else {
                for (uint32_t i = 0; i < NA; ++i) cand[i] = i;
                int take = pool_size < (int)NA ? pool_size : (int)NA;
                for (int k = 0; k < take; ++k) {
                    size_t pick = (size_t)(orc_rng_uniform(&rng) * (double)(NA - (uint32_t)k)) +
                                  (size_t)k;
                    size_t j = pick < (size_t)NA - 1 ? pick : (size_t)NA - 1;
                    uint32_t t = cand[k];
                    cand[k] = cand[j];
                    cand[j] = t;
                    push(&pool[post], cand[k]);
                }
            }
        }
    }
    u32v* exc_t = (u32v*)calloc(NE ? NE : 1, sizeof(u32v));
    u32v* ast_t = (u32v*)calloc(NE ? NE : 1, sizeof(u32v));
    u32v* a2n_t = (u32v*)calloc(na, sizeof(u32v));
    u32v* inh_t = (u32v*)calloc(NI ? NI : 1, sizeof(u32v));
    kset seen = {0, 0, 0};
    for (int blk = 0; blk < 2; ++blk) {
        uint32_t off = blk ? NE : 0, cnt = blk ? NI : NE;
        for (uint32_t pre = 0; pre < NE; ++pre) {
            for (uint32_t l = 0; l < cnt; ++l) {
                uint32_t post = off + l;
                if (!autapses && pre == post) continue;
                if (orc_rng_uniform(&rng) >= pp) continue;
                push(&exc_t[pre], post);
                if (NA == 0 || orc_rng_uniform(&rng) >= p3) continue;
                const u32v* pl = &pool[post];
                uint32_t a = pl->v[(size_t)(orc_rng_uniform(&rng) * (double)pl->n) % pl->n];
                push(&ast_t[pre], a);
                if (!unique3 || kset_insert(&seen, ((uint64_t)a << 32) | post)) push(&a2n_t[a], post);
            }
        }
    }
    for (uint32_t pre = 0; pre < NI; ++pre) {
        uint32_t pg = NE + pre;
        for (uint32_t post = 0; post < N; ++post) {
            if (!autapses && pg == post) continue;
            if (orc_rng_uniform(&rng) < pp) push(&inh_t[pre], post);
        }
    }
    for (uint32_t i = 0; i < N; ++i) free(pool[i].v);
    free(pool);
    free(cand);
    free(seen.k);
    flatten(exc_t, NE, &n->set[0]);
    flatten(inh_t, NI, &n->set[1]);
    flatten(ast_t, NE, &n->set[2]);
    flatten(a2n_t, NA, &n->set[3]);
    free(exc_t); free(inh_t); free(ast_t); free(a2n_t);
    const double de = cfg[ORC_D_E], di = cfg[ORC_D_I], da = cfg[ORC_D_A2N];
    n->set[0].w = cfg[ORC_W_E]; n->set[0].delay = delay_steps(de, n->dt);
    n->set[1].w = cfg[ORC_W_I]; n->set[1].delay = delay_steps(di, n->dt);
    n->set[2].w = cfg[ORC_W_N2A]; n->set[2].delay = delay_steps(de, n->dt);
    n->set[3].w = cfg[ORC_W_A2N]; n->set[3].delay = delay_steps(da, n->dt);
    for (int s = 0; s < 3; ++s) finalise(&n->set[s], n->stp_on, n->U);

    /* rings (network.cpp:73-107) */
    int md = 1;
    if (delay_steps(de, n->dt) > md) md = delay_steps(de, n->dt);
    if (delay_steps(di, n->dt) > md) md = delay_steps(di, n->dt);
    if (delay_steps(da, n->dt) > md) md = delay_steps(da, n->dt);
    n->slots = md + 1;
    n->sic_delay = delay_steps(da, n->dt);
    n->sic_src = (uint32_t*)malloc(na * 4);
    for (uint32_t a = 0; a < NA; ++a)
        if (n->set[3].rs[a] < n->set[3].rs[a + 1]) n->sic_src[n->n_sic_src++] = a;
    char* seen_a = (char*)calloc(na, 1);
    n->sinks = (uint32_t*)malloc(na * 4);
    for (int64_t k = 0; k < n->set[2].m; ++k) seen_a[n->set[2].tg[k]] = 1;
    for (uint32_t a = 0; a < NA; ++a)
        if (seen_a[a]) n->sinks[n->n_sinks++] = a; /* sorted ascending by construction */
    free(seen_a);
    size_t S = (size_t)n->slots;
    n->r_ex = (double*)calloc(S * nn, 8);
    n->r_in = (double*)calloc(S * nn, 8);
    n->r_sic = (double*)calloc(S * nn, 8);
    n->r_astro = (double*)calloc(S * na, 8);
    n->pending = (char*)calloc(S, 1);
    return n;
}

void orc_net_free(orc_net* n) {
    if (!n) return;
    for (int s = 0; s < 4; ++s) {
        free(n->set[s].rs); free(n->set[s].tg);
        free(n->set[s].x); free(n->set[s].u); free(n->set[s].t);
    }
    free(n->V_reset); free(n->b); free(n->V); free(n->w); free(n->gex); free(n->dgex);
    free(n->gin); free(n->dgin); free(n->Isic); free(n->exc_in); free(n->inh_in); free(n->refr);
    free(n->Ca); free(n->IP3); free(n->h); free(n->Ca_tot); free(n->IP3_0); free(n->tau);
    free(n->delta); free(n->ip3_in); free(n->r_ex); free(n->r_in); free(n->r_sic);
    free(n->r_astro); free(n->pending); free(n->sic_src); free(n->sinks);
    free(n);
}

int64_t orc_net_table_size(const orc_net* n, int which) { return n->set[which].m; }

void orc_net_table(const orc_net* n, int which, uint32_t* rs, uint32_t* tg) {
    const orc_set* s = &n->set[which];
    memcpy(rs, s->rs, ((size_t)s->rows + 1) * 4);
    if (s->m) memcpy(tg, s->tg, (size_t)s->m * 4);
}

void orc_net_cells(const orc_net* n, double* V_reset, double* b, double* Ca_tot, double* IP3_0,
                   double* tau, double* delta) {
    memcpy(V_reset, n->V_reset, (size_t)n->N * 8);
    memcpy(b, n->b, (size_t)n->N * 8);
    memcpy(Ca_tot, n->Ca_tot, (size_t)n->NA * 8);
    memcpy(IP3_0, n->IP3_0, (size_t)n->NA * 8);
    memcpy(tau, n->tau, (size_t)n->NA * 8);
    memcpy(delta, n->delta, (size_t)n->NA * 8);
}

void orc_net_state(const orc_net* n, double* n7, int32_t* refr, double* a3) {
    size_t N = n->N, NA = n->NA;
    const double* src[7] = {n->V, n->w, n->gex, n->dgex, n->gin, n->dgin, n->Isic};
    for (int k = 0; k < 7; ++k) memcpy(n7 + k * N, src[k], N * 8);
    for (size_t i = 0; i < N; ++i) refr[i] = n->refr[i];
    memcpy(a3, n->Ca, NA * 8);
    memcpy(a3 + NA, n->IP3, NA * 8);
    memcpy(a3 + 2 * NA, n->h, NA * 8);
}

static void add_syn(orc_net* n, uint32_t i, double w) {
    /* neuron.cpp:77-83 */
    if (w > 0.0) n->exc_in[i] += w;
    else if (w < 0.0) n->inh_in[i] -= w;
}

static double stp(orc_net* n, orc_set* s, int64_t k, double t_now) {
    /* network.cpp:230-247 */
    if (!n->stp_on) return s->w;
    double d = t_now - s->t[k];
    double xd = exp(-d / n->tau_rec);
    double ud = n->tau_fac < 1e-10 ? 0.0 : exp(-d / n->tau_fac);
    s->x[k] = 1.0 + (s->x[k] - s->x[k] * s->u[k] - 1.0) * xd;
    s->u[k] = n->U + s->u[k] * (1.0 - n->U) * ud;
    s->t[k] = t_now;
    return s->w * s->x[k] * s->u[k];
}

static void adex(const orc_pop* p, double Vr, double V, double w, double gex, double gin,
                 double Iext, double* dV, double* dw) {
    /* neuron.cpp:85-99 (V_reset does not enter the rates) */
    (void)Vr;
    double Vc = p->V_peak < V ? p->V_peak : V;
    double Isp = p->g_L * p->Delta_T * exp((Vc - p->V_th) / p->Delta_T);
    double Iex = gex * (Vc - p->E_ex);
    double Iin = gin * (Vc - p->E_in);
    *dV = (-p->g_L * (Vc - p->E_L) + Isp - Iex - Iin - w + p->I_e + Iext) / p->C_m;
    *dw = (p->a * (Vc - p->E_L) - w) / p->tau_w;
}

static int cmp_u32(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return x < y ? -1 : x > y;
}

int orc_net_step(orc_net* n, int64_t step, uint32_t* spikes, int cap) {
    const uint32_t N = n->N, NA = n->NA, NE = n->NE;
    const size_t S = (size_t)n->slots;
    /* 1. apply_arrivals (network.cpp:301-338) */
    {
        size_t slot = (size_t)(step % (int64_t)S);
        int sic = n->pending[slot] != 0;
        n->pending[slot] = 0;
        double* ex = n->r_ex + slot * N;
        double* in = n->r_in + slot * N;
        double* sc = n->r_sic + slot * N;
        for (uint32_t i = 0; i < N; ++i) {
            if (ex[i] != 0.0) { add_syn(n, i, ex[i]); ex[i] = 0.0; }
            if (in[i] != 0.0) { add_syn(n, i, -in[i]); in[i] = 0.0; }
            if (sic) { n->Isic[i] = sc[i]; sc[i] = 0.0; }
        }
        double* ai = n->r_astro + slot * NA;
        for (uint32_t k = 0; k < n->n_sinks; ++k) {
            uint32_t a = n->sinks[k];
            if (ai[a] != 0.0) { n->ip3_in[a] += ai[a]; ai[a] = 0.0; }
        }
    }
    /* 2. drive_astrocytes (network.cpp:340-355) */
    if (n->in_a.rate > 0.0) {
        double lam = n->in_a.rate * n->dt * 1e-3;
        for (uint32_t a = 0; a < NA; ++a) {
            orc_rng r;
            orc_rng_init(&r, n->seed ^ 0xC2B2AE3D27D4EB4FULL, (uint64_t)step * 1000003ULL + a);
            int ev = orc_rng_poisson(&r, lam);
            if (ev > 0) n->ip3_in[a] += n->in_a.weight * (double)ev;
        }
    }
    /* 3. astrocyte update (astrocyte.cpp:233-329) */
    {
        const double hs = n->dt / (double)n->substeps;
        long spn = lround(n->in_a.noise_dt / n->dt);
        int steps_per_noise = (int)spn < 1 ? 1 : (int)spn;
        uint64_t idx = (uint64_t)(step / steps_per_noise);
        uint64_t nseed = n->seed ^ 0x9E3779B97F4A7C15ULL;
        double sd = n->in_a.std;
        double shared = (sd > 0.0 && !n->in_a.indep) ? sd * orc_normal(nseed, idx) : 0.0;
        for (uint32_t i = 0; i < NA; ++i) {
            double noise = (sd > 0.0 && n->in_a.indep) ? sd * orc_normal(nseed, idx * 1000003ULL + i)
                                                        : shared;
            orc_astro_advance(n->ac, n->Ca_tot[i], n->IP3_0[i], n->tau[i], n->delta[i],
                              n->ip3_in[i], noise, hs, n->substeps, n->Ca + i, n->IP3 + i,
                              n->h + i);
            n->ip3_in[i] = 0.0;
        }
    }
    /* 4. neuron update (neuron.cpp:101-250) */
    int nsp = 0;
    uint32_t* list = (uint32_t*)malloc((size_t)(N ? N : 1) * 4);
    {
        const double hs = n->dt / (double)n->substeps, dt = n->dt;
        long se = lround(n->in_e.noise_dt / dt), si = lround(n->in_i.noise_dt / dt);
        int spe = (int)se < 1 ? 1 : (int)se, spi = (int)si < 1 ? 1 : (int)si;
        uint64_t ie = (uint64_t)(step / spe), ii = (uint64_t)(step / spi);
        double sh_e = 0.0, sh_i = 0.0;
        if (n->in_e.std > 0.0 && !n->in_e.indep) {
            orc_rng r;
            orc_rng_init(&r, n->seed ^ 0xD1B54A32D192ED03ULL, ie);
            sh_e = 0.0 + n->in_e.std * orc_rng_normal(&r);
        }
        if (n->in_i.std > 0.0 && !n->in_i.indep) {
            orc_rng r;
            orc_rng_init(&r, n->seed ^ 0xA24BAED4963EE407ULL, ii);
            sh_i = 0.0 + n->in_i.std * orc_rng_normal(&r);
        }
        for (uint32_t c = 0; c < N; ++c) {
            const int exc = c < NE;
            const orc_pop* p = exc ? &n->pe : &n->pi;
            const orc_input* in = exc ? &n->in_e : &n->in_i;
            if (in->rate > 0.0) {
                orc_rng r;
                orc_rng_init(&r, n->seed ^ 0x2545F4914F6CDD1DULL, (uint64_t)step * 1000003ULL + c);
                int ev = orc_rng_poisson(&r, in->rate * dt * 1e-3);
                if (ev > 0) n->exc_in[c] += in->weight * (double)ev;
            }
            double Iext = n->Isic[c];
            if (in->std > 0.0) {
                if (in->indep) {
                    orc_rng r;
                    orc_rng_init(&r, n->seed ^ 0x9E3779B185EBCA87ULL,
                                 (exc ? ie : ii) * 1000033ULL + c);
                    Iext += 0.0 + in->std * orc_rng_normal(&r);
                } else {
                    Iext += exc ? sh_e : sh_i;
                }
            }
            const double pex = 2.7182818284590452353602874713527 / p->tau_syn_ex;
            const double pin = 2.7182818284590452353602874713527 / p->tau_syn_in;
            if (n->exc_in[c] != 0.0) { n->dgex[c] += n->exc_in[c] * pex; n->exc_in[c] = 0.0; }
            if (n->inh_in[c] != 0.0) { n->dgin[c] += n->inh_in[c] * pin; n->inh_in[c] = 0.0; }
            double V = n->V[c], w = n->w[c], ge = n->gex[c], dge = n->dgex[c];
            double gi = n->gin[c], dgi = n->dgin[c];
            int spiked = 0;
            orc_pop pc = *p;
            pc.V_reset = n->V_reset[c];
            pc.b = n->b[c];
            for (int s = 0; s < n->substeps; ++s) {
                double xe = exp(-hs / pc.tau_syn_ex), xi = exp(-hs / pc.tau_syn_in);
                double ge1 = xe * (ge + hs * dge), dge1 = xe * dge;
                double gi1 = xi * (gi + hs * dgi), dgi1 = xi * dgi;
                if (n->refr[c] > 0) {
                    V = pc.V_reset;
                    double dV, dw;
                    adex(&pc, pc.V_reset, V, w, ge, gi, Iext, &dV, &dw);
                    w += hs * dw;
                } else {
                    double gem = 0.5 * (ge + ge1), gim = 0.5 * (gi + gi1);
                    double k1V, k1w, k2V, k2w, k3V, k3w, k4V, k4w;
                    adex(&pc, 0, V, w, ge, gi, Iext, &k1V, &k1w);
                    adex(&pc, 0, V + 0.5 * hs * k1V, w + 0.5 * hs * k1w, gem, gim, Iext, &k2V, &k2w);
                    adex(&pc, 0, V + 0.5 * hs * k2V, w + 0.5 * hs * k2w, gem, gim, Iext, &k3V, &k3w);
                    adex(&pc, 0, V + hs * k3V, w + hs * k3w, ge1, gi1, Iext, &k4V, &k4w);
                    V += (hs / 6.0) * (k1V + 2.0 * k2V + 2.0 * k3V + k4V);
                    w += (hs / 6.0) * (k1w + 2.0 * k2w + 2.0 * k3w + k4w);
                }
                ge = ge1; dge = dge1; gi = gi1; dgi = dgi1;
                if (n->refr[c] > 0) {
                    --n->refr[c];
                } else if (V >= pc.V_peak) {
                    V = pc.V_reset;
                    w += pc.b;
                    n->refr[c] = (int)(pc.t_ref / hs + 0.5);
                    spiked = 1;
                }
            }
            n->V[c] = V; n->w[c] = w; n->gex[c] = ge; n->dgex[c] = dge; n->gin[c] = gi;
            n->dgin[c] = dgi;
            if (spiked) list[nsp++] = c;
        }
        qsort(list, (size_t)nsp, 4, cmp_u32); /* ascending already; kept explicit */
    }
    /* 5. deliver_spikes (network.cpp:249-279) */
    {
        double t_now = (double)step * n->dt;
        for (int k = 0; k < nsp; ++k) {
            uint32_t src = list[k];
            if (src < NE) {
                orc_set* e = &n->set[0];
                for (uint32_t q = e->rs[src]; q < e->rs[src + 1]; ++q) {
                    size_t slot = (size_t)((step + e->delay) % (int64_t)S);
                    n->r_ex[slot * N + e->tg[q]] += stp(n, e, q, t_now);
                }
                orc_set* a = &n->set[2];
                for (uint32_t q = a->rs[src]; q < a->rs[src + 1]; ++q) {
                    size_t slot = (size_t)((step + a->delay) % (int64_t)S);
                    n->r_astro[slot * NA + a->tg[q]] += stp(n, a, q, t_now);
                }
            } else {
                orc_set* i = &n->set[1];
                uint32_t s2 = src - NE;
                for (uint32_t q = i->rs[s2]; q < i->rs[s2 + 1]; ++q) {
                    size_t slot = (size_t)((step + i->delay) % (int64_t)S);
                    n->r_in[slot * N + i->tg[q]] -= stp(n, i, q, t_now);
                }
            }
        }
    }
    /* 6. deliver_sic (network.cpp:281-299) */
    if (step % n->sic_interval == 0) {
        n->pending[(size_t)((step + n->sic_delay) % (int64_t)S)] = 1;
        orc_set* s = &n->set[3];
        for (uint32_t k = 0; k < n->n_sic_src; ++k) {
            uint32_t a = n->sic_src[k];
            double y = (n->Ca[a] - n->SIC_th) * 1000.0;
            double f = y <= 1.0 ? 0.0 : n->SIC_scale * log(y);
            if (f == 0.0) continue;
            for (uint32_t q = s->rs[a]; q < s->rs[a + 1]; ++q) {
                size_t slot = (size_t)((step + s->delay) % (int64_t)S);
                n->r_sic[slot * N + s->tg[q]] += s->w * f;
            }
        }
    }
    for (int k = 0; k < nsp && k < cap; ++k) spikes[k] = list[k];
    free(list);
    return nsp;
}
