/* TEST INFRASTRUCTURE ONLY -- the CPU oracle for the parity tests.
 *
 * A plain-C restatement of EDLUT's time-driven simulation path as the reference
 * CPU implementation runs it (event engine + time-driven CPU twins + STDP), used
 * by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
 * checker.  Nothing in the shipped library links or calls it.
 *
 * Two arithmetic modes share one implementation (oracle_core.h):
 *   fp64=0  float32 operation-for-operation mirror of the reference CPU code,
 *           including its lookup tables (ExponentialTable, HH rate table, NMDA table);
 *   fp64=1  FP64 state and exact exp(): the error yardstick.
 *
 * Semantics restated (paths relative to the reference's Kernel/ directory):
 *  - synapse order: qsort_inters (source, delay, target), src/spike/Network.cpp:45-68,
 *    made stable by original index for exact ties;
 *  - delays: RoundPropagationDelay, src/spike/Network.cpp:1311-1317
 *    (floor(d*1e4 + 5e-5)*1e-4, minimum 1e-4 s);
 *  - update times: first at dt, then t += dt (double of the float step),
 *    src/simulation/Simulation.cpp:246, src/simulation/TimeEventUpdateNeurons.cpp:115;
 *  - an arrival at time a affects the first update at time > a (update events outrank
 *    propagated spikes at equal time, include/simulation/Event.h:37);
 *  - internal spike at update time t: one delivery event per distinct delay d at t+d,
 *    sources in index order (src/spike/TimeDrivenInternalSpike.cpp:38-58,66-104);
 *  - input spike at time t (float from the input file): delivery at t+d0, then for the
 *    next distinct delay at (a_j - d_j) + d_{j+1}, src/spike/PropagatedSpike.cpp:60-100;
 *  - delivery per synapse: g[type] += w (src/neuron_model/LIFTimeDrivenModel.cpp:77-83),
 *    then the STDP pre hook (src/spike/PropagatedSpikeGroup.cpp:112-149);
 *  - STDP: src/learning_rules/STDPWeightChange.cpp:43-76, STDPState.cpp:74-97,
 *    clipping include/spike/Interconnection.h:400-407.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define EO_MAXV 8
enum { EO_INPUT = 0, EO_LIF = 1, EO_ADEX = 2, EO_HH = 3, EO_POISSON = 4 };
enum { EO_EULER = 0, EO_RK2 = 1, EO_RK4 = 2, EO_BDF = 3 };

/* ExponentialTable constants, include/simulation/ExponentialTable.h / ExponentialTable.cpp */
#define EXPT_SIZE (1024 * 16)
static const float EXPT_MIN = -20.0f, EXPT_MAX = 20.0f;
static float EXPT_AUX;
static float g_exptable[EXPT_SIZE];
/* HH table constants, HHTimeDrivenModel.cpp:27-30, HHTimeDrivenModel.h:79 */
#define HH_TABLE (1024 * 256)
static const float HH_MIN_V = -90.0f, HH_MAX_V = 50.0f;
static float HH_AUX;
#define NMDA_TABLE 256

typedef struct eo_pop {
    int32_t kind, integ, bdf_order, first, n, pad;
    float dt;          /* integration step in seconds (float, as parsed from .cfg) */
    float params[16];  /* model parameters in .cfg order */
} eo_pop;

typedef struct eo_popstate {
    int kind, integ, bdf_order, ndiff, nvars;
    int64_t first, n;
    float p[16];
    float dt_s, dt_ms;
    int en[4];                  /* EXC, INH, NMDA, EXT_I enabled (CheckSynapseType) */
    float inv_c_m, inv_thr_slo_fac, inv_tau_w, inv_tau[3];
    float decay_f32[1][3];
    double decay_f64[1][3];
    float bdf_coef[7][7];
    float *hh_table;
    float nmda_table[NMDA_TABLE];
    float nmda_aux;
    int *bdf_state;
    void *bdf_D_f32, *bdf_P_f32, *bdf_D_f64, *bdf_P_f64;
    float init[EO_MAXV];
    uint32_t *rng;              /* Poisson generators: RandomGenerator::next_element per neuron */
} eo_popstate;

#define R float
#define SFX(n) n##_f32
#define ORACLE_F32 1
#include "oracle_core.h"
#undef R
#undef SFX
#undef ORACLE_F32
#define R double
#define SFX(n) n##_f64
#define ORACLE_F32 0
#include "oracle_core.h"
#undef R
#undef SFX
#undef ORACLE_F32

static int g_tables_ready = 0;
static void build_global_tables(void) {
    if (g_tables_ready) return;
    EXPT_AUX = (EXPT_SIZE - 1) / (EXPT_MAX - EXPT_MIN);
    HH_AUX = (HH_TABLE - 1) / (HH_MAX_V - HH_MIN_V);
    for (int i = 0; i < EXPT_SIZE; ++i) {
        float e = EXPT_MIN + ((EXPT_MAX - EXPT_MIN) * i) / (EXPT_SIZE - 1);
        g_exptable[i] = (float)exp((double)e); /* double exp, ExponentialTable.h:76-83 */
    }
    g_tables_ready = 1;
}

/* Generate_channel_values, HHTimeDrivenModel.h:372-421 (float expf arithmetic). */
static void build_hh_table(eo_popstate *ps) {
    float vt = ps->p[5];
    ps->hh_table = (float *)malloc(sizeof(float) * (size_t)HH_TABLE * 6);
    for (int i = 0; i < HH_TABLE; ++i) {
        float V = HH_MIN_V + ((HH_MAX_V - HH_MIN_V) * i) / (HH_TABLE - 1);
        float *o = ps->hh_table + (size_t)i * 6;
        float x = 13.0f - V + vt;
        o[0] = (x == 0.0) ? 1.279999894092334f : 0.32f * x / (expf(x * 0.25f) - 1.0f);
        x = V - vt - 40.0f;
        o[1] = (x == 0.0) ? 1.400030971093304f : 0.28f * x / (expf(x * 0.2f) - 1.0f);
        o[2] = 0.128f * expf((17.0f - V + vt) * 0.05555555f);
        o[3] = 4.0f / (1.0f + expf((40.0f - V + vt) * 0.2f));
        x = 15.0f - V + vt;
        o[4] = (x == 0.0) ? 0.1599999867615418f : 0.032f * x / (expf(x * 0.2f) - 1.0f);
        o[5] = 0.5f * expf((10.0f - V + vt) * 0.025f);
    }
}

/* Generate_g_nmda_inf_values, LIFTimeDrivenModel.cpp:26-36 (float expf). */
static void build_nmda_table(eo_popstate *ps, float e_exc, float e_inh) {
    ps->nmda_aux = (NMDA_TABLE - 1) / (e_exc - e_inh);
    for (int i = 0; i < NMDA_TABLE; ++i) {
        float V = e_inh + ((e_exc - e_inh) * i) / (NMDA_TABLE - 1);
        ps->nmda_table[i] = 1.0f / (1.0f + expf(-0.062f * V) * (1.2f / 3.57f));
    }
}

static void init_pop(eo_popstate *ps, const eo_pop *pp, int fp64) {
    memset(ps, 0, sizeof(*ps));
    ps->kind = pp->kind; ps->integ = pp->integ; ps->bdf_order = pp->bdf_order;
    ps->first = pp->first; ps->n = pp->n;
    memcpy(ps->p, pp->params, sizeof(ps->p));
    ps->dt_s = pp->dt;
    ps->dt_ms = pp->dt * 1000.0f; /* IntegrationMethodFast.h:192 */
    const float *p = ps->p;
    float tau[3] = {0, 0, 0};
    if (ps->kind == EO_POISSON) {
        /* PoissonGeneratorDeviceVector: sampling period 0.1f ms in a millisecond-scale
         * model, step = 0.1f / 1000 s (PoissonGeneratorDeviceVector.cpp:26,137) */
        ps->ndiff = 0; ps->nvars = 0;
        ps->dt_s = 0.1f / 1000.0f;
        ps->dt_ms = ps->dt_s * 1000.0f;
        ps->rng = (uint32_t *)calloc((size_t)ps->n, sizeof(uint32_t));
        return;
    }
    if (ps->kind == EO_LIF) {
        ps->ndiff = 1; ps->nvars = 5;
        ps->inv_c_m = (float)(1. / (double)p[4]);
        tau[0] = p[5]; tau[1] = p[6]; tau[2] = p[9];
        float init[5] = {p[2], 0, 0, 0, 0};
        memcpy(ps->init, init, sizeof(init));
        build_nmda_table(ps, p[0], p[1]);
    } else if (ps->kind == EO_ADEX) {
        ps->ndiff = 2; ps->nvars = 6;
        ps->inv_c_m = (float)(1. / (double)p[10]);
        ps->inv_thr_slo_fac = (float)(1. / (double)p[2]);
        ps->inv_tau_w = (float)(1. / (double)p[4]);
        tau[0] = p[11]; tau[1] = p[12]; tau[2] = p[13];
        float init[6] = {p[8], 0, 0, 0, 0, 0};
        memcpy(ps->init, init, sizeof(init));
        build_nmda_table(ps, p[5], p[6]);
    } else if (ps->kind == EO_HH) {
        ps->ndiff = 4; ps->nvars = 8;
        ps->inv_c_m = (float)(1. / (double)p[4]);
        tau[0] = p[6]; tau[1] = p[7]; tau[2] = p[8];
        build_hh_table(ps);
        build_nmda_table(ps, p[0], p[1]);
        /* HHTimeDrivenModel::InitializeStates, HHTimeDrivenModel.cpp:141-166 */
        float e_leak = p[2];
        if (!fp64) {
            int pos = (int)((e_leak - HH_MIN_V) * HH_AUX);
            if (pos < 0) pos = 0; else if (pos > HH_TABLE - 1) pos = HH_TABLE - 1;
            const float *v = ps->hh_table + (size_t)pos * 6;
            float init[8] = {e_leak, v[0] / (v[0] + v[1]), v[2] / (v[2] + v[3]), v[4] / (v[4] + v[5]), 0, 0, 0, 0};
            memcpy(ps->init, init, sizeof(init));
        } else {
            double r[6];
            hh_rates_f64(ps, (double)e_leak, r);
            float init[8] = {e_leak, (float)(r[0] / (r[0] + r[1])), (float)(r[2] / (r[2] + r[3])),
                             (float)(r[4] / (r[4] + r[5])), 0, 0, 0, 0};
            memcpy(ps->init, init, sizeof(init));
        }
    }
    for (int c = 0; c < 3; ++c) ps->inv_tau[c] = tau[c] > 0 ? (float)(1.0 / (double)tau[c]) : 0.0f;
    /* Calculate_conductance_exp_values: factor at dt (Euler/RK2/BDF) or dt/2 (RK4), RK4.h:362 */
    float el = (ps->integ == EO_RK4) ? ps->dt_ms * 0.5f : ps->dt_ms;
    double eld = (ps->integ == EO_RK4) ? (double)ps->dt_ms * 0.5 : (double)ps->dt_ms;
    for (int c = 0; c < 3; ++c) {
        ps->decay_f32[0][c] = expf(-el * ps->inv_tau[c]);
        ps->decay_f64[0][c] = tau[c] > 0 ? exp(-eld / (double)tau[c]) : 0.0;
    }
    /* BDF coefficients, BDFn.h:620-668 */
    static const float num[7][7] = {{1, 1, 0, 0, 0, 0, 0}, {1, 1, 0, 0, 0, 0, 0}, {2, 4, -1, 0, 0, 0, 0},
                                    {6, 18, -9, 2, 0, 0, 0}, {12, 48, -36, 16, -3, 0, 0},
                                    {60, 300, -300, 200, -75, 12, 0}, {60, 360, -450, 400, -225, 72, -10}};
    static const float den[7] = {1, 1, 3, 11, 25, 137, 147};
    for (int r = 0; r < 7; ++r)
        for (int c = 0; c < 7; ++c) ps->bdf_coef[r][c] = num[r][c] / den[r];
    if (ps->kind != EO_INPUT && ps->integ == EO_BDF) {
        int o = ps->bdf_order;
        ps->bdf_state = (int *)calloc((size_t)ps->n, sizeof(int));
        ps->bdf_D_f32 = calloc((size_t)o * ps->n * ps->ndiff, sizeof(float));
        ps->bdf_P_f32 = calloc((size_t)(o > 1 ? o - 1 : 1) * ps->n * ps->ndiff, sizeof(float));
        ps->bdf_D_f64 = calloc((size_t)o * ps->n * ps->ndiff, sizeof(double));
        ps->bdf_P_f64 = calloc((size_t)(o > 1 ? o - 1 : 1) * ps->n * ps->ndiff, sizeof(double));
    }
}

static void free_pop(eo_popstate *ps) {
    free(ps->hh_table); free(ps->bdf_state); free(ps->rng);
    free(ps->bdf_D_f32); free(ps->bdf_P_f32); free(ps->bdf_D_f64); free(ps->bdf_P_f64);
}

/* ------------------------------------------------------------- events -- */
typedef struct {
    double t;       /* arrival time */
    int64_t seq;    /* creation order, breaks exact ties */
    int64_t src;    /* source neuron */
    int32_t didx;   /* index into the source's distinct delays */
    int32_t cascade;/* input spikes: schedule the next delay group from this one */
} eo_event;

typedef struct { eo_event *a; int64_t n, cap; } eo_heap;
static int ev_less(const eo_event *x, const eo_event *y) {
    return x->t < y->t || (x->t == y->t && x->seq < y->seq);
}
static void heap_push(eo_heap *h, eo_event e) {
    if (h->n == h->cap) { h->cap = h->cap ? 2 * h->cap : 1024; h->a = (eo_event *)realloc(h->a, sizeof(eo_event) * h->cap); }
    int64_t i = h->n++;
    h->a[i] = e;
    while (i > 0) {
        int64_t p = (i - 1) / 2;
        if (!ev_less(&h->a[i], &h->a[p])) break;
        eo_event t = h->a[i]; h->a[i] = h->a[p]; h->a[p] = t; i = p;
    }
}
static eo_event heap_pop(eo_heap *h) {
    eo_event top = h->a[0];
    h->a[0] = h->a[--h->n];
    int64_t i = 0;
    for (;;) {
        int64_t l = 2 * i + 1, r = l + 1, m = i;
        if (l < h->n && ev_less(&h->a[l], &h->a[m])) m = l;
        if (r < h->n && ev_less(&h->a[r], &h->a[m])) m = r;
        if (m == i) break;
        eo_event t = h->a[i]; h->a[i] = h->a[m]; h->a[m] = t; i = m;
    }
    return top;
}

/* ------------------------------------------------------------- network -- */
static const int64_t *g_sort_src, *g_sort_tgt;
static const double *g_sort_delay;
static int cmp_syn(const void *a, const void *b) {
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    if (g_sort_src[x] != g_sort_src[y]) return g_sort_src[x] < g_sort_src[y] ? -1 : 1;
    if (g_sort_delay[x] != g_sort_delay[y]) return g_sort_delay[x] < g_sort_delay[y] ? -1 : 1;
    if (g_sort_tgt[x] != g_sort_tgt[y]) return g_sort_tgt[x] < g_sort_tgt[y] ? -1 : 1;
    return x < y ? -1 : (x > y);
}

/* RoundPropagationDelay, src/spike/Network.cpp:1311-1317 */
double eo_round_delay(float d) {
    const double minpd = 0.0001, invminpd = 1.0 / 0.0001;
    double r = floor((double)d * invminpd + minpd * 0.5) * minpd;
    return r <= 0 ? minpd : r;
}

/* RandomGenerator (include/simulation/RandomGenerator.h:61-107): srand value;
 * EDLUTKernel calls srand(1) (src/EDLUTKernel.cpp:88). */
static uint32_t g_seed = 1;
void eo_set_seed(uint32_t seed) { g_seed = seed & 0x7fffffffu; }
static uint32_t next_seed(uint32_t g) { return (g * 765426813u + 54321u) & 0x7fffffffu; }

/* Error codes */
#define EO_OK 0
#define EO_ERR_ARG -1
#define EO_ERR_SINGULAR -2
#define EO_ERR_SPIKECAP -3

/* Run a whole simulation.  All arrays are caller-owned.
 *  pops[n_pops]            populations (kind EO_INPUT for InputSpikeNeuronModel layers)
 *  synapses (m)            network-file order
 *  stdp[4*n_rules]         max_LTP tau_LTP max_LTD tau_LTD per rule (rule[k] = -1: static)
 *  inputs (n_in)           input-spike times (float seconds) and cells
 *  trace                   trace_steps x trace_n x EO_MAXV doubles, state after each update
 *  outputs                 spikes (step 1-based, cell), final weights (original order),
 *                          sorted_perm[pos] = original index, n_events delivered before the
 *                          last update (tail=1: and within 0.05 dt after it, as the harness
 *                          that slices the reference run does)
 */
int eo_run(int32_t n_pops, const eo_pop *pops, int64_t n_neurons,
           int64_t m, const int64_t *src, const int64_t *tgt, const float *delay,
           const int32_t *type, const float *weight, const float *max_weight, const int32_t *rule,
           int32_t n_rules, const float *stdp,
           int64_t n_in, const float *in_time, const int64_t *in_cell,
           int64_t nsteps, int32_t fp64, int32_t tail,
           int64_t trace_steps, int64_t trace_first, int64_t trace_n, double *trace,
           int64_t spike_cap, int64_t *n_spikes, int64_t *spike_step, int64_t *spike_cell,
           double *w_final, int64_t *sorted_perm, int64_t *n_events) {
    build_global_tables();
    if (n_pops <= 0 || n_neurons <= 0 || nsteps < 0) return EO_ERR_ARG;
    int rc = EO_OK;
    eo_popstate *ps = (eo_popstate *)calloc((size_t)n_pops, sizeof(eo_popstate));
    int32_t *pop_of = (int32_t *)malloc(sizeof(int32_t) * (size_t)n_neurons);
    for (int q = 0; q < n_pops; ++q) {
        init_pop(&ps[q], &pops[q], fp64);
        for (int64_t i = pops[q].first; i < pops[q].first + pops[q].n; ++i) pop_of[i] = q;
    }
    /* Generator seeds: one RandomGenerator for the weights file (Network.cpp:662), then
     * one per generator neuron in Network::InitializeStates: model types (equal
     * parameters share one, Network.cpp:1023-1036) in order of first appearance, the
     * neurons of a type in index order (PoissonGeneratorDeviceVector.cpp:96-99). */
    {
        uint32_t g = next_seed(g_seed);
        for (int q = 0; q < n_pops; ++q) {
            if (ps[q].kind != EO_POISSON) continue;
            int first_of_type = 1;
            for (int r = 0; r < q; ++r)
                if (ps[r].kind == EO_POISSON && ps[r].p[0] == ps[q].p[0]) first_of_type = 0;
            if (!first_of_type) continue;
            for (int r = q; r < n_pops; ++r) {
                if (ps[r].kind != EO_POISSON || ps[r].p[0] != ps[q].p[0]) continue;
                for (int64_t j = 0; j < ps[r].n; ++j) { ps[r].rng[j] = g; g = next_seed(g); }
            }
        }
    }
    /* Synapse types enable the conductances of the target model (CheckSynapseType). */
    for (int64_t k = 0; k < m; ++k) {
        eo_popstate *t = &ps[pop_of[tgt[k]]];
        if (type[k] >= 0 && type[k] < 4) t->en[type[k]] = 1;
    }
    /* Neuron state: float and double copies (one is used). */
    float *xf = (float *)calloc((size_t)n_neurons * EO_MAXV, sizeof(float));
    double *xd = (double *)calloc((size_t)n_neurons * EO_MAXV, sizeof(double));
    double *lst = (double *)malloc(sizeof(double) * (size_t)n_neurons);
    for (int64_t i = 0; i < n_neurons; ++i) {
        eo_popstate *p = &ps[pop_of[i]];
        for (int v = 0; v < EO_MAXV; ++v) { xf[i * EO_MAXV + v] = p->init[v]; xd[i * EO_MAXV + v] = p->init[v]; }
        lst[i] = 100.0; /* VectorNeuronState::InitializeStates, VectorNeuronState.cpp:272-274 */
    }
    /* Sorted synapse order and per-source delay groups. */
    double *dly = (double *)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    int64_t *ord = (int64_t *)malloc(sizeof(int64_t) * (size_t)(m > 0 ? m : 1));
    for (int64_t k = 0; k < m; ++k) { dly[k] = eo_round_delay(delay[k]); ord[k] = k; }
    g_sort_src = src; g_sort_tgt = tgt; g_sort_delay = dly;
    qsort(ord, (size_t)m, sizeof(int64_t), cmp_syn);
    if (sorted_perm) memcpy(sorted_perm, ord, sizeof(int64_t) * (size_t)m);
    int64_t *out_ptr = (int64_t *)calloc((size_t)n_neurons + 1, sizeof(int64_t));
    for (int64_t k = 0; k < m; ++k) out_ptr[src[k] + 1]++;
    for (int64_t i = 0; i < n_neurons; ++i) out_ptr[i + 1] += out_ptr[i];
    /* distinct delays per source: grp_ptr[s]..grp_ptr[s+1] into grp_start (positions in ord) */
    int64_t *grp_ptr = (int64_t *)calloc((size_t)n_neurons + 1, sizeof(int64_t));
    int64_t *grp_start = (int64_t *)malloc(sizeof(int64_t) * (size_t)(m + n_neurons + 1));
    int64_t ng = 0;
    for (int64_t s = 0; s < n_neurons; ++s) {
        grp_ptr[s] = ng;
        for (int64_t k = out_ptr[s]; k < out_ptr[s + 1]; ++k)
            if (k == out_ptr[s] || dly[ord[k]] != dly[ord[k - 1]]) grp_start[ng++] = k;
    }
    grp_ptr[n_neurons] = ng;
    grp_start[ng] = m;
    /* group g spans [grp_start[g], end) where end = next group's start within the source */
    /* Plastic inputs per target (for the post-synaptic STDP hook). */
    int64_t *in_ptr = (int64_t *)calloc((size_t)n_neurons + 1, sizeof(int64_t));
    for (int64_t k = 0; k < m; ++k) if (rule[k] >= 0) in_ptr[tgt[k] + 1]++;
    for (int64_t i = 0; i < n_neurons; ++i) in_ptr[i + 1] += in_ptr[i];
    int64_t *in_syn = (int64_t *)malloc(sizeof(int64_t) * (size_t)(in_ptr[n_neurons] + 1));
    int64_t *fill = (int64_t *)calloc((size_t)n_neurons, sizeof(int64_t));
    for (int64_t k = 0; k < m; ++k)
        if (rule[k] >= 0) in_syn[in_ptr[tgt[k]] + fill[tgt[k]]++] = k;
    /* Weights and STDP state (float mirror or double). */
    float *wf = (float *)malloc(sizeof(float) * (size_t)(m > 0 ? m : 1));
    double *wd = (double *)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    float *pre_f = (float *)calloc((size_t)(m > 0 ? m : 1), sizeof(float));
    float *post_f = (float *)calloc((size_t)(m > 0 ? m : 1), sizeof(float));
    double *pre_d = (double *)calloc((size_t)(m > 0 ? m : 1), sizeof(double));
    double *post_d = (double *)calloc((size_t)(m > 0 ? m : 1), sizeof(double));
    double *last = (double *)calloc((size_t)(m > 0 ? m : 1), sizeof(double));
    for (int64_t k = 0; k < m; ++k) { wf[k] = weight[k]; wd[k] = weight[k]; }
    float *inv_ltp = (float *)malloc(sizeof(float) * (size_t)(n_rules + 1));
    float *inv_ltd = (float *)malloc(sizeof(float) * (size_t)(n_rules + 1));
    for (int r = 0; r < n_rules; ++r) { inv_ltp[r] = 1.0f / stdp[4 * r + 1]; inv_ltd[r] = 1.0f / stdp[4 * r + 3]; }

    eo_heap heap = {0, 0, 0};
    int64_t seq = 0;
    for (int64_t q = 0; q < n_in; ++q) {
        int64_t s = in_cell[q];
        if (grp_ptr[s] == grp_ptr[s + 1]) continue;
        eo_event e = {(double)in_time[q] + dly[ord[grp_start[grp_ptr[s]]]], seq++, s, 0, 1};
        heap_push(&heap, e);
    }
    int64_t nspk = 0, nev = 0;
    double t_now = 0.0;
    float dt_f = 0;
    for (int q = 0; q < n_pops; ++q) if (ps[q].kind != EO_INPUT && ps[q].kind != EO_POISSON) { dt_f = ps[q].dt_s; break; }
    if (dt_f == 0) dt_f = 0.1f / 1000.0f;
    /* Poisson generators run on their own grid: TimeEventUpdateNeurons of their model
     * at t' = t' + (double)(0.1f / 1000) (TimeEventUpdateNeurons.cpp:115); their k-th
     * update falls between the k-th and (k+1)-th neuron updates for the runs here. */
    double t_gen = 0.0;

    for (int64_t step = 1; step <= nsteps + (tail ? 1 : 0) && rc == EO_OK; ++step) {
        int last_pass = step > nsteps;
        /* tail: after the last update, also deliver what arrives within 0.05 dt of it */
        double t_lim = last_pass ? t_now + 0.05 * (double)dt_f : t_now + (double)dt_f;
        if (!last_pass) t_now += (double)dt_f;
        /* 1. deliveries with arrival time < t_now */
        while (heap.n > 0 && heap.a[0].t < t_lim) {
            eo_event e = heap_pop(&heap);
            int64_t s = e.src, g = grp_ptr[s] + e.didx;
            int64_t gend = (g + 1 < grp_ptr[s + 1]) ? grp_start[g + 1] : out_ptr[s + 1];
            for (int64_t pos = grp_start[g]; pos < gend; ++pos) {
                int64_t k = ord[pos];
                int64_t t = tgt[k];
                eo_popstate *tp = &ps[pop_of[t]];
                int ty = type[k];
                if (ty >= 0 && ty < 3) {
                    int v = tp->ndiff + ty;
                    if (fp64) xd[t * EO_MAXV + v] += wd[k];
                    else xf[t * EO_MAXV + v] += wf[k];
                }
                nev++;
                int r = rule[k];
                if (r >= 0) { /* STDPWeightChange::ApplyPreSynapticSpike */
                    if (fp64) {
                        double el = e.t - last[k];
                        pre_d[k] *= exp(-el / (double)stdp[4 * r + 1]);
                        post_d[k] *= exp(-el / (double)stdp[4 * r + 3]);
                        last[k] = e.t;
                        pre_d[k] += 1.0;
                        wd[k] += -(double)stdp[4 * r + 2] * post_d[k];
                        if (wd[k] > max_weight[k]) wd[k] = max_weight[k]; else if (wd[k] < 0.0) wd[k] = 0.0;
                    } else {
                        float el = (float)(e.t - last[k]);
                        pre_f[k] *= expt_f32(-el * inv_ltp[r]);
                        post_f[k] *= expt_f32(-el * inv_ltd[r]);
                        last[k] = e.t;
                        pre_f[k] += 1.0f;
                        wf[k] += -stdp[4 * r + 2] * post_f[k];
                        if (wf[k] > max_weight[k]) wf[k] = max_weight[k]; else if (wf[k] < 0.0f) wf[k] = 0.0f;
                    }
                }
            }
            if (e.cascade && e.didx + 1 < grp_ptr[s + 1] - grp_ptr[s]) {
                double d0 = dly[ord[grp_start[g]]], d1 = dly[ord[grp_start[g + 1]]];
                eo_event n2 = {e.t - d0 + d1, seq++, s, e.didx + 1, 1};
                heap_push(&heap, n2);
            }
        }
        if (last_pass) break;
        t_gen += (double)(0.1f / 1000.0f);
        /* 2. neuron updates, 3. spikes (per population, ascending index) */
        for (int q = 0; q < n_pops && rc == EO_OK; ++q) {
            eo_popstate *p = &ps[q];
            if (p->kind == EO_INPUT) continue;
            for (int64_t j = 0; j < p->n; ++j) {
                int64_t i = p->first + j;
                int sp;
                if (p->kind == EO_POISSON) {
                    /* PoissonGeneratorDeviceVector::UpdateState, PoissonGeneratorDeviceVector.cpp:56-70 */
                    sp = 0;
                    if (p->p[0] > 0.0f) {
                        p->rng[j] = (p->rng[j] * 1103515245u + 12345u) & 0x7fffffffu;
                        float r = ((float)p->rng[j]) / 2147483647;
                        sp = (double)p->p[0] * (double)p->dt_s > (double)r;
                    }
                } else {
                    sp = fp64 ? step_neuron_f64(p, j, xd + i * EO_MAXV, &lst[i])
                              : step_neuron_f32(p, j, xf + i * EO_MAXV, &lst[i]);
                    if (sp < 0) { rc = EO_ERR_SINGULAR; break; }
                    /* CheckValidIntegration: reset neurons whose V became NaN */
                    if (fp64 ? isnan(xd[i * EO_MAXV]) : isnan(xf[i * EO_MAXV]))
                        for (int v = 0; v < EO_MAXV; ++v) { xf[i * EO_MAXV + v] = p->init[v]; xd[i * EO_MAXV + v] = p->init[v]; }
                }
                if (!sp) continue;
                if (nspk >= spike_cap) { rc = EO_ERR_SPIKECAP; break; }
                spike_step[nspk] = step; spike_cell[nspk] = i; nspk++;
                /* STDPWeightChange::ApplyPostSynapticSpike over the neuron's plastic inputs */
                for (int64_t a = in_ptr[i]; a < in_ptr[i + 1]; ++a) {
                    int64_t k = in_syn[a];
                    int r = rule[k];
                    if (fp64) {
                        double el = t_now - last[k];
                        pre_d[k] *= exp(-el / (double)stdp[4 * r + 1]);
                        post_d[k] *= exp(-el / (double)stdp[4 * r + 3]);
                        last[k] = t_now;
                        post_d[k] += 1.0;
                        wd[k] += (double)stdp[4 * r + 0] * pre_d[k];
                        if (wd[k] > max_weight[k]) wd[k] = max_weight[k]; else if (wd[k] < 0.0) wd[k] = 0.0;
                    } else {
                        float el = (float)(t_now - last[k]);
                        pre_f[k] *= expt_f32(-el * inv_ltp[r]);
                        post_f[k] *= expt_f32(-el * inv_ltd[r]);
                        last[k] = t_now;
                        post_f[k] += 1.0f;
                        wf[k] += stdp[4 * r + 0] * pre_f[k];
                        if (wf[k] > max_weight[k]) wf[k] = max_weight[k]; else if (wf[k] < 0.0f) wf[k] = 0.0f;
                    }
                }
                /* one delivery event per distinct delay at t + d */
                const double t_spk = p->kind == EO_POISSON ? t_gen : t_now;
                for (int64_t g = grp_ptr[i]; g < grp_ptr[i + 1]; ++g) {
                    eo_event e = {t_spk + dly[ord[grp_start[g]]], seq++, i, (int32_t)(g - grp_ptr[i]), 0};
                    heap_push(&heap, e);
                }
            }
        }
        if (trace && step <= trace_steps) {
            for (int64_t c = 0; c < trace_n; ++c)
                for (int v = 0; v < EO_MAXV; ++v)
                    trace[((step - 1) * trace_n + c) * EO_MAXV + v] =
                        fp64 ? xd[(trace_first + c) * EO_MAXV + v] : (double)xf[(trace_first + c) * EO_MAXV + v];
        }
    }
    *n_spikes = nspk;
    if (n_events) *n_events = nev;
    if (w_final) for (int64_t k = 0; k < m; ++k) w_final[k] = fp64 ? wd[k] : (double)wf[k];

    for (int q = 0; q < n_pops; ++q) free_pop(&ps[q]);
    free(ps); free(pop_of); free(xf); free(xd); free(lst); free(dly); free(ord); free(out_ptr);
    free(grp_ptr); free(grp_start); free(in_ptr); free(in_syn); free(fill); free(wf); free(wd);
    free(pre_f); free(post_f); free(pre_d); free(post_d); free(last); free(inv_ltp); free(inv_ltd);
    free(heap.a);
    return rc;
}

/* Exposed for table checks against the reference's own tables. */
void eo_exp_table(float *out) { build_global_tables(); memcpy(out, g_exptable, sizeof(g_exptable)); }
void eo_hh_table(float v_thr, float *out) {
    build_global_tables();
    eo_popstate ps; memset(&ps, 0, sizeof(ps)); ps.p[5] = v_thr;
    build_hh_table(&ps);
    memcpy(out, ps.hh_table, sizeof(float) * (size_t)HH_TABLE * 6);
    free(ps.hh_table);
}
void eo_nmda_table(float e_exc, float e_inh, float *out) {
    eo_popstate ps; build_nmda_table(&ps, e_exc, e_inh);
    memcpy(out, ps.nmda_table, sizeof(ps.nmda_table));
}
