// Shared host/device types of the edlut_b200 runtime.
#pragma once
#include <cstdint>

namespace eb {

enum Kind : int { KIND_INPUT = 0, KIND_LIF = 1, KIND_ADEX = 2, KIND_HH = 3, KIND_POISSON = 4 };
enum Integ : int { INTEG_EULER = 0, INTEG_RK2 = 1, INTEG_RK4 = 2, INTEG_BDF = 3 };

constexpr int kMaxVars = 8;
// Deferred post-synaptic STDP: each neuron keeps its last kPostRing spike times.
// A flush runs at least every kPostGraph steps and brings up to date every neuron
// with more than kPostRing - kPostGraph spikes not yet applied to its synapses, so
// no synapse ever has more than kPostRing of its target's spikes pending.
constexpr int kPostRing = 128;
constexpr int kPostGraph = 64;
constexpr int kNmdaTable = 256;
constexpr int kExptTable = 1024 * 16;
constexpr int kHHTable = 1024 * 256;

// Device error flags (ORed into NetDev::flags).
constexpr uint32_t FLAG_BUCKET_OVERFLOW = 1u;
constexpr uint32_t FLAG_BDF_SINGULAR = 2u;
constexpr uint32_t FLAG_RECORD_OVERFLOW = 4u;
constexpr uint32_t FLAG_SPIKELIST_OVERFLOW = 8u;
constexpr uint32_t FLAG_BARRIER_TIMEOUT = 16u;
constexpr uint32_t FLAG_PERSIST_UNSUPPORTED = 32u;  // persistent kernel met an integrator outside its class
constexpr uint32_t FLAG_MONITOR_OVERFLOW = 64u;     // more deliveries into monitored neurons than the log holds

// One delivery waiting in a target's bucket: the arrival time (double seconds,
// as the reference computes it) and the synapse, both in source-major order
// (spos, the reference's sorted synapse order, breaks ties) and in the
// target-major layout (tpos, where weight and plasticity state live).
struct alignas(16) Arrival {
    double a;
    uint32_t spos;
    uint32_t tpos;
};

// Trace decay factors of one interval (pre- and post-synaptic time constants).
struct alignas(8) DecayPair {
    float pre;
    float post;
};

// One synapse in target-major order: everything a delivered spike and the two
// STDP hooks read or write, in one 32-byte record (one DRAM sector per arrival).
struct alignas(32) SynRec {
    float w;        // weight
    float maxw;     // max weight (clipping of the STDP update)
    float pre;      // STDP pre-synaptic trace
    float post;     // STDP post-synaptic trace
    double last;    // time of the last trace update (s)
    uint8_t stype;  // 0 AMPA, 1 GABA, 2 NMDA
    int8_t rule;    // learning rule, -1 none
    uint8_t pad[6];
};
static_assert(sizeof(SynRec) == 32, "SynRec is one sector");

// One delivery into a monitored neuron: its time and synapse (the fold order
// within a step is (a, spos)), the neuron's index in the monitored list, the
// conductance type and the weight it added, and the step that folded it.
struct alignas(32) MonDelivery {
    double a;
    uint32_t spos;
    uint32_t cell;
    float w;
    int32_t ty;
    int64_t k;
};
static_assert(sizeof(MonDelivery) == 32, "MonDelivery is one sector");

// Per-population parameters, passed by value to the kernels.
struct PopDev {
    int kind, integ, bdf_order, ndiff, nvars;
    int en;          // bit0 EXC, bit1 INH, bit2 NMDA conductances enabled
    int64_t first;   // first global neuron index
    int64_t n;       // neurons in the population
    float p[16];     // model parameters in .cfg order
    float dt_s, dt_ms;
    float inv_c_m, inv_slope, inv_tau_w;
    float adex_vmax, adex_glslope;  // AdEx: vthr + 6 * slope, gl * slope
    float decay[3];  // conductance decay factor per step (RK4: per half step)
    float bdf_coef[7][7];
    float init[kMaxVars];
    float expt_aux, hh_aux, nmda_aux;
    const float *exp_table;
    const float *hh_table;
    const float *nmda_table;
    // state (SoA); x[v] == nullptr for variables that are not stored
    float *x[kMaxVars];
    int32_t *refr;       // LIF: updates since last spike (-1 never)
    int8_t *bdf_state;
    float *bdf_D, *bdf_P;
    // spike list (local indices) with a double-buffered count
    uint32_t *spk;
    uint32_t *spk_count;  // [2]
    // in-synapse ranges (target-major) for neurons of this population
    int wide;            // 1: block-per-neuron update (large in-degree)
    int may_repeat;      // a synapse may deliver twice in one step (input-neuron sources)
    unsigned long long *events;  // delivered synaptic events into this population
    // Poisson generators: LCG state and firing threshold rate * step per neuron
    uint32_t *lcg;
    const double *pthr;
    // Deferred post-synaptic STDP: the times of each neuron's recent spikes,
    // post_t[i * kPostRing + slot] with slot = spike number % kPostRing, and spike counts;
    // null when the population applies post-synaptic STDP eagerly.
    double *post_t;
    uint32_t *post_n;
    uint32_t *post_flushed;  // post_n at the last flush
    // The trace decay factors of the interval ending at each ring spike (from the
    // spike before it), post_f[i * kPostRing + slot] = {pre, post}, for the population's one
    // plastic rule post_rule; null (post_rule -1) when its plastic synapses mix rules.
    DecayPair *post_f;
    int post_rule;
    uint32_t *flush_list;  // [n + 1]: neurons a flush takes, their count last (zero between flushes)
    // state monitor: nonzero when the population's neurons are monitored; their
    // first index in the monitored list
    int mon;
    int64_t mon_base;
};

// Network-wide device pointers, passed by value to the kernels.
struct NetDev {
    int64_t n_neurons;
    int R;                       // delay-ring slots (a power of two)
    const int64_t *step;         // current step counter (steps completed)
    const double *tstep;         // update times t_k, k = 0..
    const double *tgen;          // Poisson generators' own update times (step 0.1f/1000 s)
    // arrival buckets
    uint32_t *cnt;               // [R][n_neurons]
    Arrival *rec;                // [R][cap_total]
    const int64_t *cap_base;     // [n_neurons] offset of each target's bucket
    const uint32_t *cap;         // [n_neurons]
    int64_t cap_total;
    // source-major synapses (reference order)
    const int64_t *out_ptr;      // [n_neurons+1]
    const uint32_t *out_tgt;
    const uint32_t *out_tpos;
    const uint16_t *out_units;   // delay in units of 0.1 ms
    const int64_t *grp_ptr;      // per-source distinct-delay groups [n_neurons+1]
    const uint16_t *grp_units;
    // target-major synapses
    const int64_t *in_ptr;       // [n_neurons+1]
    const int64_t *plastic_end;  // [n_neurons] end of the plastic prefix of each target's range
    SynRec *syn;                 // [m] target-major synapse records
    const float *rule_par;       // [n_rules][6]: max_LTP, tau_LTP, max_LTD, tau_LTD, inv_LTP, inv_LTD
    const float *exp_table;
    float expt_aux;
    // input spikes
    const double *in_time;
    const uint32_t *in_cell;
    const int64_t *in_start;     // [step] first input with time >= t_{step-1}
    // recording
    unsigned long long *rec_buf; // (step << 32) | neuron
    unsigned long long *rec_count;
    int64_t rec_cap;
    float *trace;                // [steps][n][kMaxVars]
    int64_t trace_first, trace_n, trace_k0, trace_steps;
    unsigned long long *events;  // delivered synaptic events, one counter per population
    uint32_t *flags;
    // state monitor: each step's state and spike flag of the monitored neurons at
    // row k % mon_steps, and the log of deliveries into them
    float *mon_x;                // [mon_steps][mon_n][kMaxVars]
    uint8_t *mon_spk;            // [mon_steps][mon_n]
    int64_t mon_n, mon_steps;
    MonDelivery *mon_del;
    unsigned long long *mon_count;
    int64_t mon_cap;
};

}  // namespace eb
