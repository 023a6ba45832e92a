// Host-side context of the device-resident network (eb_runtime.cu).
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <functional>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "eb_types.h"
#include "eb_kernels.h"

namespace eb {

void set_error(const char *fmt, ...);

// Most steps one launch of a captured graph runs for one population.
constexpr int kMaxFuse = 8;

struct HostPop {
    int kind = KIND_INPUT, integ = 0, bdf_order = 0;
    int64_t n = 0, first = 0;
    float dt = 0.0f;
    std::vector<float> params;
    int en = 0;                 // enabled conductance types (from the synapse types targeting it)
    bool has_out = false, has_plastic_in = false;
    bool output = true;         // spikes go to eb_write_spikes (the layer line's output column)
    bool monitor = false;       // states go to the state monitor file (the layer line's log column)
    int post_chunks = 1;
    int push_threads = 32;
    std::vector<float> rates;   // Poisson generators: per-neuron frequency (Hz)
    PopDev dev{};
};

struct PendingIn {
    float t;
    int64_t cell;
    int64_t seq;
};

}  // namespace eb

struct eb_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // description
    std::vector<eb::HostPop> pops;
    int64_t n_neurons = 0;
    std::vector<std::array<float, 4>> rules;
    std::vector<int64_t> src, tgt;
    std::vector<float> delay, weight, max_weight;
    std::vector<int32_t> stype, rule;
    uint32_t bucket_limit = 8192, input_multiplicity = 2;
    int64_t wide_indegree = 1024;  // block-per-neuron update above this in-degree (0: whenever a bucket holds > 16)
    unsigned long long barrier_spin_limit = eb::kBarrierSpinLimit;  // persistent kernel: polls per barrier wait
    bool barrier_withhold = false;  // block 0 withholds its barrier arrivals (failure-path test)
    size_t bar_words = 0;           // words of pinfo.bar
    uint32_t rng_seed = 1;  // RandomGenerator::srand value (the reference's EDLUTKernel uses 1)
    int64_t rec_cap = 16 << 20;
    // derived
    bool finalized = false;
    float dt_f = 0.0f;
    double dt_s = 0.0;
    int R = 0;
    std::vector<int> pop_of;
    std::vector<int64_t> spos_of, tpos_of;
    eb::NetDev net{};
    int64_t *d_step = nullptr;
    bool has_inputs = false;
    bool inputs_concurrent = false;  // input fan-out can overlap the neuron updates
    int input_threads = 32;
    // persistent multi-step kernel
    bool persistent = false;        // opt-in (eb_set_persistent): grid barriers cost more than launches here
    bool persist_ok = false;        // set at finalize
    int persist_class = 0, persist_grid = 0;
    eb::PersistInfo pinfo{};
    eb::PopDev *d_pops = nullptr;
    bool pops_dirty = true;
    // side streams and events for the parallel branches of a step
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> fork_ev, join_ev;
    // captured graphs as one kernel chain per population (plan_chains)
    struct ChainDep { int other, lag; };       // wait for chain `other` at step r - lag
    std::vector<int> chain_pop;                // chain -> population (-1: all input neurons)
    std::vector<std::vector<ChainDep>> chain_deps;
    std::vector<cudaEvent_t> chain_ev;         // [chain][step of the graph]
    bool chains_ok = false, chains_enabled = true;
    int chain_fuse = 1;                        // steps per launch in a chain (a power of two)
    // time grid and inputs
    std::vector<double> t_host;
    double *d_tstep = nullptr;
    double *d_tgen = nullptr;             // generator update times (when there are generators)
    std::vector<double> tgen_host{0.0};
    bool has_generators = false;
    int64_t *d_instart = nullptr;
    int64_t tcap = 0, tstep_uploaded = 0;
    std::vector<int64_t> in_start_host;
    std::vector<eb::PendingIn> pending;
    int64_t pending_seq = 0;
    std::vector<double> in_times_host;   // staged input times (sorted) and their neurons
    std::vector<uint32_t> in_cells_host;
    double *d_in_time = nullptr;
    uint32_t *d_in_cell = nullptr;
    int64_t in_total = 0, in_cap = 0;
    // run state
    int64_t steps_done = 0;
    int64_t spikes_drained = 0;
    // spike record drain: every recorded step is above rec_step_lo; device sort
    // workspace and the pinned buffer the sorted records are copied through
    int64_t rec_step_lo = 0;
    unsigned long long *rec_tmp = nullptr, *rec_host = nullptr;
    uint32_t *rec_hist = nullptr;
    int64_t rec_sort_cap = 0;
    int graph_steps = 0;
    struct CachedGraph { int K, kernels; cudaGraphExec_t exec; };
    std::vector<CachedGraph> graph_cache;   // captured graphs by step count (at most 8)
    static constexpr int kMinGraph = 8;     // shorter remainders run launch by launch
    static constexpr int kDefaultGraph = 512;  // steps per captured graph
    bool graph_inputs = false;
    bool graphs_valid = false;
    bool trace_pending = false;
    size_t trace_bytes = 0;
    int64_t staged_until = 0;
    int64_t launches = 0;          // kernels launched (graph nodes counted per replay)
    int enq_count = 0;                      // kernels enqueued by the current capture or step
    // per-kernel profiling (plain launches with CUDA events around each kernel)
    bool profile = false;
    cudaStream_t prof_stream = nullptr;
    struct ProfRec { int kind, pop; cudaEvent_t a, b; };
    std::vector<ProfRec> prof_pending;
    struct ProfSum { int kind, pop; int64_t launches; double ms; };
    std::vector<ProfSum> prof_sum;
    std::vector<cudaEvent_t> ev_pool;
    // allocations
    std::vector<void *> allocs;
    int64_t dev_bytes = 0;
    // dynamic device state (what a snapshot copies): (pointer, bytes)
    std::vector<std::pair<void *, size_t>> dyn;
    std::vector<std::pair<int, std::vector<void *>>> snapshots;
    // state monitor file (the reference's -logp): the file, the global neuron and
    // population of each monitored index, and the host copy of their states
    std::FILE *mon_file = nullptr;
    std::vector<int64_t> mon_cell;
    std::vector<int> mon_pop;
    std::vector<float> mon_cur;           // [mon_n][kMaxVars]
    int64_t mon_steps = 0, mon_cap = 0;
    struct HostSnap { int slot; int64_t steps_done, spikes_drained; int steps_since_flush; };
    std::vector<HostSnap> snap_host;

    int dalloc(void **p, size_t bytes);
    void dfree(void *p);
    void dfree_all();
    int add_population(int kind, int64_t n, int integ, int bdf_order, float dt, const float *params, int n_params,
                       int64_t *out_first);
    int finalize(int64_t *out_sorted_perm);
    int ensure_tables(int64_t kmax);
    int stage_inputs(int64_t k0, int64_t k_end);
    void enqueue_step(int rel);
    void fork_join(std::vector<std::function<void(cudaStream_t)>> &work);
    void prof_begin(int kind, int pop, cudaEvent_t *a);
    void prof_end(int kind, int pop, cudaEvent_t a);
    int prof_collect();
    int build_graph(int K);
    CachedGraph *graph_for(int K);
    void plan_chains(const std::vector<int64_t> &out_ptr, const std::vector<uint32_t> &out_tgt,
                     const std::vector<uint16_t> &out_units);
    void enqueue_chains(int K);
    int setup_persistent();
    int seed_generators();
    void enqueue_flush(bool full);
    void enqueue_flush_pop(int q, bool full, cudaStream_t s);
    int flush_post();
    bool lazy_post = false;       // some population defers post-synaptic STDP
    int steps_since_flush = 0;
    int run_async(int64_t n);
    int run_monitored(int64_t n);
    int write_monitor(int64_t k0, int64_t n);
    int close_monitor();
    int sync();
    int snapshot(int slot);
    int restore(int slot);
    ~eb_ctx();
};
