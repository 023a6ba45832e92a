// Shared definitions of the batched sweep (eb_sweep.cu: build, forward kernel,
// runs) and its adjoint (eb_adjoint.cu: backward kernels, gradients).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "edlut_b200.h"
#include "eb_runtime.h"
#include "eb_types.h"

namespace ebsw {

using namespace eb;

constexpr int kSweepMaxN = 16384;   // neurons per network
constexpr int kListCap = 512;       // sources per delivery pass
constexpr int kBatch = 4;           // synapses per thread per delivery batch
constexpr int kMaxGroups = 3;       // source steps arriving in one step
constexpr int kMaxFrac = 4;         // steps with a partial refractory fraction

// Per neuron-step trajectory code: bits 0-1 refractory class (0 none, 1 frozen,
// 2 fraction), bits 2-3 fraction index, bit 4 spike.
constexpr int kCodeSpike = 16;

// LIF parameters and refractory classes of one network.
struct SweepLif {
    float e_exc, e_inh, e_leak, v_thr, g_leak, inv_c_m;
    float decay[2];         // AMPA, GABA decay factors per (half) step
    int en;                 // bit0 AMPA, bit1 GABA conductances enabled
    int r_free;             // refr >= r_free (or < 0): no refractory scaling
    int r_frac0;            // r_frac0 <= refr < r_free: derivative x frac[refr - r_frac0]
    float frac[kMaxFrac];   // refr < r_frac0: derivative 0
};

struct SweepNet {
    int32_t n, n_in, n_exc, wn;   // wn = bitmask words = ceil(n / 32)
    float p;
    float w_max[3];               // uniform weight range: excitatory, inhibitory, input sources
    int32_t explicit_syn;         // synapses given by the caller (no hash generation)
    int32_t pad;
    int64_t src_off;              // into optr (n + n_in + 1 entries, relative offsets)
    int64_t syn_off;              // first synapse
    int64_t state_off;            // into V / refr / gE / gI
    int64_t in_off, n_in_spikes;  // into in_key / in_src
    int64_t ring_off;             // R * wn words
    int64_t sum_off;              // R * ceil(wn / 32) words
    int64_t rec_off, rec_cap;     // into rec (uint16 neurons)
    float params[10];             // LIF .cfg order
    SweepLif L;
};

struct SweepDev {
    const SweepNet *nets;
    int n_nets;
    const int32_t *order;      // network processing order (largest first)
    int R;                     // delay-ring slots
    int steps_max;
    const int32_t *grp_lo;     // [k] first source step arriving at step k
    const int8_t *grp_n;       // [k] number of source steps arriving at step k
    const uint32_t *optr;      // per source: synapse offset relative to syn_off
    const uint16_t *tgt;
    const float *w;
    float *V, *gE, *gI;
    int32_t *refr;
    uint32_t *ring, *rsum;     // saved bitmask ring and summaries
    const int32_t *in_key;     // arrival step * 4 + phase, sorted per network
    const uint16_t *in_src;    // input neuron (local)
    int64_t *in_cursor;        // per network
    uint16_t *rec;             // recorded neurons, step-major
    int32_t *rec_end;          // [net][step-1] record count after the step
    uint32_t *rec_cnt;         // per network
    unsigned long long *events;  // per network delivered synaptic events
    uint32_t *flags;
    int *queue;
    int64_t *step;             // steps completed
    float dt_ms;
    int integ;
    // observed membrane traces: trace[(net * steps_max + k - 1) * n_obs + m] = V of neuron obs[net * n_obs + m] after step k
    int n_obs;
    const int32_t *obs;
    float *trace;
    // trajectory of one segment (recomputation for the adjoint): per step in the
    // segment and neuron (global index), the integration inputs and the code
    int64_t n_total;
    float *tV, *tE, *tI;
    uint8_t *tcode;
};

// Derivative of V (lif_deriv of the plain path) with the refractory test given as
// a class: 0 none, 1 frozen (derivative 0), 2 scaled by f.
__device__ __forceinline__ float sw_deriv(const SweepLif &L, float V, float gE, float gI, int cls, float f) {
    if (cls == 1) return 0.0f;
    float current = 0.0f;
    if (L.en & 1) current += gE * (L.e_exc - V);
    if (L.en & 2) current += gI * (L.e_inh - V);
    const float full = (current + L.g_leak * (L.e_leak - V)) * L.inv_c_m;
    return cls == 2 ? f * full : full;
}

// EvaluateTimeDependentEquation: g <- 0 below 1e-9, else g * factor.
__device__ __forceinline__ void sw_decay(const SweepLif &L, float &gE, float &gI) {
    const float limit = 1e-9;
    if (L.en & 1) { if (gE < limit) gE = 0.0f; else gE *= L.decay[0]; }
    if (L.en & 2) { if (gI < limit) gI = 0.0f; else gI *= L.decay[1]; }
}

}  // namespace ebsw

struct eb_sweep {
    int device = 0;
    cudaStream_t stream = nullptr;
    int n_nets = 0;
    int integ = eb::INTEG_RK2;
    float dt = 1e-4f;
    float delay = 1e-3f;
    uint64_t seed = 1;
    std::vector<ebsw::SweepNet> nets;
    std::vector<std::vector<float>> in_time;
    std::vector<std::vector<int32_t>> in_cell;
    // explicit connectivity (caller order) of networks that have it
    std::vector<std::vector<int32_t>> xsrc, xtgt;
    std::vector<std::vector<float>> xw;
    ebsw::SweepDev G{};
    ebsw::SweepNet *d_nets = nullptr;
    std::vector<void *> allocs;
    std::vector<float> v_init;
    std::vector<int32_t> h_in_key;      // host copy of the input arrival keys
    std::vector<int32_t> h_arr_step;    // arrival step of the spikes of each source step
    int32_t *d_arr_step = nullptr;
    int64_t *perm = nullptr;            // sweep synapse position -> caller position
    int64_t steps_done = 0;
    bool needs_reset = false;
    int64_t total_syn = 0, dev_bytes = 0, state_n = 0, ring_words = 0, sum_words = 0;
    int max_n = 0;
    int block = 512, npt = 0, wc = 0, swc = 0;
    int steps_per_launch = 1000;
    int grid = 0;
    size_t smem = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_chunks = 0;
    bool built = false;
    // observation and checkpoints
    int ckpt_every = 0, n_ckpt = 0;
    int64_t ckpt_upto = -1;             // a checkpointed run from step 0 has reached this step
    std::vector<int32_t> h_obs;         // observed neurons [n_nets][n_obs]
    std::vector<void *> ckpt;           // per slot: one block holding every state array
    // adjoint scratch (allocated on first use)
    float *lamV = nullptr, *lamE = nullptr, *lamI = nullptr;
    double *gacc = nullptr;             // [4][n_total]: g_leak, e_leak, decay AMPA, decay GABA
    float *muE = nullptr, *muI = nullptr;
    float *gw_sorted = nullptr;
    int32_t *obs_slot = nullptr;        // per neuron: observed slot or -1
    double *red_out = nullptr;          // [n_nets][4] parameter gradient sums
    int64_t traj_steps = 0;
    ~eb_sweep() {
        if (graph) cudaGraphExecDestroy(graph);
        for (void *p : allocs) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
    int dalloc(void **p, size_t b) {
        if (!b) b = 16;
        cudaError_t e = cudaMalloc(p, b);
        if (e != cudaSuccess) { eb::set_error("cudaMalloc(%zu): %s", b, cudaGetErrorString(e)); return EB_ERR_NOMEM; }
        allocs.push_back(*p);
        dev_bytes += (int64_t)b;
        return EB_OK;
    }
    int upload(void **d, const void *src, size_t b) {
        int r = dalloc(d, b);
        if (r) return r;
        if (b && src) {
            cudaError_t e = cudaMemcpy(*d, src, b, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) { eb::set_error("upload: %s", cudaGetErrorString(e)); return EB_ERR_CUDA; }
        }
        return EB_OK;
    }
};

#define SK(call)                                                                                \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            eb::set_error("%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return EB_ERR_CUDA;                                                                 \
        }                                                                                       \
    } while (0)

namespace ebsw {
// Launch one forward chunk of nsteps (TRAJ: record the segment starting at traj_k0).
int enqueue_chunk(eb_sweep *h, int nsteps, cudaStream_t st, bool traj = false, int64_t traj_k0 = 0);
// Bytes of one checkpoint slot; copy the live state into / out of slot c.
size_t checkpoint_bytes(eb_sweep *h);
int checkpoint_save(eb_sweep *h, int c, cudaStream_t st);
int checkpoint_restore(eb_sweep *h, int c, int64_t step, cudaStream_t st);
}  // namespace ebsw
