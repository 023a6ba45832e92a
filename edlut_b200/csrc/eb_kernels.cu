// Kernels of one simulation step of the device-resident network.
//
// Per step k (update time t_k), in stream order:
//   k_input_push   fan out the input-neuron spikes of [t_{k-1}, t_k) into the
//                  arrival buckets of the steps they reach
//   k_update_*     per model population: fold this step's arrivals into the
//                  conductances in the reference's delivery order (arrival time,
//                  then synapse order) with the STDP pre-synaptic update, advance
//                  the neuron one integration step, test the spike condition,
//                  compact the spiking neurons (warp ballot) and record them
//   k_post_stdp    per population with plastic inputs: post-synaptic STDP update
//                  of every plastic input synapse of each neuron that spiked
//   k_push         per population with outputs: fan each spike out into the
//                  arrival buckets of its targets (integer atomics only; the
//                  fold sorts, so results do not depend on atomic order)
// The step index is read from device memory (base + offset baked into the
// launch), so one captured CUDA graph of K steps replays for any K steps.
//
// Reference behaviour restated here (paths relative to the reference's Kernel/):
//   delivery g[type] += w then STDP pre hook: src/spike/PropagatedSpikeGroup.cpp:112-149,
//     src/neuron_model/LIFTimeDrivenModel.cpp:77-83
//   STDP: src/learning_rules/STDPWeightChange.cpp:43-76, STDPState.cpp:74-97,
//     include/spike/Interconnection.h:400-407
//   arrival after update at equal time: include/simulation/Event.h:37
//   input-spike delay cascade: src/spike/PropagatedSpike.cpp:60-100
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include "eb_device.cuh"
#include "eb_kernels.h"

namespace eb {

__device__ __forceinline__ bool arr_less(const Arrival &x, const Arrival &y) {
    return x.a < y.a || (x.a == y.a && x.spos < y.spos);
}

__device__ __forceinline__ float expt_net(const NetDev &N, float v) {
    if (v >= kExptMin && v <= kExptMax) {
        int pos = (int)((v - kExptMin) * N.expt_aux);
        return __ldg(N.exp_table + pos);
    }
    if (v > kExptMax) return (float)exp((double)v);
    return 0.0f;
}

// STDPWeightChange::ApplyPreSynapticSpike on the record r of a synapse at arrival
// time a (src/learning_rules/STDPWeightChange.cpp:43-56), in place.
__device__ __forceinline__ void stdp_pre_rec(const NetDev &N, SynRec &r, double a) {
    const float *rp = N.rule_par + r.rule * 6;
    float el = (float)(a - r.last);
    float pre = r.pre * expt_net(N, -el * rp[4]);
    float post = r.post * expt_net(N, -el * rp[5]);
    pre += 1.0f;
    float w = r.w;
    w += -rp[2] * post;
    const float mw = r.maxw;
    if (w > mw) w = mw; else if (w < 0.0f) w = 0.0f;
    r.w = w;
    r.pre = pre;
    r.post = post;
    r.last = a;
}

// The same on synapse tp: r is its state as loaded; the updated fields are stored.
__device__ __forceinline__ void stdp_pre(const NetDev &N, uint32_t tp, const SynRec &r, double a) {
    SynRec u = r;
    stdp_pre_rec(N, u, a);
    SynRec *s = N.syn + tp;
    s->w = u.w;
    s->pre = u.pre;
    s->post = u.post;
    s->last = u.last;
}

// STDPWeightChange::ApplyPostSynapticSpike on a synapse record for a spike of its
// target at time t (src/learning_rules/STDPWeightChange.cpp:58-76).
__device__ __forceinline__ void stdp_post(const NetDev &N, SynRec &r, double t) {
    const float *rp = N.rule_par + r.rule * 6;
    const float el = (float)(t - r.last);
    float pre = r.pre * expt_net(N, -el * rp[4]);
    float post = r.post * expt_net(N, -el * rp[5]);
    post += 1.0f;
    float w = r.w + rp[0] * pre;
    if (w > r.maxw) w = r.maxw; else if (w < 0.0f) w = 0.0f;
    r.w = w;
    r.pre = pre;
    r.post = post;
    r.last = t;
}

// Deferred post-synaptic STDP: apply to record r of a plastic synapse onto
// neuron i the target's spikes it has not seen (time > r.last), oldest first --
// the same updates in the same order as at each spike, only later.  Every spike
// of the ring is at most the arrival time being processed (spikes of this step
// are recorded after the fold), and at an equal time the spike came first.
// The ring holds the target's last kPostRing spike times (slot = spike number %
// kPostRing) and, when the population has one plastic rule, the trace decay
// factors of the interval ending at each spike; in global memory (RingGlobal) or
// staged in shared memory (RingSmem).
struct RingGlobal {
    const double *t;     // the neuron's kPostRing times
    const DecayPair *f;  // and factors
    __device__ double time(uint32_t slot) const { return t[slot]; }
    __device__ DecayPair fac(uint32_t slot) const { return f[slot]; }
};
struct RingSmem {
    const double *t;
    const DecayPair *f;
    __device__ double time(uint32_t slot) const { return t[slot]; }
    __device__ DecayPair fac(uint32_t slot) const { return f[slot]; }
};

// Apply to r the ring's spikes after r.last, oldest first, as stdp_post would one
// by one.  Spike times increase with the spike number, so the first pending one
// is found by bisection.  After the first, r.last is the previous spike, so each
// update's elapsed time -- and its two table lookups -- are the interval's: they
// come from the factor ring when r follows the ring's rule (rule >= 0).
template <class Ring>
__device__ __forceinline__ void apply_pending(const NetDev &N, const Ring &ring, uint32_t c, int rule, SynRec &r) {
    const uint32_t lim = c < (uint32_t)kPostRing ? c : (uint32_t)kPostRing;
    uint32_t lo = c - lim, hi = c;  // first spike number in [lo, hi) with time > r.last
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (ring.time(mid % kPostRing) > r.last) hi = mid;
        else lo = mid + 1;
    }
    if (lo == c) return;
    stdp_post(N, r, ring.time(lo % kPostRing));
    if (rule >= 0 && r.rule == rule) {
        const float a = N.rule_par[rule * 6];
        float w = r.w, pre = r.pre, post = r.post;
#pragma unroll 4
        for (uint32_t q = lo + 1; q < c; ++q) {
            const DecayPair f = ring.fac(q % kPostRing);
            pre = pre * f.pre;
            post = post * f.post;
            post += 1.0f;
            w = w + a * pre;
            if (w > r.maxw) w = r.maxw; else if (w < 0.0f) w = 0.0f;
        }
        r.w = w;
        r.pre = pre;
        r.post = post;
        r.last = ring.time((c - 1) % kPostRing);
    } else {
        for (uint32_t q = lo + 1; q < c; ++q) stdp_post(N, r, ring.time(q % kPostRing));
    }
}

__device__ __forceinline__ void apply_pending_post(const PopDev &P, const NetDev &N, int64_t i, SynRec &r) {
    const int64_t o = i * kPostRing;
    apply_pending(N, RingGlobal{P.post_t + o, P.post_f ? P.post_f + o : nullptr}, P.post_n[i],
                  P.post_f ? P.post_rule : -1, r);
}

__device__ __forceinline__ void prefetch_l1(const void *p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// State monitor (the reference's -logp): the state after step k and the spike
// flag of monitored neuron i, at row k % mon_steps.
__device__ __forceinline__ void monitor_state(const PopDev &P, const NetDev &N, int64_t k, int64_t i, const float *x,
                                              int nv, bool sp) {
    const int64_t o = (k % N.mon_steps) * N.mon_n + P.mon_base + i;
    float *d = N.mon_x + o * kMaxVars;
    for (int v = 0; v < nv; ++v) d[v] = x[v];
    N.mon_spk[o] = sp ? 1 : 0;
}

// A delivery of weight w (type ty) into monitored neuron i, folded by step k.
__device__ __forceinline__ void monitor_delivery(const PopDev &P, const NetDev &N, int64_t k, int64_t i,
                                                 const Arrival &v, int ty, float w) {
    const unsigned long long o = atomicAdd(N.mon_count, 1ull);
    if (o < (unsigned long long)N.mon_cap) {
        MonDelivery d;
        d.a = v.a;
        d.spos = v.spos;
        d.cell = (uint32_t)(P.mon_base + i);
        d.w = w;
        d.ty = ty;
        d.k = k;
        N.mon_del[o] = d;
    } else {
        atomicOr(N.flags, FLAG_MONITOR_OVERFLOW);
    }
}

// Monitor hooks: MON 0 compiles them out, 1 keeps them on, 2 asks P.mon at run
// time (the persistent kernel).  The hot kernels are instantiated with 0 and 1:
// a run-time test in the thread-per-neuron update cost the stiff HH network
// 70 % of its step.
template <int MON>
__device__ __forceinline__ bool mon_on(const PopDev &P) { return MON == 1 || (MON == 2 && P.mon != 0); }

template <int ND>
__device__ __forceinline__ void add_conductance(float *x, int ty, float w) {
    if (ty == 0) x[ND] += w;
    else if (ty == 1) x[ND + 1] += w;
    else x[ND + 2] += w;
}

// Apply one arrival at neuron i: g[type] += w (weight before plasticity), then
// STDP pre (after the target's deferred post updates, when it keeps a ring).
template <int ND, int MON = 2>
__device__ __forceinline__ void apply_arrival(const PopDev &P, const NetDev &N, int64_t k, int64_t i, const Arrival &r,
                                              float *x) {
    const uint32_t tp = r.tpos;
    SynRec s = N.syn[tp];
    if (s.rule >= 0 && P.post_t) apply_pending_post(P, N, i, s);
    add_conductance<ND>(x, s.stype, s.w);
    if (mon_on<MON>(P)) monitor_delivery(P, N, k, i, r, s.stype, s.w);
    if (s.rule >= 0) stdp_pre(N, tp, s, r.a);
}

// Record a spike of neuron i at step k for deferred post-synaptic STDP, with the
// decay factors of the interval from its previous spike (stdp_post's lookups for
// a synapse last updated at that spike).
__device__ __forceinline__ void note_post_spike(const PopDev &P, const NetDev &N, int64_t i, int64_t k) {
    const uint32_t c = P.post_n[i];
    const double t = N.tstep[k];
    const int64_t o = i * kPostRing + c % kPostRing;
    if (P.post_f && c > 0) {
        const float *rp = N.rule_par + P.post_rule * 6;
        const float el = (float)(t - P.post_t[i * kPostRing + (c - 1) % kPostRing]);
        P.post_f[o] = DecayPair{expt_net(N, -el * rp[4]), expt_net(N, -el * rp[5])};
    }
    P.post_t[o] = t;
    P.post_n[i] = c + 1;
}

__device__ __forceinline__ int64_t cur_step(const NetDev &N, int rel) { return *N.step + rel + 1; }

// ---------------------------------------------------------------- state io --
template <int KIND>
__device__ __forceinline__ void load_state(const PopDev &P, int64_t i, float *x) {
    constexpr int NV = Model<KIND>::NV;
#pragma unroll
    for (int v = 0; v < NV; ++v) x[v] = P.x[v] ? P.x[v][i] : 0.0f;
}
template <int KIND>
__device__ __forceinline__ void store_state(const PopDev &P, int64_t i, const float *x) {
    constexpr int NV = Model<KIND>::NV;
#pragma unroll
    for (int v = 0; v < NV; ++v) if (P.x[v]) P.x[v][i] = x[v];
}

// Per-neuron integer state next to the variables: LIF updates since the last
// spike, BDF history depth.
struct NeuronAux {
    int refr;
    int bst;
};

template <int KIND, int INTEG>
__device__ __forceinline__ NeuronAux load_aux(const PopDev &P, int64_t i) {
    NeuronAux a;
    a.refr = (KIND == KIND_LIF) ? P.refr[i] : -1;
    a.bst = (INTEG == INTEG_BDF) ? (int)P.bdf_state[i] : 0;
    return a;
}

template <int KIND, int INTEG>
__device__ __forceinline__ void store_aux(const PopDev &P, int64_t i, const NeuronAux &a) {
    if (KIND == KIND_LIF) P.refr[i] = a.refr;
    if (INTEG == INTEG_BDF) P.bdf_state[i] = (int8_t)a.bst;
}

// Advance one neuron (after its arrivals were folded); returns spike flag.  The
// integer state is updated in ax (store_aux writes it back).
template <int KIND, int INTEG, int EN = -1>
__device__ __forceinline__ bool advance_neuron(const PopDev &P, const NetDev &N, int64_t i, float *x, NeuronAux &ax) {
    constexpr int NV = Model<KIND>::NV;
    int refr = ax.refr;
    int bst = ax.bst;
    BdfRef H{P.bdf_D, P.bdf_P, P.n, i};
    const float prevV = x[0];
    if (!integrate<KIND, INTEG, EN>(P, x, refr, bst, H)) atomicOr(N.flags, FLAG_BDF_SINGULAR);
    if (KIND == KIND_LIF && refr >= 0) refr++;  // AddElapsedTime
    bool reset = false;
    const bool sp = spike_condition<KIND>(P, x, prevV, reset);
    if (sp) {
        if (KIND == KIND_LIF) refr = 0;  // NewFiredSpike
        if (reset && INTEG == INTEG_BDF) bst = 0;
    }
    if (x[0] != x[0]) {  // CheckValidIntegration: reset a neuron whose V became NaN
#pragma unroll
        for (int v = 0; v < NV; ++v) x[v] = P.init[v];
    }
    ax.refr = refr;
    ax.bst = bst;
    return sp;
}

__device__ __forceinline__ void record_trace(const PopDev &P, const NetDev &N, int64_t k, int64_t gi, const float *x, int nv) {
    if (!N.trace) return;
    int64_t c = gi - N.trace_first, s = k - N.trace_k0;
    if (c < 0 || c >= N.trace_n || s < 0 || s >= N.trace_steps) return;
    float *o = N.trace + (s * N.trace_n + c) * kMaxVars;
    for (int v = 0; v < nv; ++v) o[v] = x[v];
}

// Warp-aggregated append of the spiking lanes to the population spike list (when
// list is set: launches of one step, whose list the eager post-synaptic and
// separate fan-out kernels read) and to the recording buffer.
__device__ __forceinline__ void compact_spikes(const PopDev &P, const NetDev &N, int64_t k, int64_t i, bool sp,
                                               bool list = true) {
    const unsigned full = 0xffffffffu;
    const unsigned m = __ballot_sync(full, sp);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    const unsigned below = m & ((1u << lane) - 1u);
    uint32_t base = 0;
    unsigned long long rbase = 0;
    if (lane == leader) {
        if (list) base = atomicAdd(&P.spk_count[k & 1], (uint32_t)__popc(m));
        if (N.rec_buf) rbase = atomicAdd(N.rec_count, (unsigned long long)__popc(m));
    }
    base = __shfl_sync(full, base, leader);
    rbase = __shfl_sync(full, rbase, leader);
    if (sp) {
        const uint32_t o = base + __popc(below);
        if (!list) {
        } else if (o < (uint32_t)P.n) {
            P.spk[o] = (uint32_t)i;
        } else {
            atomicOr(N.flags, FLAG_SPIKELIST_OVERFLOW);
        }
        if (N.rec_buf) {
            const unsigned long long ro = rbase + __popc(below);
            if (ro < (unsigned long long)N.rec_cap)
                N.rec_buf[ro] = ((unsigned long long)k << 32) | (unsigned long long)(P.first + i);
            else atomicOr(N.flags, FLAG_RECORD_OVERFLOW);
        }
    }
}

// ------------------------------------------------------------ spike fan-out --
// Arrival step of a delivery at time a: the first update time strictly after a
// (never below k_lo).  The guess floor(a/dt)+1 is confirmed by two independent
// table reads in the common case; the loops only run when it is off by rounding.
__device__ __forceinline__ int64_t arrival_step(const NetDev &N, double a, int64_t k_lo, double inv_dt) {
    int64_t ka = (int64_t)(a * inv_dt) + 1;
    if (ka < k_lo) ka = k_lo;
    const double lo = N.tstep[ka - 1], hi = N.tstep[ka];
    if (hi > a && (lo <= a || ka == k_lo)) return ka;
    while (N.tstep[ka] <= a) ++ka;
    while (ka > k_lo && N.tstep[ka - 1] > a) --ka;
    return ka;
}

// Reserve a bucket entry of the target for step ka and store the arrival.
// Loads that do not depend on the reservation are issued before the atomic.
__device__ __forceinline__ void bucket_put(const NetDev &N, int64_t ka, double a, int64_t o) {
    const uint32_t tg = N.out_tgt[o];
    const uint32_t tp = N.out_tpos[o];
    const uint32_t capg = N.cap[tg];
    const int64_t base = N.cap_base[tg];
    const int slot = (int)(ka & (N.R - 1));
    const uint32_t idx = atomicAdd(N.cnt + (int64_t)slot * N.n_neurons + tg, 1u);
    if (idx < capg) {
        Arrival v;
        v.a = a;
        v.spos = (uint32_t)o;
        v.tpos = tp;
        N.rec[(int64_t)slot * N.cap_total + base + idx] = v;
    } else {
        atomicOr(N.flags, FLAG_BUCKET_OVERFLOW);
    }
}

// One spike of population P at step k (update time t_k): the block's threads
// cover the source's out-synapses (sorted by delay, then target).
// Fan-out of source neuron src's spike at step k: lanes lane, lane + width, ...
// of the caller's group take its out-synapses.
__device__ __forceinline__ void push_from(const PopDev &P, const NetDev &N, int64_t k, int64_t src, int lane, int width,
                                          double inv_dt) {
    const double tk = P.kind == KIND_POISSON ? N.tgen[k] : N.tstep[k];  // generators spike on their own grid
    const int64_t o0 = N.out_ptr[src], o1 = N.out_ptr[src + 1];
    for (int64_t o = o0 + lane; o < o1; o += width) {
        const double a = tk + (double)N.out_units[o] * 0.0001;
        bucket_put(N, arrival_step(N, a, k + 1, inv_dt), a, o);
    }
}

__device__ __forceinline__ void push_spike(const PopDev &P, const NetDev &N, int64_t k, int64_t s, double inv_dt) {
    push_from(P, N, k, P.first + P.spk[s], threadIdx.x, blockDim.x, inv_dt);
}

// Fan-out inside the update kernel (graph path): a spike at step k only reaches
// buckets of steps >= k+1, which no kernel of this step reads, so the spiking
// warp delivers it at once instead of a separate launch after the update.  The
// warp takes its spiking lanes one at a time, lanes over the out-synapses.
__device__ __forceinline__ void warp_push(const PopDev &P, const NetDev &N, int64_t k, int64_t i, bool sp,
                                          double inv_dt) {
    unsigned m = __ballot_sync(0xffffffffu, sp);
    const int lane = threadIdx.x & 31;
    while (m) {
        const int l = __ffs(m) - 1;
        m &= m - 1u;
        const int64_t src = P.first + __shfl_sync(0xffffffffu, i, l);
        push_from(P, N, k, src, lane, 32, inv_dt);
    }
}

// ----------------------------------------------------------- narrow update --
// One thread per neuron.  Arrivals of this step are sorted in registers
// (insertion sort; at most 16 in the fast path) and folded in order.
constexpr int kLocalSort = 16;
constexpr int kNarrowTile = 256;

// One step of neuron i (lanes with active unset only join the warp collectives);
// x and ax hold its state, loaded and stored by the caller.
template <int KIND, int INTEG, int EN = -1, int MON = 2>
__device__ __forceinline__ void narrow_step(const PopDev &P, const NetDev &N, int64_t k, int64_t i, bool active,
                                            float *x, NeuronAux &ax, bool list, double push_inv_dt) {
    constexpr int ND = Model<KIND>::ND;
    bool sp = false;
    uint32_t c = 0;
    if (active) {
        const int64_t gi = P.first + i;
        const int slot = (int)(k & (N.R - 1));
        uint32_t *cp = N.cnt + (int64_t)slot * N.n_neurons + gi;
        c = *cp;
        if (c) {
            *cp = 0;
            const uint32_t capg = N.cap[gi];
            if (c > capg) { atomicOr(N.flags, FLAG_BUCKET_OVERFLOW); c = capg; }
            Arrival *r = N.rec + (int64_t)slot * N.cap_total + N.cap_base[gi];
            if (c == 1) {
                apply_arrival<ND, MON>(P, N, k, i, r[0], x);
            } else if (c <= kLocalSort) {
                Arrival loc[kLocalSort];
                for (uint32_t a = 0; a < c; ++a) {
                    Arrival v = r[a];
                    int b = (int)a - 1;
                    while (b >= 0 && arr_less(v, loc[b])) { loc[b + 1] = loc[b]; --b; }
                    loc[b + 1] = v;
                }
                for (uint32_t a = 0; a < c; ++a) apply_arrival<ND, MON>(P, N, k, i, loc[a], x);
            } else {
                for (uint32_t a = 1; a < c; ++a) {  // in-place insertion sort (rare path)
                    Arrival v = r[a];
                    int b = (int)a - 1;
                    while (b >= 0 && arr_less(v, r[b])) { r[b + 1] = r[b]; --b; }
                    r[b + 1] = v;
                }
                for (uint32_t a = 0; a < c; ++a) apply_arrival<ND, MON>(P, N, k, i, r[a], x);
            }
        }
        sp = advance_neuron<KIND, INTEG, EN>(P, N, i, x, ax);
        record_trace(P, N, k, gi, x, Model<KIND>::NV);
        if (mon_on<MON>(P)) monitor_state(P, N, k, i, x, Model<KIND>::NV, sp);
        if (sp && P.post_t) note_post_spike(P, N, i, k);
    }
    // delivered-event counter: one atomic per warp
    if (__any_sync(0xffffffffu, c != 0)) {
        unsigned long long cw = c;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cw += __shfl_down_sync(0xffffffffu, cw, o);
        if ((threadIdx.x & 31) == 0 && cw) atomicAdd(P.events, cw);
    }
    compact_spikes(P, N, k, i, sp, list);
    if (push_inv_dt > 0.0) warp_push(P, N, k, i, sp, push_inv_dt);
}

template <int KIND, int INTEG>
__device__ __forceinline__ void update_narrow_tile(const PopDev &P, const NetDev &N, int64_t k, int64_t tile,
                                                   double push_inv_dt = 0.0) {
    const int64_t i = tile * kNarrowTile + threadIdx.x;
    const bool active = i < P.n;
    float x[kMaxVars];
    NeuronAux ax{-1, 0};
    if (active) {
        load_state<KIND>(P, i, x);
        ax = load_aux<KIND, INTEG>(P, i);
    }
    narrow_step<KIND, INTEG>(P, N, k, i, active, x, ax, true, push_inv_dt);
    if (active) {
        store_state<KIND>(P, i, x);
        store_aux<KIND, INTEG>(P, i, ax);
    }
}

// Steps k .. k+nsteps-1 of one tile, the state in registers between them.  Only a
// launch of one step keeps the population spike list (with several, no kernel
// reads it: fan-out is done here and post-synaptic STDP is deferred).
// push_inv_dt > 0: also fan out the spikes (1 / step, for arrival_step).
// HH under BDF holds the Newton state (Jacobian, inverse, history) in about 120
// registers, which leaves 2 blocks per SM; bounded to 3 blocks (80 registers, a
// 44-byte spill) a 100k-neuron population fits one wave and its steps take a
// quarter less time.  LIF and AdEx under the explicit methods are bounded to 6
// blocks (40 registers, spills of 8-12 bytes): a fifth more resident neurons than
// at the compiler's 48, so a 250k-neuron population takes 1.06 waves, not 1.32.
// EN >= 0: the population's enabled conductance types fixed at compile time.
constexpr int narrow_min_blocks(int kind, int integ) {
    return (kind == KIND_HH && integ == INTEG_BDF) ? 3 : (kind != KIND_HH && integ != INTEG_BDF) ? 6 : 0;
}

template <int KIND, int INTEG, int EN, int MON>
__global__ void __launch_bounds__(kNarrowTile, narrow_min_blocks(KIND, INTEG)) k_update_narrow(PopDev P, NetDev N, int rel, int nsteps,
                                                                double push_inv_dt) {
    const int64_t k = cur_step(N, rel);
    const bool list = nsteps == 1;
    if (list && blockIdx.x == 0 && threadIdx.x == 0) P.spk_count[(k + 1) & 1] = 0;
    const int64_t i = (int64_t)blockIdx.x * kNarrowTile + threadIdx.x;
    const bool active = i < P.n;
    float x[kMaxVars];
    NeuronAux ax{-1, 0};
    if (active) {
        load_state<KIND>(P, i, x);
        ax = load_aux<KIND, INTEG>(P, i);
    }
    for (int s = 0; s < nsteps; ++s) narrow_step<KIND, INTEG, EN, MON>(P, N, k + s, i, active, x, ax, list, push_inv_dt);
    if (active) {
        store_state<KIND>(P, i, x);
        store_aux<KIND, INTEG>(P, i, ax);
    }
}

// ------------------------------------------------------------- wide update --
// One block per neuron, for populations whose neurons receive many arrivals per
// step (e.g. Purkinje-like cells with 10^4-10^5 inputs).
//
// Up to kRankSort arrivals, every arrival finds its delivery position by counting
// the arrivals ordered before it -- (time, synapse order) compared as integers,
// since the bits of a non-negative double order like its value -- with all the
// block's threads sharing the comparisons.  Each arrival's synapse record is
// fetched while the positions are counted, its STDP pre-synaptic update applied
// in parallel (synapses are independent; a synapse that can arrive twice in one
// step -- only from input neurons -- forces the serial path) and its weight stored
// at its position; one thread per conductance then adds the weights in delivery
// order.  Up to kWideSmem arrivals: bitonic sort in shared memory; beyond, a
// serial insertion sort in global memory.
// A 512-arrival stage keeps a block at about 70 KB of shared memory, so three
// fit an SM (85 registers a thread): the wide population packs onto fewer SMs
// and leaves the others whole to the thread-per-neuron populations.
constexpr int kWideThreads = 256;
constexpr int kWideSmem = 1024;
constexpr int kRankSort = 256;
static_assert(kRankSort <= kWideThreads && kWideThreads <= kNarrowTile, "wide blocks rank with one thread per arrival");

// Steps of one launch (the runtime's window length).
constexpr int kMaxWindow = 8;

struct WideSmem {
    int spiked;                         // the block's neuron spiked this step (fused fan-out)
    int ring_ok;                        // ring, ring_f and ring_n hold the neuron's ring
    uint32_t ring_n;                    // post-synaptic spikes noted so far (deferred STDP)
    uint32_t next_c;                    // next step's arrival count (copied ahead)
    float g[3];                         // conductances handed to the per-type adders
    uint32_t wcnt[kMaxWindow];          // staged window: arrivals of each step
    uint32_t woff[kMaxWindow + 1];      // and their offsets (exclusive scan)
    unsigned long long kmin[kMaxWindow];  // smallest and largest time key of each step's arrivals
    unsigned long long kmax[kMaxWindow];
    int dup;                            // a synapse of the staged chunk delivers twice
    int next_s;                         // first step of the chunk's next round
    unsigned long long khi[kRankSort];  // arrival time keys
    uint32_t klo[kRankSort];            // synapse order
    uint32_t rank[kRankSort];           // delivery position
    double ring[kPostRing];             // the neuron's deferred post-synaptic spike times
    DecayPair ring_f[kPostRing];           // and the decay factors of their intervals
    Arrival next_rec[kRankSort];        // next step's first arrivals (copied ahead)
    Arrival sbuf[kWideSmem];
    float sw[kWideSmem];
    uint8_t sty[kWideSmem];
};

// Asynchronous global -> shared copies (cp.async): the block copies the next
// step's arrivals while it works on this one; the copies complete at
// cp_async_wait_all, before the next step's first barrier.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Copy step k's arrival count and its first n records (n <= the neuron's bucket
// capacity) of neuron gi into S.next_c / S.next_rec.  Only for a step whose
// bucket is final: a later step of the same launch (every delivery into it comes
// from steps before the launch, or from input fan-out that precedes it).
__device__ __forceinline__ void wide_prefetch(const NetDev &N, WideSmem &S, int64_t k, int64_t gi, int64_t rbase,
                                              int n) {
    const int slot = (int)(k & (N.R - 1));
    const Arrival *r = N.rec + (int64_t)slot * N.cap_total + rbase;
    for (int a = threadIdx.x; a < n; a += blockDim.x) cp_async16(&S.next_rec[a], r + a);
    if (threadIdx.x == 0) cp_async4(&S.next_c, N.cnt + (int64_t)slot * N.n_neurons + gi);
    cp_async_commit();
}

// Order-preserving integer key of an arrival time (-0 folded into +0).
__device__ __forceinline__ unsigned long long time_key(double a) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(a + 0.0);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// STDP pre hook for one arrival with every synapse load issued up front (they
// only depend on tp); returns the weight before the update through w_old.
__device__ __forceinline__ void stdp_pre_gather(const PopDev &P, const NetDev &N, int64_t i, uint32_t tp, double a,
                                                float &w_old, int &ty) {
    SynRec r = N.syn[tp];
    if (r.rule >= 0 && P.post_t) apply_pending_post(P, N, i, r);
    w_old = r.w;
    ty = r.stype;
    if (r.rule < 0) return;
    stdp_pre(N, tp, r, a);
}

// Add the c weights sw[] (types sty[]) to the conductances x[ND..ND+2] in order.
// Each conductance only sees its own type's weights, in order, so one thread per
// type (lane 0 of warps 0-2) adding its type's weights reproduces the interleaved
// sequential sum.  Thread 0 owns x; block-wide, with barriers.
template <int ND>
__device__ __forceinline__ void wide_fold(WideSmem &S, float *x, uint32_t c) {
    const int tid = threadIdx.x;
    if (tid == 0) { S.g[0] = x[ND]; S.g[1] = x[ND + 1]; S.g[2] = x[ND + 2]; }
    __syncthreads();
    const int T = tid >> 5;
    if ((tid & 31) == 0 && T < 3) {
        float g = S.g[T];
        uint32_t a = 0;
        for (; a + 8 <= c; a += 8) {
            float w[8];
            int t[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) { w[u] = S.sw[a + u]; t[u] = S.sty[a + u]; }
#pragma unroll
            for (int u = 0; u < 8; ++u) g = ((t[u] < 2 ? t[u] : 2) == T) ? g + w[u] : g;
        }
        for (; a < c; ++a) {
            const int t = S.sty[a];
            g = ((t < 2 ? t : 2) == T) ? g + S.sw[a] : g;
        }
        S.g[T] = g;
    }
    __syncthreads();
    if (tid == 0) { x[ND] = S.g[0]; x[ND + 1] = S.g[1]; x[ND + 2] = S.g[2]; }
}

// One step of wide neuron i by the whole block; thread 0 holds its state in x and
// ax (loaded and stored by the caller).
template <int KIND, int INTEG, int MON = 2, int EN = -1>
// pf_n: records of this step already copied to S.next_rec (with the count in
// S.next_c; 0: none), updated for the next step when has_next (the next step is
// in the same launch).
__device__ __forceinline__ void wide_step(const PopDev &P, const NetDev &N, int64_t k, int64_t i, WideSmem &S,
                                          float *x, NeuronAux &ax, bool list, double push_inv_dt, int &pf_n,
                                          bool has_next) {
    constexpr int ND = Model<KIND>::ND;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int slot = (int)(k & (N.R - 1));
    const int64_t gi = P.first + i;
    if (pf_n > 0) cp_async_wait_all();
    __syncthreads();  // the block's previous step is done with S; copied arrivals visible
    // every load that does not depend on another goes out first
    uint32_t *cp = N.cnt + (int64_t)slot * N.n_neurons + gi;
    uint32_t c = pf_n > 0 ? S.next_c : *cp;
    const uint32_t capg = N.cap[gi];
    const int64_t rbase = N.cap_base[gi];
    int next_n = 0;
    // after a barrier that follows every thread's read of S.next_*: copy the next
    // step's count and about as many records as this step had
    auto issue_next = [&]() {
        if (!has_next) return;
        const uint32_t guess = ((c + c / 2 + 32) + 31) / 32 * 32;
        next_n = (int)min(min(guess, capg), (uint32_t)kRankSort);
        wide_prefetch(N, S, k + 1, gi, rbase, next_n);
    };
    if (c) {
        if (c > capg) { if (tid == 0) atomicOr(N.flags, FLAG_BUCKET_OVERFLOW); c = capg; }
        Arrival *r = N.rec + (int64_t)slot * N.cap_total + rbase;
        if (c <= (uint32_t)kRankSort) {
            const bool own = tid < (int)c;
            const bool ring = P.post_t != nullptr && !P.may_repeat;
            Arrival v;
            SynRec rec;
            if (own) {
                v = tid < pf_n ? S.next_rec[tid] : r[tid];
                if (!P.may_repeat) rec = N.syn[v.tpos];  // in flight while the positions are counted
                S.khi[tid] = time_key(v.a);
                S.klo[tid] = v.spos;
                S.rank[tid] = 0;
            }
            if (ring && !S.ring_ok) {  // the neuron's deferred post-synaptic spikes (slots past the count are unused)
                for (int q = tid; q < kPostRing; q += nt) {
                    S.ring[q] = P.post_t[i * kPostRing + q];
                    if (P.post_f) S.ring_f[q] = P.post_f[i * kPostRing + q];
                }
                if (tid == nt - 1) S.ring_n = P.post_n[i];
            }
            if (tid == 32) prefetch_l1(N.rule_par);
            __syncthreads();
            if (tid == 0) {
                *cp = 0;
                if (ring) S.ring_ok = 1;
            }
            issue_next();
            // position = arrivals before this one in (time, synapse order, bucket index)
            // order; per threads share each arrival's comparisons
            const int per = nt / (int)c;
            if (tid < per * (int)c) {
                const int e = tid % (int)c, s = tid / (int)c;
                const int b0 = s * (int)c / per, b1 = (s + 1) * (int)c / per;
                const unsigned long long kh = S.khi[e];
                const uint32_t kl = S.klo[e];
                uint32_t n = 0;
#pragma unroll 4
                for (int b = b0; b < b1; ++b) {
                    const unsigned long long uh = S.khi[b];
                    const uint32_t ul = S.klo[b];
                    n += (uh < kh || (uh == kh && (ul < kl || (ul == kl && b < e)))) ? 1u : 0u;
                }
                if (per == 1) S.rank[e] = n;
                else if (n) atomicAdd(&S.rank[e], n);
            }
            __syncthreads();
            if (P.may_repeat) {
                if (own) S.sbuf[S.rank[tid]] = v;
                __syncthreads();
                if (tid == 0)
                    for (uint32_t a = 0; a < c; ++a) apply_arrival<ND, MON>(P, N, k, i, S.sbuf[a], x);
            } else {
                if (own) {
                    if (rec.rule >= 0) {
                        if (ring) apply_pending(N, RingSmem{S.ring, S.ring_f}, S.ring_n, P.post_f ? P.post_rule : -1, rec);
                        S.sw[S.rank[tid]] = rec.w;
                        stdp_pre(N, v.tpos, rec, v.a);
                    } else {
                        S.sw[S.rank[tid]] = rec.w;
                    }
                    S.sty[S.rank[tid]] = rec.stype;
                    if (mon_on<MON>(P)) monitor_delivery(P, N, k, i, v, rec.stype, S.sw[S.rank[tid]]);
                }
                wide_fold<ND>(S, x, c);
            }
        } else if (c <= (uint32_t)kWideSmem) {
            int n2 = 1;
            while (n2 < (int)c) n2 <<= 1;
            for (int a = tid; a < n2; a += nt) {
                if (a < (int)c) S.sbuf[a] = r[a];
                else { S.sbuf[a].a = __longlong_as_double(0x7ff0000000000000LL); S.sbuf[a].spos = 0xffffffffu; S.sbuf[a].tpos = 0; }
            }
            __syncthreads();
            if (tid == 0) *cp = 0;
            issue_next();
            for (int size = 2; size <= n2; size <<= 1)
                for (int stride = size >> 1; stride > 0; stride >>= 1) {
                    for (int a = tid; a < n2; a += nt) {
                        const int b = a ^ stride;
                        if (b > a) {
                            const bool up = ((a & size) == 0);
                            const Arrival ea = S.sbuf[a], eb = S.sbuf[b];
                            if (up ? arr_less(eb, ea) : arr_less(ea, eb)) { S.sbuf[a] = eb; S.sbuf[b] = ea; }
                        }
                    }
                    __syncthreads();
                }
            if (P.may_repeat) {
                if (tid == 0)
                    for (uint32_t a = 0; a < c; ++a) apply_arrival<ND, MON>(P, N, k, i, S.sbuf[a], x);
            } else {
                for (int a = tid; a < (int)c; a += nt) {
                    const Arrival v = S.sbuf[a];
                    float w_old;
                    int ty;
                    stdp_pre_gather(P, N, i, v.tpos, v.a, w_old, ty);
                    S.sw[a] = w_old;
                    S.sty[a] = (uint8_t)ty;
                    if (mon_on<MON>(P)) monitor_delivery(P, N, k, i, v, ty, w_old);
                }
                __syncthreads();
                wide_fold<ND>(S, x, c);
            }
        } else {
            __syncthreads();  // every thread has read the count before it is cleared
            issue_next();
            if (tid == 0) {
                *cp = 0;
                for (uint32_t a = 1; a < c; ++a) {  // rare: insertion sort in global memory
                    Arrival v = r[a];
                    int b = (int)a - 1;
                    while (b >= 0 && arr_less(v, r[b])) { r[b + 1] = r[b]; --b; }
                    r[b + 1] = v;
                }
                for (uint32_t a = 0; a < c; ++a) apply_arrival<ND, MON>(P, N, k, i, r[a], x);
            }
        }
        if (tid == 0) atomicAdd(P.events, (unsigned long long)c);
    } else if (has_next) {
        __syncthreads();  // every thread has read S.next_c
        issue_next();
    }
    if (tid == 0) {
        const bool sp = advance_neuron<KIND, INTEG, EN>(P, N, i, x, ax);
        S.spiked = sp ? 1 : 0;
        if (sp && P.post_t) {
            note_post_spike(P, N, i, k);
            if (S.ring_ok) {  // keep the staged ring current
                const uint32_t n1 = P.post_n[i], q = (n1 - 1) % kPostRing;
                S.ring_n = n1;
                S.ring[q] = P.post_t[i * kPostRing + q];
                if (P.post_f) S.ring_f[q] = P.post_f[i * kPostRing + q];
            }
        }
        record_trace(P, N, k, gi, x, Model<KIND>::NV);
        if (mon_on<MON>(P)) monitor_state(P, N, k, i, x, Model<KIND>::NV, sp);
        if (sp) {
            if (list) {
                const uint32_t o = atomicAdd(&P.spk_count[k & 1], 1u);
                if (o < (uint32_t)P.n) P.spk[o] = (uint32_t)i;
                else atomicOr(N.flags, FLAG_SPIKELIST_OVERFLOW);
            }
            if (N.rec_buf) {
                const unsigned long long ro = atomicAdd(N.rec_count, 1ull);
                if (ro < (unsigned long long)N.rec_cap)
                    N.rec_buf[ro] = ((unsigned long long)k << 32) | (unsigned long long)gi;
                else atomicOr(N.flags, FLAG_RECORD_OVERFLOW);
            }
        }
    }
    __syncthreads();
    if (push_inv_dt > 0.0 && S.spiked) push_from(P, N, k, gi, tid, blockDim.x, push_inv_dt);
    pf_n = next_n;
}

template <int KIND, int INTEG>
__device__ __forceinline__ void update_wide_neuron(const PopDev &P, const NetDev &N, int64_t k, int64_t i, WideSmem &S,
                                                   double push_inv_dt = 0.0) {
    float x[kMaxVars];
    NeuronAux ax{-1, 0};
    if (threadIdx.x == 0) {
        load_state<KIND>(P, i, x);
        ax = load_aux<KIND, INTEG>(P, i);
        S.ring_ok = 0;
    }
    int pf_n = 0;
    wide_step<KIND, INTEG>(P, N, k, i, S, x, ax, true, push_inv_dt, pf_n, false);
    if (threadIdx.x == 0) {
        store_state<KIND>(P, i, x);
        store_aux<KIND, INTEG>(P, i, ax);
    }
}

// ------------------------------------------------------ staged wide window --
// A launch's window of steps for one wide neuron with every delivery of the
// window taken in at once.  All buckets of the window's steps are final when the
// launch starts, so the block stages the arrivals of as many consecutive steps as
// fit in shared memory (a chunk) and every arrival's delivery position within its
// step, in parallel: a few dependent global round trips per chunk instead of per
// step.  When every synapse of the chunk delivers once (the usual case), the
// chunk's steps run in rounds: the whole block computes, in parallel, every
// remaining arrival's synapse update -- deferred post-synaptic catch-up on the
// target's spikes so far and the delivered weight at its position -- then warp 0
// runs the steps in order (ordered sums, integration, spike, fan-out) until the
// neuron spikes.  A spike adds one update to the catch-up of the later arrivals:
// the next round applies it to their staged records.  The STDP pre updates are
// applied as the chunk writes its records back.  A chunk in which a synapse
// delivers on two steps runs its steps serially on warp 0 over one staged record
// per synapse; a step with more arrivals than the stage holds runs on the
// per-step path (wide_step).
constexpr int kStage = 512;           // arrivals of one chunk
constexpr int kStageHashBits = 10;    // open-addressing table of the chunk's synapses
constexpr int kStageHash = 1 << kStageHashBits;
constexpr uint32_t kHashEmpty = 0xffffffffu;
static_assert(kStage <= kWideSmem, "a staged chunk's weights fit the fold buffer");

struct StageSmem {
    Arrival arr[kStage];               // the chunk's arrivals, step by step in bucket order
    SynRec rec[kStage];                // updated synapse records (serial path: at the owning arrival)
    unsigned long long key[kStage];    // order-preserving integer key of each arrival time
    uint32_t hkey[kStageHash];         // tpos of the synapse claiming a slot
    uint16_t hval[kStageHash];         // its owning arrival
    uint16_t own[kStage];              // per arrival: the arrival whose staged record it uses
    uint16_t rank[kStage];             // per arrival: delivery position within its step
};

__host__ __device__ constexpr size_t stage_smem_bytes() { return sizeof(StageSmem); }

__device__ __forceinline__ int stage_step_of(const WideSmem &S, int s0, uint32_t g) {
    int s = s0;
    while (S.woff[s + 1] <= g) ++s;
    return s;
}

// Sum of the c weights sw[o0..o0+c) onto g in order, loads issued 8 at a time.
__device__ __forceinline__ float ordered_sum1(const WideSmem &S, uint32_t o0, uint32_t c, float g) {
    uint32_t q = 0;
    for (; q + 8 <= c; q += 8) {
        float w[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) w[u] = S.sw[o0 + q + u];
#pragma unroll
        for (int u = 0; u < 8; ++u) g += w[u];
    }
    for (; q < c; ++q) g += S.sw[o0 + q];
    return g;
}

// Add the c weights sw[o0..o0+c) (types sty[]) to the conductances x[ND..ND+2] in
// order: each conductance sees its own type's weights in delivery order, as the
// reference's successive additions.  A population with one enabled conductance
// receives weights of that type only.
template <int ND>
__device__ __forceinline__ void ordered_sum(const WideSmem &S, uint32_t o0, uint32_t c, float *x, int en) {
    if (en == 1) { x[ND] = ordered_sum1(S, o0, c, x[ND]); return; }
    if (en == 2) { x[ND + 1] = ordered_sum1(S, o0, c, x[ND + 1]); return; }
    if (en == 4) { x[ND + 2] = ordered_sum1(S, o0, c, x[ND + 2]); return; }
    float g0 = x[ND], g1 = x[ND + 1], g2 = x[ND + 2];
    uint32_t q = 0;
    for (; q + 8 <= c; q += 8) {
        float w[8];
        int t[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) { w[u] = S.sw[o0 + q + u]; t[u] = S.sty[o0 + q + u]; }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (t[u] == 0) g0 += w[u];
            else if (t[u] == 1) g1 += w[u];
            else g2 += w[u];
        }
    }
    for (; q < c; ++q) {
        const int t = S.sty[o0 + q];
        const float w = S.sw[o0 + q];
        if (t == 0) g0 += w;
        else if (t == 1) g1 += w;
        else g2 += w;
    }
    x[ND] = g0;
    x[ND + 1] = g1;
    x[ND + 2] = g2;
}

// Lane 0 of warp 0, after step ks's conductances are in x: integrate, test the
// spike, note it for deferred post-synaptic STDP (global ring and its staged
// copy), trace, spike list and recording.  Returns the spike flag.
template <int KIND, int INTEG, int MON = 2, int EN = -1>
__device__ __forceinline__ int wide_advance(const PopDev &P, const NetDev &N, int64_t ks, int64_t i, WideSmem &S,
                                            float *x, NeuronAux &ax, bool list, bool ring) {
    const int64_t gi = P.first + i;
    const int sp = advance_neuron<KIND, INTEG, EN>(P, N, i, x, ax) ? 1 : 0;
    if (sp && ring) {
        note_post_spike(P, N, i, ks);
        const uint32_t n1 = P.post_n[i], q = (n1 - 1) % kPostRing;
        S.ring_n = n1;
        S.ring[q] = P.post_t[i * kPostRing + q];
        if (P.post_f) S.ring_f[q] = P.post_f[i * kPostRing + q];
    }
    record_trace(P, N, ks, gi, x, Model<KIND>::NV);
    if (mon_on<MON>(P)) monitor_state(P, N, ks, i, x, Model<KIND>::NV, sp != 0);
    if (sp) {
        if (list) {
            const uint32_t o = atomicAdd(&P.spk_count[ks & 1], 1u);
            if (o < (uint32_t)P.n) P.spk[o] = (uint32_t)i;
            else atomicOr(N.flags, FLAG_SPIKELIST_OVERFLOW);
        }
        if (N.rec_buf) {
            const unsigned long long ro = atomicAdd(N.rec_count, 1ull);
            if (ro < (unsigned long long)N.rec_cap)
                N.rec_buf[ro] = ((unsigned long long)ks << 32) | (unsigned long long)gi;
            else atomicOr(N.flags, FLAG_RECORD_OVERFLOW);
        }
    }
    return sp;
}

template <int KIND, int INTEG, int MON = 2, int EN = -1>
__device__ __forceinline__ void wide_window(const PopDev &P, const NetDev &N, int64_t k, int64_t i, WideSmem &S,
                                            StageSmem &G, float *x, NeuronAux &ax, int nsteps, bool list,
                                            double push_inv_dt) {
    constexpr int ND = Model<KIND>::ND;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    const int64_t gi = P.first + i;
    const uint32_t capg = N.cap[gi];
    const int64_t rbase = N.cap_base[gi];
    const bool ring = P.post_t != nullptr;
    const int prule = P.post_f ? P.post_rule : -1;
    if (tid < nsteps) {
        uint32_t c = N.cnt[(int64_t)((k + tid) & (N.R - 1)) * N.n_neurons + gi];
        if (c > capg) { atomicOr(N.flags, FLAG_BUCKET_OVERFLOW); c = capg; }
        S.wcnt[tid] = c;
    }
    if (ring && !S.ring_ok) {
        for (int q = tid; q < kPostRing; q += nt) {
            S.ring[q] = P.post_t[i * kPostRing + q];
            if (P.post_f) S.ring_f[q] = P.post_f[i * kPostRing + q];
        }
        if (tid == nt - 1) S.ring_n = P.post_n[i];
    }
    __syncthreads();
    if (tid == 0) {
        S.woff[0] = 0;
        for (int s = 0; s < nsteps; ++s) S.woff[s + 1] = S.woff[s] + S.wcnt[s];
        if (ring) S.ring_ok = 1;
    }
    if (tid < nsteps) {
        S.kmin[tid] = ~0ull;
        S.kmax[tid] = 0ull;
    }
    __syncthreads();
    int s0 = 0;
    while (s0 < nsteps) {
        int s1 = s0;
        while (s1 < nsteps && S.woff[s1 + 1] - S.woff[s0] <= (uint32_t)kStage) ++s1;
        if (s1 == s0) {  // this step alone overflows the stage
            int pf_n = 0;
            wide_step<KIND, INTEG, MON, EN>(P, N, k + s0, i, S, x, ax, list, push_inv_dt, pf_n, false);
            __syncthreads();
            ++s0;
            continue;
        }
        const uint32_t a0 = S.woff[s0], T = S.woff[s1] - a0;
        for (uint32_t a = tid; a < T; a += nt) {
            const int s = stage_step_of(S, s0, a0 + a);
            const int slot = (int)((k + s) & (N.R - 1));
            const Arrival v = N.rec[(int64_t)slot * N.cap_total + rbase + (a0 + a - S.woff[s])];
            G.arr[a] = v;
            const unsigned long long key = time_key(v.a);
            G.key[a] = key;
            atomicMin(&S.kmin[s], key);
            atomicMax(&S.kmax[s], key);
            // the synapse record, copied while the chunk is hashed and ranked
            const SynRec *src = N.syn + v.tpos;
            cp_async16(&G.rec[a], src);
            cp_async16(reinterpret_cast<unsigned char *>(&G.rec[a]) + 16, reinterpret_cast<const unsigned char *>(src) + 16);
        }
        cp_async_commit();
        for (int h = tid; h < kStageHash; h += nt) G.hkey[h] = kHashEmpty;
        if (tid == 0) S.dup = 0;
        __syncthreads();
        if (tid >= s0 && tid < s1) N.cnt[(int64_t)((k + tid) & (N.R - 1)) * N.n_neurons + gi] = 0;
        if (tid == 0 && T) atomicAdd(P.events, (unsigned long long)T);
        // synapses of the chunk: the arrival that claims a synapse's slot owns it
        for (uint32_t a = tid; a < T; a += nt) {
            const uint32_t tp = G.arr[a].tpos;
            uint32_t h = (tp * 2654435761u) >> (32 - kStageHashBits);
            for (;;) {
                const uint32_t prev = atomicCAS(&G.hkey[h], kHashEmpty, tp);
                if (prev == kHashEmpty) { G.hval[h] = (uint16_t)a; break; }
                if (prev == tp) { S.dup = 1; break; }
                h = (h + 1) & (kStageHash - 1);
            }
            G.own[a] = (uint16_t)h;
            // a step whose arrival times span less than 2^32 key units ranks on
            // one 64-bit key: (time key - the step's smallest) << 32 | synapse order
            const int s = stage_step_of(S, s0, a0 + a);
            const unsigned long long k0 = S.kmin[s];
            if (S.kmax[s] - k0 <= 0xffffffffull) G.key[a] = ((G.key[a] - k0) << 32) | G.arr[a].spos;
        }
        __syncthreads();
        const bool dup = S.dup != 0;
        if (dup) cp_async_wait_all();  // the serial path below rewrites staged records
        for (uint32_t a = tid; a < T; a += nt) {
            const uint32_t o = G.hval[G.own[a]];
            G.own[a] = (uint16_t)o;
            if (dup && o == a) {  // serial path: one staged record per synapse, caught up to the chunk
                SynRec r = N.syn[G.arr[a].tpos];
                if (r.rule >= 0 && ring) apply_pending(N, RingSmem{S.ring, S.ring_f}, S.ring_n, prule, r);
                G.rec[a] = r;
            }
            // delivery position: arrivals of the same step before it in (time,
            // synapse order) order -- a step's synapses are distinct here -- on the
            // integer keys of the times
            const int s = stage_step_of(S, s0, a0 + a);
            const uint32_t b0 = S.woff[s] - a0, b1 = S.woff[s + 1] - a0;
            const unsigned long long ka = G.key[a];
            uint32_t r = 0;
            if (S.kmax[s] - S.kmin[s] <= 0xffffffffull) {
#pragma unroll 8
                for (uint32_t b = b0; b < b1; ++b) r += G.key[b] < ka ? 1u : 0u;
            } else {
                const uint32_t pa = G.arr[a].spos;
#pragma unroll 4
                for (uint32_t b = b0; b < b1; ++b) {
                    const unsigned long long kb = G.key[b];
                    r += (kb < ka || (kb == ka && G.arr[b].spos < pa)) ? 1u : 0u;
                }
            }
            G.rank[a] = (uint16_t)r;
        }
        cp_async_wait_all();
        __syncthreads();
        if (!dup) {
            int s = s0;
            while (s < s1) {
                for (uint32_t a = S.woff[s] - a0 + tid; a < T; a += nt) {
                    // the staged record, caught up to the spikes of the earlier rounds:
                    // this round adds the spike that ended the last one (the same
                    // updates in the same order as one catch-up from the original);
                    // the pre-synaptic update is applied at the write-back
                    SynRec r = G.rec[a];
                    if (r.rule >= 0 && ring) apply_pending(N, RingSmem{S.ring, S.ring_f}, S.ring_n, prule, r);
                    const uint32_t pos = S.woff[stage_step_of(S, s0, a0 + a)] - a0 + G.rank[a];
                    S.sw[pos] = r.w;
                    S.sty[pos] = r.stype;
                    if (mon_on<MON>(P)) monitor_delivery(P, N, k + stage_step_of(S, s0, a0 + a), i, G.arr[a], r.stype, r.w);
                    G.rec[a] = r;
                }
                __syncthreads();
                if (tid < 32) {
                    int next = s1;
                    for (int j = s; j < s1; ++j) {
                        int sp = 0;
                        if (lane == 0) {
                            ordered_sum<ND>(S, S.woff[j] - a0, S.wcnt[j], x, en_mask<EN>(P));
                            sp = wide_advance<KIND, INTEG, MON, EN>(P, N, k + j, i, S, x, ax, list, ring);
                        }
                        sp = __shfl_sync(0xffffffffu, sp, 0);
                        if (sp && push_inv_dt > 0.0) push_from(P, N, k + j, gi, lane, 32, push_inv_dt);
                        if (sp && ring) { next = j + 1; break; }
                    }
                    if (lane == 0) S.next_s = next;
                }
                __syncthreads();
                s = S.next_s;
            }
        } else if (tid < 32) {
            for (int s = s0; s < s1; ++s) {
                const int64_t ks = k + s;
                const uint32_t o0 = S.woff[s] - a0, c = S.wcnt[s];
                for (uint32_t a = o0 + lane; a < o0 + c; a += 32) {
                    SynRec &sr = G.rec[G.own[a]];
                    SynRec r = sr;
                    if (r.rule >= 0 && ring) apply_pending(N, RingSmem{S.ring, S.ring_f}, S.ring_n, prule, r);
                    S.sw[o0 + G.rank[a]] = r.w;
                    S.sty[o0 + G.rank[a]] = r.stype;
                    if (mon_on<MON>(P)) monitor_delivery(P, N, ks, i, G.arr[a], r.stype, r.w);
                    if (r.rule >= 0) {
                        stdp_pre_rec(N, r, G.arr[a].a);
                        sr = r;
                    }
                }
                __syncwarp();
                int sp = 0;
                if (lane == 0) {
                    ordered_sum<ND>(S, o0, c, x, en_mask<EN>(P));
                    sp = wide_advance<KIND, INTEG, MON, EN>(P, N, ks, i, S, x, ax, list, ring);
                }
                sp = __shfl_sync(0xffffffffu, sp, 0);
                if (sp && push_inv_dt > 0.0) push_from(P, N, ks, gi, lane, 32, push_inv_dt);
                __syncwarp();
            }
        }
        __syncthreads();
        for (uint32_t a = tid; a < T; a += nt) {
            if (G.own[a] != a || G.rec[a].rule < 0) continue;
            SynRec r = G.rec[a];
            if (!dup) stdp_pre_rec(N, r, G.arr[a].a);  // the serial path applied it already
            SynRec *d = N.syn + G.arr[a].tpos;
            d->w = r.w;
            d->pre = r.pre;
            d->post = r.post;
            d->last = r.last;
        }
        __syncthreads();
        s0 = s1;
    }
}

// Steps k .. k+nsteps-1 of the block's neurons (spike list as in k_update_narrow).
// Populations whose synapses cannot deliver twice in one step take the staged
// window; the others run step by step.  At most 72 registers a thread: three
// blocks per SM leave room for one thread-per-neuron block of 256 at 40.
template <int KIND, int INTEG, int MON, int EN>
__global__ void __maxnreg__(72) k_update_wide(PopDev P, NetDev N, int rel, int nsteps,
                                                                 double push_inv_dt) {
    __shared__ WideSmem S;
    extern __shared__ __align__(32) unsigned char stage_raw[];
    StageSmem &G = *reinterpret_cast<StageSmem *>(stage_raw);
    const int64_t k = cur_step(N, rel);
    const bool list = nsteps == 1;
    if (list && blockIdx.x == 0 && threadIdx.x == 0) P.spk_count[(k + 1) & 1] = 0;
    for (int64_t i = blockIdx.x; i < P.n; i += gridDim.x) {
        float x[kMaxVars];
        NeuronAux ax{-1, 0};
        if (threadIdx.x == 0) {
            load_state<KIND>(P, i, x);
            ax = load_aux<KIND, INTEG>(P, i);
            S.ring_ok = 0;
        }
        __syncthreads();  // S.ring_ok reset before any thread reads it
        if (!P.may_repeat && nsteps <= kMaxWindow) {
            wide_window<KIND, INTEG, MON, EN>(P, N, k, i, S, G, x, ax, nsteps, list, push_inv_dt);
        } else {
            int pf_n = 0;
            for (int s = 0; s < nsteps; ++s)
                wide_step<KIND, INTEG, MON, EN>(P, N, k + s, i, S, x, ax, list, push_inv_dt, pf_n, s + 1 < nsteps);
        }
        if (threadIdx.x == 0) {
            store_state<KIND>(P, i, x);
            store_aux<KIND, INTEG>(P, i, ax);
        }
        __syncthreads();  // the next neuron's staging reuses S
    }
}

// PoissonGeneratorDeviceVector::UpdateState (src/neuron_model/PoissonGeneratorDeviceVector.cpp:56-70):
// a generator with frequency > 0 draws frand() from its own RandomGenerator --
// x <- (x * 1103515245 + 12345) & 0x7fffffff, frand = (float)x / MAX_RAND
// (include/simulation/RandomGenerator.h:91-107) -- and fires when
// frequency * step > frand.  The low 31 bits of the product only depend on its low
// 32 bits, so 32-bit arithmetic gives the reference's sequence.
__global__ void __launch_bounds__(256) k_update_poisson(PopDev P, NetDev N, int rel, int nsteps, double push_inv_dt) {
    const int64_t k0 = cur_step(N, rel);
    const bool list = nsteps == 1;
    if (list && blockIdx.x == 0 && threadIdx.x == 0) P.spk_count[(k0 + 1) & 1] = 0;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const double thr = i < P.n ? P.pthr[i] : 0.0;
    uint32_t x = i < P.n ? P.lcg[i] : 0u;
    for (int s = 0; s < nsteps; ++s) {
        const int64_t k = k0 + s;
        bool sp = false;
        if (thr > 0.0) {
            x = (x * 1103515245u + 12345u) & 0x7fffffffu;
            const float r = (float)x / (float)2147483647;
            sp = thr > (double)r;
        }
        compact_spikes(P, N, k, i, sp, list);
        if (push_inv_dt > 0.0) warp_push(P, N, k, i, sp, push_inv_dt);
    }
    if (i < P.n && thr > 0.0) P.lcg[i] = x;
}

// ------------------------------------------------------------ spike fan-out --
// One input-neuron spike q emitted in [t_{k-1}, t_k).  A source with several
// distinct delays delivers group j+1 at (a_j - d_j) + d_{j+1}, as the reference's
// PropagatedSpike chain does.
__device__ __forceinline__ void input_spike(const NetDev &N, int64_t k, int64_t q, double inv_dt) {
    const int64_t src = N.in_cell[q];
    const double tin = N.in_time[q];
    const int64_t o0 = N.out_ptr[src], o1 = N.out_ptr[src + 1];
    const int64_t g0 = N.grp_ptr[src], g1 = N.grp_ptr[src + 1];
    for (int64_t o = o0 + threadIdx.x; o < o1; o += blockDim.x) {
        const uint16_t u = N.out_units[o];
        double a = tin + (double)N.grp_units[g0] * 0.0001;
        for (int64_t g = g0 + 1; g < g1 && N.grp_units[g - 1] != u; ++g)
            a = a - (double)N.grp_units[g - 1] * 0.0001 + (double)N.grp_units[g] * 0.0001;
        bucket_put(N, arrival_step(N, a, k, inv_dt), a, o);
    }
}

// Post-synaptic STDP (STDPWeightChange::ApplyPostSynapticSpike) for work item
// (spike s, chunk ch of blockDim plastic inputs): one synapse per thread.
__device__ __forceinline__ void post_item(const PopDev &P, const NetDev &N, int64_t k, int64_t s, int64_t ch) {
    const double tk = N.tstep[k];
    const int64_t t = P.first + P.spk[s];
    const int64_t tp = N.in_ptr[t] + ch * blockDim.x + threadIdx.x;
    if (tp >= N.plastic_end[t]) return;
    const SynRec r = N.syn[tp];
    const float *rp = N.rule_par + r.rule * 6;
    float pre = r.pre, post = r.post, w = r.w;
    const float el = (float)(tk - r.last);
    pre *= expt_net(N, -el * rp[4]);
    post *= expt_net(N, -el * rp[5]);
    post += 1.0f;
    w += rp[0] * pre;
    if (w > r.maxw) w = r.maxw; else if (w < 0.0f) w = 0.0f;
    SynRec *o = N.syn + tp;
    o->w = w;
    o->pre = pre;
    o->post = post;
    o->last = tk;
}

__global__ void __launch_bounds__(256) k_push(PopDev P, NetDev N, int rel, double inv_dt) {
    const int64_t k = cur_step(N, rel);
    const uint32_t ns = min(P.spk_count[k & 1], (uint32_t)P.n);
    for (int64_t s = blockIdx.x; s < ns; s += gridDim.x) push_spike(P, N, k, s, inv_dt);
}

// Input spikes of steps k .. k+nsteps-1.  Their deliveries are independent, so the
// window's inputs -- one contiguous range of the staged list -- are spread over
// the blocks at once; each block finds its spike's step among the window's
// input ranges.
__global__ void __launch_bounds__(256) k_input_push(NetDev N, int rel, int nsteps, double inv_dt) {
    const int64_t k0 = cur_step(N, rel);
    const int64_t q0 = N.in_start[k0], q1 = N.in_start[k0 + nsteps];
    for (int64_t q = q0 + blockIdx.x; q < q1; q += gridDim.x) {
        int64_t k = k0;
        while (k + 1 < k0 + nsteps && N.in_start[k + 1] <= q) ++k;
        input_spike(N, k, q, inv_dt);
    }
}

__global__ void __launch_bounds__(256) k_post_stdp(PopDev P, NetDev N, int rel, int max_chunks) {
    const int64_t k = cur_step(N, rel);
    const uint32_t ns = min(P.spk_count[k & 1], (uint32_t)P.n);
    const int64_t items = (int64_t)ns * max_chunks;
    for (int64_t item = blockIdx.x; item < items; item += gridDim.x) post_item(P, N, k, item / max_chunks, item % max_chunks);
}

// -------------------------------------------------------- persistent kernel --
// All phases of K consecutive steps in one cooperative launch.  Per step:
//   [inputs]  input-spike fan-out (its own phase only when an input delivery can
//             reach the step being updated)
//   phase A   neuron updates of every population (+ input fan-out when it cannot
//             reach this step): narrow tiles of 256 neurons / one block per
//             wide neuron, items spread over the blocks
//   phase B   post-synaptic STDP chunks and spike fan-out of every population
// separated by grid barriers.  Removes the per-launch cost (about 3 us per
// kernel on this part) and the graph dependency latency of the K x (2..3)
// launches it replaces.  Every barrier wait is bounded: on timeout the block
// records FLAG_BARRIER_TIMEOUT and the kernel ends (I.spin_limit polls).
constexpr int kTlSlots = 6;
constexpr int kBarrierGroup = 16;     // blocks per first-level counter
constexpr int kBarrierStride = 32;    // words between counters (own 128-byte line)

// Two-level grid barrier: blocks arrive on the counter of their group of
// kBarrierGroup; the last of a group arrives on the root counter; the last at
// the root resets the counters and advances the generation word every block
// polls.  Spreads the arrival atomics over many cache lines instead of
// serialising gridDim.x of them on one.  Layout of bar (words):
//   [0] generation, [kBarrierStride] root count, [(g+2)*kBarrierStride] group g.
// I.withhold: block 0 does not arrive, so every block's wait runs out -- the
// failure path, exercised on purpose with a short I.spin_limit.
__device__ __forceinline__ bool grid_sync(const PersistInfo &I, unsigned nblocks, uint32_t *flags) {
    unsigned *bar = I.bar;
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_ok = 1;
        volatile unsigned *gen = bar;
        const unsigned g = *gen;
        const unsigned grp = blockIdx.x / kBarrierGroup;
        const unsigned ngroups = (nblocks + kBarrierGroup - 1) / kBarrierGroup;
        const unsigned in_grp = min((unsigned)kBarrierGroup, nblocks - grp * kBarrierGroup);
        unsigned *gc = bar + (grp + 2) * kBarrierStride;
        unsigned *root = bar + kBarrierStride;
        __threadfence();
        bool last = false;
        if (I.withhold && blockIdx.x == 0) {
        } else if (atomicAdd(gc, 1u) == in_grp - 1) {
            *gc = 0;
            __threadfence();
            if (atomicAdd(root, 1u) == ngroups - 1) {
                *root = 0;
                last = true;
            }
        }
        if (last) {
            __threadfence();
            atomicAdd(bar, 1u);
        } else {
            unsigned long long spins = 0;
            while (*gen == g) {
                __nanosleep(32);
                if (++spins > I.spin_limit) {
                    atomicOr(flags, FLAG_BARRIER_TIMEOUT);
                    s_ok = 0;
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return s_ok != 0;
}

template <int KIND, int INTEG>
__device__ __forceinline__ void update_item(const PopDev &P, const NetDev &N, int64_t k, int64_t local, WideSmem &S) {
    if (P.wide) update_wide_neuron<KIND, INTEG>(P, N, k, local, S);
    else update_narrow_tile<KIND, INTEG>(P, N, k, local);
}

// Register classes of the persistent kernel: the switch below compiles in only
// the model/integrator pairs of its class, so a network without HH or BDF does
// not pay their register pressure.
//   0: LIF, AdEx x Euler, RK2, RK4   1: + HH x Euler, RK2, RK4   2: everything
template <int CLASS, int KIND>
__device__ __forceinline__ void update_item_k(const PopDev &P, const NetDev &N, int64_t k, int64_t local, WideSmem &S) {
    switch (P.integ) {
    case INTEG_EULER: update_item<KIND, INTEG_EULER>(P, N, k, local, S); break;
    case INTEG_RK2: update_item<KIND, INTEG_RK2>(P, N, k, local, S); break;
    case INTEG_RK4: update_item<KIND, INTEG_RK4>(P, N, k, local, S); break;
    default:
        if constexpr (CLASS >= 2) update_item<KIND, INTEG_BDF>(P, N, k, local, S);
        else if (threadIdx.x == 0) atomicOr(N.flags, FLAG_PERSIST_UNSUPPORTED);
        break;
    }
}

int persist_class_of(int kind, int integ) {
    if (integ == INTEG_BDF) return 2;
    return kind == KIND_HH ? 1 : 0;
}

__device__ __forceinline__ int64_t update_items(const PopDev &P) {
    return P.wide ? P.n : (P.n + kNarrowTile - 1) / kNarrowTile;
}

// The item code reads its population's parameters many times per neuron; a
// block keeps the descriptor of the population it is working on in shared
// memory (broadcast reads) and reloads it only when it moves to another one.
__device__ __forceinline__ const PopDev &stage_pop(const PopDev *pops, int q, PopDev &sp, int &cur) {
    if (cur != q) {
        __syncthreads();
        const int *src = reinterpret_cast<const int *>(pops + q);
        int *dst = reinterpret_cast<int *>(&sp);
        for (int w = threadIdx.x; w < (int)(sizeof(PopDev) / sizeof(int)); w += blockDim.x) dst[w] = src[w];
        __syncthreads();
        cur = q;
    }
    return sp;
}

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Optional timeline (I.tl): per step r < I.tl_steps and block b, globaltimer at
// phase start, phase-A barrier arrival, phase-A barrier exit, phase-B barrier arrival.
__device__ __forceinline__ void tl_mark(const PersistInfo &I, int r, int slot) {
    if (I.tl && r < I.tl_steps && threadIdx.x == 0) I.tl[((int64_t)r * kTlSlots + slot) * gridDim.x + blockIdx.x] = gtimer();
}
__device__ __forceinline__ void tl_put(const PersistInfo &I, int r, int slot, unsigned long long v) {
    if (I.tl && r < I.tl_steps && threadIdx.x == 0) I.tl[((int64_t)r * kTlSlots + slot) * gridDim.x + blockIdx.x] = v;
}

// Dynamic item queue of one phase: each block starts with item blockIdx.x and
// then takes the next free index from the phase's counter (gridDim.x + n), so a
// block held up by a long item (a wide neuron) does not also receive later items.
// Thread 0 requests the following index as soon as it starts an item, hiding the
// atomic's latency behind the item's work.
struct ItemQueue {
    unsigned long long *ctr;
    int64_t cur, next;
    __device__ __forceinline__ void begin(unsigned long long *c) {
        ctr = c;
        cur = blockIdx.x;
    }
    __device__ __forceinline__ void prefetch() {
        if (threadIdx.x == 0) next = (int64_t)gridDim.x + (int64_t)atomicAdd(ctr, 1ull);
    }
    __device__ __forceinline__ int64_t advance(int64_t *s_next) {
        __syncthreads();
        if (threadIdx.x == 0) *s_next = next;
        __syncthreads();
        cur = *s_next;
        return cur;
    }
};

template <int CLASS>
__global__ void __launch_bounds__(kNarrowTile, CLASS == 0 ? 3 : (CLASS == 1 ? 2 : 1)) k_persistent(const PopDev *__restrict__ pops, PersistInfo I, NetDev N,
                                                            int K) {
    __shared__ WideSmem S;
    __shared__ PopDev sp;
    __shared__ int64_t s_next;
    int cur = -1;
    ItemQueue Q;
    const int64_t base = *N.step;
    const unsigned nb = gridDim.x;
    for (int r = 0; r < K; ++r) {
        const int64_t k = base + r + 1;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            for (int q = 0; q < I.n_pops; ++q) pops[q].spk_count[(k + 1) & 1] = 0;
            I.queue[(((k + 1) & 1) * 2 + 0) * 16] = 0;  // counters of the next step's phases
            I.queue[(((k + 1) & 1) * 2 + 1) * 16] = 0;
        }
        int64_t n_in = 0, q0 = 0;
        if (I.has_inputs) { q0 = N.in_start[k]; n_in = N.in_start[k + 1] - q0; }
        if (I.has_inputs && !I.inputs_concurrent) {
            for (int64_t it = blockIdx.x; it < n_in; it += nb) input_spike(N, k, q0 + it, I.inv_dt);
            if (!grid_sync(I, nb, N.flags)) return;
            n_in = 0;
        }
        // phase A: longest items first -- the populations in I.order (wide ones
        // first), with the input fan-out after the wide populations
        tl_mark(I, r, 0);
        int64_t total = n_in;
        for (int q = 0; q < I.n_pops; ++q) total += update_items(pops[q]);
        int n_items = 0;
        Q.begin(I.queue + ((k & 1) * 2 + 0) * 16);
        for (int64_t it = Q.cur; it < total; it = Q.advance(&s_next)) {
            Q.prefetch();
            if (n_items == 1) tl_mark(I, r, 4);
            ++n_items;
            int64_t local = it;
            int j = 0, q = -1;
            for (; j < I.n_pops; ++j) {
                if (j == I.n_wide) {
                    if (local < n_in) break;
                    local -= n_in;
                }
                const int64_t ni = update_items(pops[I.order[j]]);
                if (local < ni) { q = I.order[j]; break; }
                local -= ni;
            }
            if (q < 0) { input_spike(N, k, q0 + local, I.inv_dt); continue; }  // (advance runs in the for header)
            const PopDev &P = stage_pop(pops, q, sp, cur);
            switch (P.kind) {
            case KIND_LIF: update_item_k<CLASS, KIND_LIF>(P, N, k, local, S); break;
            case KIND_ADEX: update_item_k<CLASS, KIND_ADEX>(P, N, k, local, S); break;
            default:
                if constexpr (CLASS >= 1) update_item_k<CLASS, KIND_HH>(P, N, k, local, S);
                break;
            }
        }
        tl_mark(I, r, 1);
        tl_put(I, r, 5, (unsigned long long)n_items);
        if (!grid_sync(I, nb, N.flags)) return;
        tl_mark(I, r, 2);
        // phase B
        int64_t cnt[kMaxPersistPops];
        total = 0;
        for (int q = 0; q < I.n_pops; ++q) {
            const int64_t ns = min((int64_t)pops[q].spk_count[k & 1], pops[q].n);
            cnt[q] = ns * ((I.has_plastic >> q) & 1 ? I.post_chunks[q] : 0) + ns * ((I.has_out >> q) & 1);
            total += cnt[q];
        }
        Q.begin(I.queue + ((k & 1) * 2 + 1) * 16);
        for (int64_t it = Q.cur; it < total; it = Q.advance(&s_next)) {
            Q.prefetch();
            int64_t local = it;
            int q = 0;
            while (local >= cnt[q]) { local -= cnt[q]; ++q; }
            const PopDev &P = stage_pop(pops, q, sp, cur);
            const int64_t np = ((I.has_plastic >> q) & 1) ? min((int64_t)P.spk_count[k & 1], P.n) * I.post_chunks[q] : 0;
            if (local < np) post_item(P, N, k, local / I.post_chunks[q], local % I.post_chunks[q]);
            else push_spike(P, N, k, local - np, I.inv_dt);
        }
        tl_mark(I, r, 3);
        if (!grid_sync(I, nb, N.flags)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *const_cast<int64_t *>(N.step) += K;
}

static const void *persist_fn(int cls) {
    if (cls == 0) return (const void *)k_persistent<0>;
    if (cls == 1) return (const void *)k_persistent<1>;
    return (const void *)k_persistent<2>;
}

int persistent_blocks_per_sm(int cls) {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, persist_fn(cls), kNarrowTile, 0);
    return nb;
}

cudaError_t launch_persistent(int cls, const PopDev *pops, const PersistInfo &I, const NetDev &N, int K, int grid,
                              cudaStream_t st) {
    void *args[] = {(void *)&pops, (void *)&I, (void *)&N, (void *)&K};
    return cudaLaunchCooperativeKernel(persist_fn(cls), dim3(grid), dim3(kNarrowTile), args, 0, st);
}

__global__ void k_advance(int64_t *step, int K) { *step += K; }

// ------------------------------------------------------------------ launch --
template <int KIND, int INTEG>
static void launch_update_t(const PopDev &P, const NetDev &N, int rel, int nsteps, double push_inv_dt, cudaStream_t st) {
    if (P.wide) {
        const int blocks = (int)std::min<int64_t>(P.n, 148 * 8);
        const size_t sm = stage_smem_bytes();
        if (P.mon) k_update_wide<KIND, INTEG, 1, -1><<<blocks, kWideThreads, sm, st>>>(P, N, rel, nsteps, push_inv_dt);
        else if (P.en == 1) k_update_wide<KIND, INTEG, 0, 1><<<blocks, kWideThreads, sm, st>>>(P, N, rel, nsteps, push_inv_dt);
        else k_update_wide<KIND, INTEG, 0, -1><<<blocks, kWideThreads, sm, st>>>(P, N, rel, nsteps, push_inv_dt);
    } else {
        // the common conductance sets get kernels with the set compiled in; a
        // monitored population takes the generic kernel with the monitor hooks
        const int blocks = (int)((P.n + 255) / 256);
        if (P.mon) k_update_narrow<KIND, INTEG, -1, 1><<<blocks, 256, 0, st>>>(P, N, rel, nsteps, push_inv_dt);
        else if (P.en == 1) k_update_narrow<KIND, INTEG, 1, 0><<<blocks, 256, 0, st>>>(P, N, rel, nsteps, push_inv_dt);
        else if (P.en == 3) k_update_narrow<KIND, INTEG, 3, 0><<<blocks, 256, 0, st>>>(P, N, rel, nsteps, push_inv_dt);
        else k_update_narrow<KIND, INTEG, -1, 0><<<blocks, 256, 0, st>>>(P, N, rel, nsteps, push_inv_dt);
    }
}

template <int KIND>
static void launch_update_k(const PopDev &P, const NetDev &N, int rel, int nsteps, double push_inv_dt, cudaStream_t st) {
    switch (P.integ) {
    case INTEG_EULER: launch_update_t<KIND, INTEG_EULER>(P, N, rel, nsteps, push_inv_dt, st); break;
    case INTEG_RK2: launch_update_t<KIND, INTEG_RK2>(P, N, rel, nsteps, push_inv_dt, st); break;
    case INTEG_RK4: launch_update_t<KIND, INTEG_RK4>(P, N, rel, nsteps, push_inv_dt, st); break;
    default: launch_update_t<KIND, INTEG_BDF>(P, N, rel, nsteps, push_inv_dt, st); break;
    }
}

template <int KIND>
static cudaError_t prepare_wide_k() {
    const int bytes = (int)stage_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(k_update_wide<KIND, INTEG_EULER, 0, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_update_wide<KIND, INTEG_EULER, 0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_update_wide<KIND, INTEG_EULER, 1, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_update_wide<KIND, INTEG_RK2, 0, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_update_wide<KIND, INTEG_RK2, 0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_update_wide<KIND, INTEG_RK2, 1, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_update_wide<KIND, INTEG_RK4, 0, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_update_wide<KIND, INTEG_RK4, 0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_update_wide<KIND, INTEG_RK4, 1, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_update_wide<KIND, INTEG_BDF, 0, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_update_wide<KIND, INTEG_BDF, 0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_update_wide<KIND, INTEG_BDF, 1, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e;
}

// Opt the wide updates into their staging area (dynamic shared memory above the
// 48 KB default) on the current device; once per device, before any launch.
cudaError_t prepare_update_kernels() {
    cudaError_t e = prepare_wide_k<KIND_LIF>();
    if (e == cudaSuccess) e = prepare_wide_k<KIND_ADEX>();
    if (e == cudaSuccess) e = prepare_wide_k<KIND_HH>();
    return e;
}

void launch_update(const PopDev &P, const NetDev &N, int rel, int nsteps, double push_inv_dt, cudaStream_t st) {
    if (P.n <= 0) return;
    switch (P.kind) {
    case KIND_LIF: launch_update_k<KIND_LIF>(P, N, rel, nsteps, push_inv_dt, st); break;
    case KIND_ADEX: launch_update_k<KIND_ADEX>(P, N, rel, nsteps, push_inv_dt, st); break;
    case KIND_HH: launch_update_k<KIND_HH>(P, N, rel, nsteps, push_inv_dt, st); break;
    case KIND_POISSON:
        k_update_poisson<<<(unsigned)((P.n + 255) / 256), 256, 0, st>>>(P, N, rel, nsteps, push_inv_dt);
        break;
    default: break;
    }
}

void launch_push(const PopDev &P, const NetDev &N, int rel, double inv_dt, int blocks, int threads, cudaStream_t st) {
    k_push<<<blocks, threads, 0, st>>>(P, N, rel, inv_dt);
}

void launch_input_push(const NetDev &N, int rel, int nsteps, double inv_dt, int blocks, int threads, cudaStream_t st) {
    k_input_push<<<blocks, threads, 0, st>>>(N, rel, nsteps, inv_dt);
}

void launch_post_stdp(const PopDev &P, const NetDev &N, int rel, int max_chunks, int blocks, cudaStream_t st) {
    k_post_stdp<<<blocks, kPostThreads, 0, st>>>(P, N, rel, max_chunks);
}

// Bring every plastic synapse onto the population up to date with its target's
// deferred post-synaptic spikes: items are (neuron, chunk of kPostThreads plastic
// synapses), neurons without spikes since the last flush skipped.
// Deferred post-synaptic flush in three launches: k_flush_select lists the neurons
// with more than keep pending spikes (P.flush_list, count P.flush_list[P.n]);
// k_flush_post brings their plastic synapses up to date, items (listed neuron,
// chunk of kPostThreads synapses) in contiguous runs per block, so a block reads a
// neuron's count and stages its ring in shared memory once for all its chunks;
// k_flush_mark records the listed neurons as flushed and clears the list.
__global__ void __launch_bounds__(256) k_flush_select(PopDev P, uint32_t keep) {
    uint32_t *list = P.flush_list, *count = P.flush_list + P.n;
    for (int64_t i = threadIdx.x; i < P.n; i += blockDim.x)
        if (P.post_n[i] - P.post_flushed[i] > keep) list[atomicAdd(count, 1u)] = (uint32_t)i;
}

__global__ void __launch_bounds__(kPostThreads) k_flush_post(PopDev P, NetDev N, int max_chunks) {
    __shared__ double ring[kPostRing];
    __shared__ DecayPair fac[kPostRing];
    __shared__ uint32_t s_c;
    const int64_t items = (int64_t)P.flush_list[P.n] * max_chunks;
    const int64_t per = (items + gridDim.x - 1) / gridDim.x;
    const int64_t it0 = (int64_t)blockIdx.x * per, it1 = min(items, it0 + per);
    const int rule = P.post_f ? P.post_rule : -1;
    int64_t cur = -1;
    for (int64_t item = it0; item < it1; ++item) {
        const int64_t li = item / max_chunks, ch = item - li * max_chunks;
        const int64_t i = P.flush_list[li];
        if (li != cur) {
            __syncthreads();  // the block is done with the previous neuron's ring
            if (threadIdx.x == 0) s_c = P.post_n[i];
            for (int q = threadIdx.x; q < kPostRing; q += blockDim.x) {
                ring[q] = P.post_t[i * kPostRing + q];
                if (P.post_f) fac[q] = P.post_f[i * kPostRing + q];
            }
            __syncthreads();
            cur = li;
        }
        const int64_t t = P.first + i;
        const int64_t tp = N.in_ptr[t] + ch * kPostThreads + threadIdx.x;
        if (tp >= N.plastic_end[t]) continue;
        SynRec r = N.syn[tp];
        apply_pending(N, RingSmem{ring, fac}, s_c, rule, r);
        SynRec *o = N.syn + tp;
        o->w = r.w;
        o->pre = r.pre;
        o->post = r.post;
        o->last = r.last;
    }
}

__global__ void __launch_bounds__(256) k_flush_mark(PopDev P) {
    uint32_t *list = P.flush_list, *count = P.flush_list + P.n;
    const uint32_t n = *count;
    for (uint32_t a = threadIdx.x; a < n; a += blockDim.x) {
        const uint32_t i = list[a];
        P.post_flushed[i] = P.post_n[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) *count = 0;
}

void launch_flush_post(const PopDev &P, const NetDev &N, int max_chunks, uint32_t keep, int blocks, cudaStream_t st) {
    k_flush_select<<<1, 256, 0, st>>>(P, keep);
    k_flush_post<<<blocks, kPostThreads, 0, st>>>(P, N, max_chunks);
    k_flush_mark<<<1, 256, 0, st>>>(P);
}

void launch_advance(int64_t *step, int K, cudaStream_t st) { k_advance<<<1, 1, 0, st>>>(step, K); }

}  // namespace eb
