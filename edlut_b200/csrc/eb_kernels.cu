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

// STDPWeightChange::ApplyPreSynapticSpike on synapse tp at arrival time a.
__device__ __forceinline__ void stdp_pre(const NetDev &N, uint32_t tp, int rl, double a) {
    const float *rp = N.rule_par + rl * 6;
    float el = (float)(a - N.last[tp]);
    float pre = N.pre[tp] * expt_net(N, -el * rp[4]);
    float post = N.post[tp] * expt_net(N, -el * rp[5]);
    N.last[tp] = a;
    pre += 1.0f;
    float w = N.w[tp];
    w += -rp[2] * post;
    float mw = N.maxw[tp];
    if (w > mw) w = mw; else if (w < 0.0f) w = 0.0f;
    N.pre[tp] = pre;
    N.post[tp] = post;
    N.w[tp] = w;
}

template <int ND>
__device__ __forceinline__ void add_conductance(float *x, int ty, float w) {
    if (ty == 0) x[ND] += w;
    else if (ty == 1) x[ND + 1] += w;
    else x[ND + 2] += w;
}

// Apply one arrival: g[type] += w (weight before plasticity), then STDP pre.
template <int ND>
__device__ __forceinline__ void apply_arrival(const NetDev &N, const Arrival &r, float *x) {
    const uint32_t tp = r.tpos;
    add_conductance<ND>(x, N.stype[tp], N.w[tp]);
    const int rl = N.rule[tp];
    if (rl >= 0) stdp_pre(N, tp, rl, r.a);
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

// Advance one neuron (after its arrivals were folded); returns spike flag.
template <int KIND, int INTEG>
__device__ __forceinline__ bool advance_neuron(const PopDev &P, const NetDev &N, int64_t i, float *x) {
    constexpr int NV = Model<KIND>::NV;
    int refr = (KIND == KIND_LIF) ? P.refr[i] : -1;
    int bst = (INTEG == INTEG_BDF) ? (int)P.bdf_state[i] : 0;
    BdfRef H{P.bdf_D, P.bdf_P, P.n, i};
    const float prevV = x[0];
    if (!integrate<KIND, INTEG>(P, x, refr, bst, H)) atomicOr(N.flags, FLAG_BDF_SINGULAR);
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
    if (KIND == KIND_LIF) P.refr[i] = refr;
    if (INTEG == INTEG_BDF) P.bdf_state[i] = (int8_t)bst;
    return sp;
}

__device__ __forceinline__ void record_trace(const PopDev &P, const NetDev &N, int64_t k, int64_t gi, const float *x, int nv) {
    if (!N.trace) return;
    int64_t c = gi - N.trace_first, s = k - N.trace_k0;
    if (c < 0 || c >= N.trace_n || s < 0 || s >= N.trace_steps) return;
    float *o = N.trace + (s * N.trace_n + c) * kMaxVars;
    for (int v = 0; v < nv; ++v) o[v] = x[v];
}

// Warp-aggregated append of the spiking lanes to the population spike list and
// to the recording buffer.
__device__ __forceinline__ void compact_spikes(const PopDev &P, const NetDev &N, int64_t k, int64_t i, bool sp) {
    const unsigned full = 0xffffffffu;
    const unsigned m = __ballot_sync(full, sp);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    const unsigned below = m & ((1u << lane) - 1u);
    uint32_t base = 0;
    unsigned long long rbase = 0;
    if (lane == leader) {
        base = atomicAdd(&P.spk_count[k & 1], (uint32_t)__popc(m));
        if (N.rec_buf) rbase = atomicAdd(N.rec_count, (unsigned long long)__popc(m));
    }
    base = __shfl_sync(full, base, leader);
    rbase = __shfl_sync(full, rbase, leader);
    if (sp) {
        const uint32_t o = base + __popc(below);
        if (o < (uint32_t)P.n) P.spk[o] = (uint32_t)i;
        else atomicOr(N.flags, FLAG_SPIKELIST_OVERFLOW);
        if (N.rec_buf) {
            const unsigned long long ro = rbase + __popc(below);
            if (ro < (unsigned long long)N.rec_cap)
                N.rec_buf[ro] = ((unsigned long long)k << 32) | (unsigned long long)(P.first + i);
            else atomicOr(N.flags, FLAG_RECORD_OVERFLOW);
        }
    }
}

// ----------------------------------------------------------- narrow update --
// One thread per neuron.  Arrivals of this step are sorted in registers
// (insertion sort; at most 16 in the fast path) and folded in order.
constexpr int kLocalSort = 16;

template <int KIND, int INTEG>
__global__ void __launch_bounds__(256) k_update_narrow(PopDev P, NetDev N, int rel) {
    constexpr int ND = Model<KIND>::ND;
    const int64_t k = cur_step(N, rel);
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x == 0 && threadIdx.x == 0) P.spk_count[(k + 1) & 1] = 0;
    const bool active = i < P.n;
    bool sp = false;
    uint32_t c = 0;
    if (active) {
        const int64_t gi = P.first + i;
        float x[kMaxVars];
        load_state<KIND>(P, i, x);
        const int slot = (int)(k % N.R);
        uint32_t *cp = N.cnt + (int64_t)slot * N.n_neurons + gi;
        c = *cp;
        if (c) {
            *cp = 0;
            const uint32_t capg = N.cap[gi];
            if (c > capg) { atomicOr(N.flags, FLAG_BUCKET_OVERFLOW); c = capg; }
            Arrival *r = N.rec + (int64_t)slot * N.cap_total + N.cap_base[gi];
            if (c == 1) {
                apply_arrival<ND>(N, r[0], x);
            } else if (c <= kLocalSort) {
                Arrival loc[kLocalSort];
                for (uint32_t a = 0; a < c; ++a) {
                    Arrival v = r[a];
                    int b = (int)a - 1;
                    while (b >= 0 && arr_less(v, loc[b])) { loc[b + 1] = loc[b]; --b; }
                    loc[b + 1] = v;
                }
                for (uint32_t a = 0; a < c; ++a) apply_arrival<ND>(N, loc[a], x);
            } else {
                for (uint32_t a = 1; a < c; ++a) {  // in-place insertion sort (rare path)
                    Arrival v = r[a];
                    int b = (int)a - 1;
                    while (b >= 0 && arr_less(v, r[b])) { r[b + 1] = r[b]; --b; }
                    r[b + 1] = v;
                }
                for (uint32_t a = 0; a < c; ++a) apply_arrival<ND>(N, r[a], x);
            }
        }
        sp = advance_neuron<KIND, INTEG>(P, N, i, x);
        store_state<KIND>(P, i, x);
        record_trace(P, N, k, gi, x, Model<KIND>::NV);
    }
    // delivered-event counter: one atomic per warp
    unsigned long long cw = c;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cw += __shfl_down_sync(0xffffffffu, cw, o);
    if ((threadIdx.x & 31) == 0 && cw) atomicAdd(N.events, cw);
    compact_spikes(P, N, k, i, sp);
}

// ------------------------------------------------------------- wide update --
// One block per neuron, for populations whose neurons receive many arrivals per
// step (e.g. Purkinje-like cells with 10^4-10^5 inputs).  The block sorts the
// arrivals in shared memory (bitonic, up to kWideSmem records), every thread
// fetches the weight of one arrival and applies its STDP pre-synaptic update in
// parallel (synapses are independent; a synapse that can arrive twice in one step
// -- only from input neurons -- forces the serial path), and thread 0 adds the
// weights into the conductances in delivery order, then integrates the neuron.
constexpr int kWideThreads = 256;
constexpr int kWideSmem = 1024;

template <int KIND, int INTEG>
__global__ void __launch_bounds__(kWideThreads) k_update_wide(PopDev P, NetDev N, int rel) {
    constexpr int ND = Model<KIND>::ND;
    __shared__ Arrival sbuf[kWideSmem];
    __shared__ float sw[kWideSmem];
    __shared__ uint8_t sty[kWideSmem];
    const int tid = threadIdx.x;
    const int64_t k = cur_step(N, rel);
    if (blockIdx.x == 0 && tid == 0) P.spk_count[(k + 1) & 1] = 0;
    const int slot = (int)(k % N.R);
    for (int64_t i = blockIdx.x; i < P.n; i += gridDim.x) {
        const int64_t gi = P.first + i;
        uint32_t *cp = N.cnt + (int64_t)slot * N.n_neurons + gi;
        uint32_t c = *cp;
        __syncthreads();
        float x[kMaxVars];
        if (tid == 0) load_state<KIND>(P, i, x);
        if (c) {
            if (tid == 0) *cp = 0;
            const uint32_t capg = N.cap[gi];
            if (c > capg) { if (tid == 0) atomicOr(N.flags, FLAG_BUCKET_OVERFLOW); c = capg; }
            Arrival *r = N.rec + (int64_t)slot * N.cap_total + N.cap_base[gi];
            if (c <= (uint32_t)kWideSmem) {
                int n2 = 1;
                while (n2 < (int)c) n2 <<= 1;
                for (int a = tid; a < n2; a += kWideThreads) {
                    if (a < (int)c) sbuf[a] = r[a];
                    else { sbuf[a].a = __longlong_as_double(0x7ff0000000000000LL); sbuf[a].spos = 0xffffffffu; sbuf[a].tpos = 0; }
                }
                __syncthreads();
                for (int size = 2; size <= n2; size <<= 1)
                    for (int stride = size >> 1; stride > 0; stride >>= 1) {
                        for (int a = tid; a < n2; a += kWideThreads) {
                            const int b = a ^ stride;
                            if (b > a) {
                                const bool up = ((a & size) == 0);
                                const Arrival ea = sbuf[a], eb = sbuf[b];
                                if (up ? arr_less(eb, ea) : arr_less(ea, eb)) { sbuf[a] = eb; sbuf[b] = ea; }
                            }
                        }
                        __syncthreads();
                    }
                if (P.may_repeat) {
                    if (tid == 0)
                        for (uint32_t a = 0; a < c; ++a) apply_arrival<ND>(N, sbuf[a], x);
                } else {
                    for (int a = tid; a < (int)c; a += kWideThreads) {
                        const Arrival v = sbuf[a];
                        const uint32_t tp = v.tpos;
                        sw[a] = N.w[tp];
                        sty[a] = N.stype[tp];
                        const int rl = N.rule[tp];
                        if (rl >= 0) stdp_pre(N, tp, rl, v.a);
                    }
                    __syncthreads();
                    if (tid == 0)
                        for (uint32_t a = 0; a < c; ++a) add_conductance<ND>(x, sty[a], sw[a]);
                }
            } else if (tid == 0) {
                for (uint32_t a = 1; a < c; ++a) {  // rare: insertion sort in global memory
                    Arrival v = r[a];
                    int b = (int)a - 1;
                    while (b >= 0 && arr_less(v, r[b])) { r[b + 1] = r[b]; --b; }
                    r[b + 1] = v;
                }
                for (uint32_t a = 0; a < c; ++a) apply_arrival<ND>(N, r[a], x);
            }
            if (tid == 0) atomicAdd(N.events, (unsigned long long)c);
        }
        if (tid == 0) {
            const bool sp = advance_neuron<KIND, INTEG>(P, N, i, x);
            store_state<KIND>(P, i, x);
            record_trace(P, N, k, gi, x, Model<KIND>::NV);
            if (sp) {
                const uint32_t o = atomicAdd(&P.spk_count[k & 1], 1u);
                if (o < (uint32_t)P.n) P.spk[o] = (uint32_t)i;
                else atomicOr(N.flags, FLAG_SPIKELIST_OVERFLOW);
                if (N.rec_buf) {
                    const unsigned long long ro = atomicAdd(N.rec_count, 1ull);
                    if (ro < (unsigned long long)N.rec_cap)
                        N.rec_buf[ro] = ((unsigned long long)k << 32) | (unsigned long long)gi;
                    else atomicOr(N.flags, FLAG_RECORD_OVERFLOW);
                }
            }
        }
    }
}

// ------------------------------------------------------------ spike fan-out --
// Arrival step of a delivery at time a: the first update time strictly after a.
// `est` is a close guess; two table reads confirm it in the common case.
__device__ __forceinline__ int64_t arrival_step(const NetDev &N, double a, int64_t k_lo, int64_t est) {
    int64_t ka = est < k_lo ? k_lo : est;
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
    const int slot = (int)(ka % N.R);
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

// Spikes of population P at step k (update time t_k): one block per spike, the
// threads cover the source's out-synapses (sorted by delay, then target).
__global__ void __launch_bounds__(256) k_push(PopDev P, NetDev N, int rel, double inv_dt) {
    const int64_t k = cur_step(N, rel);
    const uint32_t ns = min(P.spk_count[k & 1], (uint32_t)P.n);
    const double tk = N.tstep[k];
    for (int64_t s = blockIdx.x; s < ns; s += gridDim.x) {
        const int64_t src = P.first + P.spk[s];
        const int64_t o0 = N.out_ptr[src], o1 = N.out_ptr[src + 1];
        for (int64_t o = o0 + threadIdx.x; o < o1; o += blockDim.x) {
            const double d = (double)N.out_units[o] * 0.0001;
            const double a = tk + d;
            bucket_put(N, arrival_step(N, a, k + 1, k + (int64_t)(d * inv_dt)), a, o);
        }
    }
}

// Input-neuron spikes emitted in [t_{k-1}, t_k): one block per spike.  A source
// with several distinct delays delivers group j+1 at (a_j - d_j) + d_{j+1}, as the
// reference's PropagatedSpike chain does.
__global__ void __launch_bounds__(256) k_input_push(NetDev N, int rel, double inv_dt) {
    const int64_t k = cur_step(N, rel);
    const int64_t q0 = N.in_start[k], q1 = N.in_start[k + 1];
    const double tprev = N.tstep[k - 1];
    for (int64_t q = q0 + blockIdx.x; q < q1; q += gridDim.x) {
        const int64_t src = N.in_cell[q];
        const double tin = N.in_time[q];
        const int64_t o0 = N.out_ptr[src], o1 = N.out_ptr[src + 1];
        const int64_t g0 = N.grp_ptr[src], g1 = N.grp_ptr[src + 1];
        for (int64_t o = o0 + threadIdx.x; o < o1; o += blockDim.x) {
            const uint16_t u = N.out_units[o];
            double a = tin + (double)N.grp_units[g0] * 0.0001;
            for (int64_t g = g0 + 1; g < g1 && N.grp_units[g - 1] != u; ++g)
                a = a - (double)N.grp_units[g - 1] * 0.0001 + (double)N.grp_units[g] * 0.0001;
            bucket_put(N, arrival_step(N, a, k, k - 1 + (int64_t)((a - tprev) * inv_dt)), a, o);
        }
    }
}

// Post-synaptic STDP (STDPWeightChange::ApplyPostSynapticSpike) for every spike
// of population P at step k.  Work items are (spike, chunk of blockDim plastic
// input synapses of that neuron); one synapse per thread.
__global__ void __launch_bounds__(256) k_post_stdp(PopDev P, NetDev N, int rel, int max_chunks) {
    const int64_t k = cur_step(N, rel);
    const uint32_t ns = min(P.spk_count[k & 1], (uint32_t)P.n);
    const double tk = N.tstep[k];
    const int64_t items = (int64_t)ns * max_chunks;
    for (int64_t item = blockIdx.x; item < items; item += gridDim.x) {
        const int64_t s = item / max_chunks, ch = item % max_chunks;
        const int64_t t = P.first + P.spk[s];
        const int64_t tp = N.in_ptr[t] + ch * blockDim.x + threadIdx.x;
        if (tp >= N.plastic_end[t]) continue;
        const int rl = N.rule[tp];
        const float *rp = N.rule_par + rl * 6;
        const double last = N.last[tp];
        float pre = N.pre[tp], post = N.post[tp], w = N.w[tp];
        const float mw = N.maxw[tp];
        const float el = (float)(tk - last);
        pre *= expt_net(N, -el * rp[4]);
        post *= expt_net(N, -el * rp[5]);
        post += 1.0f;
        w += rp[0] * pre;
        if (w > mw) w = mw; else if (w < 0.0f) w = 0.0f;
        N.last[tp] = tk;
        N.pre[tp] = pre;
        N.post[tp] = post;
        N.w[tp] = w;
    }
}

__global__ void k_advance(int64_t *step, int K) { *step += K; }

// ------------------------------------------------------------------ launch --
template <int KIND, int INTEG>
static void launch_update_t(const PopDev &P, const NetDev &N, int rel, cudaStream_t st) {
    if (P.wide) {
        const int blocks = (int)std::min<int64_t>(P.n, 148 * 8);
        k_update_wide<KIND, INTEG><<<blocks, kWideThreads, 0, st>>>(P, N, rel);
    } else {
        const int blocks = (int)((P.n + 255) / 256);
        k_update_narrow<KIND, INTEG><<<blocks, 256, 0, st>>>(P, N, rel);
    }
}

template <int KIND>
static void launch_update_k(const PopDev &P, const NetDev &N, int rel, cudaStream_t st) {
    switch (P.integ) {
    case INTEG_EULER: launch_update_t<KIND, INTEG_EULER>(P, N, rel, st); break;
    case INTEG_RK2: launch_update_t<KIND, INTEG_RK2>(P, N, rel, st); break;
    case INTEG_RK4: launch_update_t<KIND, INTEG_RK4>(P, N, rel, st); break;
    default: launch_update_t<KIND, INTEG_BDF>(P, N, rel, st); break;
    }
}

void launch_update(const PopDev &P, const NetDev &N, int rel, cudaStream_t st) {
    if (P.n <= 0) return;
    switch (P.kind) {
    case KIND_LIF: launch_update_k<KIND_LIF>(P, N, rel, st); break;
    case KIND_ADEX: launch_update_k<KIND_ADEX>(P, N, rel, st); break;
    case KIND_HH: launch_update_k<KIND_HH>(P, N, rel, st); break;
    default: break;
    }
}

void launch_push(const PopDev &P, const NetDev &N, int rel, double inv_dt, int blocks, int threads, cudaStream_t st) {
    k_push<<<blocks, threads, 0, st>>>(P, N, rel, inv_dt);
}

void launch_input_push(const NetDev &N, int rel, double inv_dt, int blocks, int threads, cudaStream_t st) {
    k_input_push<<<blocks, threads, 0, st>>>(N, rel, inv_dt);
}

void launch_post_stdp(const PopDev &P, const NetDev &N, int rel, int max_chunks, int blocks, cudaStream_t st) {
    k_post_stdp<<<blocks, kPostThreads, 0, st>>>(P, N, rel, max_chunks);
}

void launch_advance(int64_t *step, int K, cudaStream_t st) { k_advance<<<1, 1, 0, st>>>(step, K); }

}  // namespace eb
