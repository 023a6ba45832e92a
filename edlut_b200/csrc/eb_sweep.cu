// Batched parameter sweep: many independent conductance-LIF networks of uneven
// size advanced together by one persistent kernel -- the sweep use of EDLUT
// (many simulations of small networks with varied parameters).
//
// A network is one LIF population (sources [0, n_exc) excitatory, [n_exc, n)
// inhibitory) plus n_in input neurons (sources n .. n+n_in-1, excitatory) whose
// spikes are given as times.  Connectivity is Bernoulli(p) from every source to
// every neuron with one delay and static weights; Euler, RK2 or RK4.
//
// One CTA owns one network for a chunk of steps (a persistent grid takes networks
// from an atomic queue, largest first, so uneven sizes balance).  Per step k:
//   1. deliveries: the source steps j whose spikes arrive at step k (one or two;
//      a host table, because the arrival step of t_j + d flips with the rounding
//      of the double step times) and the input spikes arriving in the step are
//      listed in the reference's delivery order -- arrival time, then synapse
//      order (source, target) -- by thread 0 from the spike bitmasks of the
//      delay ring held in shared memory.  Every thread loads a batch of the
//      listed sources' synapses (target, weight) at once, then the batch is
//      applied one source at a time with a barrier in between: targets of one
//      source are distinct, so each target receives its additions in list order
//      without atomics (src/spike/PropagatedSpikeGroup.cpp:112-149);
//   2. update: each thread advances neurons tid, tid + blockDim, ... (the whole
//      state -- V, refractory counter, gE, gI -- of the network lives in shared
//      memory for the chunk) with the model/integrator arithmetic of
//      the plain path, with the refractory test precomputed per network as step
//      counts (src/neuron_model/LIFTimeDrivenModel.cpp:160-242);
//   3. spikes: one warp ballot per 32 neurons is the bitmask word of the step's
//      ring slot (plus a summary bit per non-zero word); spiking lanes append
//      their neuron to the network's record.
// So each network's spikes equal a solo run of the same network on the plain
// path.  Connectivity and weights come from a counter-based hash of (seed,
// network, source, target), generated on the device at build time.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "eb_sweep.h"
#include "eb_tables.h"

using namespace eb;
using namespace ebsw;

namespace {

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ uint64_t net_key(uint64_t seed, int net) {
    return splitmix64(seed ^ ((uint64_t)(net + 1) * 0xD1B54A32D192ED03ull));
}

// Bernoulli(p) draw of synapse (src, tgt) of a network; returns the hash for the weight.
__device__ __forceinline__ bool syn_draw(uint64_t key, int src, int tgt, double p, uint64_t &h) {
    h = splitmix64(key ^ (((uint64_t)(uint32_t)src << 32) | (uint32_t)tgt));
    return (double)(h >> 11) * (1.0 / 9007199254740992.0) < p;
}

// ------------------------------------------------------- connectivity build --
// Synapse counts per source: blockIdx.y = network.
__global__ void k_sweep_count(const SweepNet *nets, uint64_t seed, uint32_t *counts) {
    const SweepNet &S = nets[blockIdx.y];
    if (S.explicit_syn) return;
    const uint64_t key = net_key(seed, blockIdx.y);
    const int nsrc = S.n + S.n_in;
    __shared__ int sc[32];
    for (int s = blockIdx.x; s < nsrc; s += gridDim.x) {
        int c = 0;
        for (int t = threadIdx.x; t < S.n; t += blockDim.x) {
            uint64_t h;
            c += syn_draw(key, s, t, (double)S.p, h) ? 1 : 0;
        }
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if ((threadIdx.x & 31) == 0) sc[threadIdx.x >> 5] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            int tot = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += sc[w];
            counts[S.src_off + s] = (uint32_t)tot;
        }
        __syncthreads();
    }
}

// One warp per source writes its targets in increasing order with their weights.
__global__ void k_sweep_fill(const SweepNet *nets, const uint32_t *optr, uint64_t seed, uint16_t *tgt, float *w) {
    const SweepNet &S = nets[blockIdx.y];
    if (S.explicit_syn) return;
    const uint64_t key = net_key(seed, blockIdx.y);
    const int nsrc = S.n + S.n_in;
    const int lane = threadIdx.x & 31;
    const int warps = blockDim.x >> 5;
    for (int s = blockIdx.x * warps + (threadIdx.x >> 5); s < nsrc; s += gridDim.x * warps) {
        int64_t pos = S.syn_off + optr[S.src_off + s];
        const float wmax = s < S.n_exc ? S.w_max[0] : (s < S.n ? S.w_max[1] : S.w_max[2]);
        for (int t0 = 0; t0 < S.n; t0 += 32) {
            const int t = t0 + lane;
            bool hit = false;
            uint64_t h = 0;
            if (t < S.n) hit = syn_draw(key, s, t, (double)S.p, h);
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (hit) {
                const int64_t o = pos + __popc(m & ((1u << lane) - 1u));
                const float u = (float)(splitmix64(h) >> 40) * (1.0f / 16777216.0f);
                tgt[o] = (uint16_t)t;
                w[o] = u * wmax;
            }
            pos += __popc(m);
        }
    }
}

// --------------------------------------------------------------- neuron update --
// One integration step, operation for operation the plain path's integrate<LIF, INTEG>.
template <int INTEG>
__device__ __forceinline__ void sw_integrate(const SweepLif &L, float dt, float &V, float &gE, float &gI, int cls, float f) {
    if (INTEG == INTEG_EULER) {
        const float k1 = sw_deriv(L, V, gE, gI, cls, f);
        V += dt * k1;
        sw_decay(L, gE, gI);
    } else if (INTEG == INTEG_RK2) {
        const float k1 = sw_deriv(L, V, gE, gI, cls, f);
        V += k1 * dt;
        sw_decay(L, gE, gI);
        const float k2 = sw_deriv(L, V, gE, gI, cls, f);
        V += (-k1 + k2) * dt * 0.5f;
    } else {
        const float h05 = dt * 0.5f;
        const float h016 = dt * 0.166666666667f;
        const float k1 = sw_deriv(L, V, gE, gI, cls, f);
        float a = V + k1 * h05;
        float aE = gE, aI = gI;
        sw_decay(L, aE, aI);
        const float k2 = sw_deriv(L, a, aE, aI, cls, f);
        a = V + k2 * h05;
        const float k3 = sw_deriv(L, a, aE, aI, cls, f);
        a = V + k3 * dt;
        sw_decay(L, aE, aI);
        const float k4 = sw_deriv(L, a, aE, aI, cls, f);
        V += (k1 + 2.0f * (k2 + k3) + k4) * h016;
        gE = aE;
        gI = aI;
    }
}

// Largest a in [0, S) with off[a] <= e (off[0] = 0 <= e < off[S]).
__device__ __forceinline__ int list_rank(const int32_t *off, int S, int e) {
    int lo = 0, hi = S;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= e) lo = mid; else hi = mid;
    }
    return lo;
}

struct SweepSmem {
    float *V, *gE, *gI;
    int32_t *rf;            // refractory counters
    uint32_t *ring, *sum;   // [R][wc], [R][swc]
    int32_t *src, *off;     // [kListCap], [kListCap + 1]
    uint32_t *base;         // [kListCap]
};

// Thread 0's delivery-list generator for one step: input spikes of phase 0, the
// spikes of the first arriving source step, inputs of phase 1, ... in order.
struct ListGen {
    int g, G, lo, part, a, q, slot;
    uint32_t sm, m;
    int64_t cur;      // input cursor
    int32_t nkey;     // key of input cur (INT_MAX when exhausted)
    int32_t nsrc;
};

template <int INTEG, bool TRAJ>
__device__ void sweep_network(const SweepDev &G, const SweepSmem &M, const SweepNet &S, const SweepLif &L, int net,
                              int64_t k0, int nsteps, int wc, int swc, int64_t traj_k0) {
    __shared__ int s_S, s_more;
    __shared__ uint32_t s_rec_n;
    const int n = S.n, n_exc = S.n_exc;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    const int nj = (n + nt - 1) / nt;
    const int R = G.R;
    const int wn = S.wn, swn = (wn + 31) >> 5;
    const int64_t so = S.state_off;
    const uint32_t *optr = G.optr + S.src_off;
    const uint16_t *tg = G.tgt + S.syn_off;
    const float *ww = G.w + S.syn_off;
    const float dt = G.dt_ms;

    for (int i = tid; i < n; i += nt) {
        M.V[i] = G.V[so + i];
        M.rf[i] = G.refr[so + i];
        M.gE[i] = G.gE[so + i];
        M.gI[i] = G.gI[so + i];
    }
    for (int x = tid; x < R * wc; x += nt) {
        const int slot = x / wc, q = x - slot * wc;
        M.ring[x] = q < wn ? G.ring[S.ring_off + (int64_t)slot * wn + q] : 0u;
    }
    for (int x = tid; x < R * swc; x += nt) {
        const int slot = x / swc, a = x - slot * swc;
        M.sum[x] = a < swn ? G.rsum[S.sum_off + (int64_t)slot * swn + a] : 0u;
    }
    ListGen gen;
    unsigned long long events = 0;
    int nx_lo = 0, nx_G = 0;
    if (tid == 0) {
        s_rec_n = G.rec_cnt[net];
        gen.cur = G.in_cursor[net];
        gen.nkey = INT_MAX;
        gen.nsrc = 0;
        if (gen.cur < S.n_in_spikes) { gen.nkey = G.in_key[S.in_off + gen.cur]; gen.nsrc = G.in_src[S.in_off + gen.cur]; }
        nx_lo = G.grp_lo[k0 + 1];
        nx_G = G.grp_n[k0 + 1];
    }
    __syncthreads();

    for (int r = 0; r < nsteps; ++r) {
        const int64_t k = k0 + r + 1;
        // ---------------------------------------------------- 1. deliveries
        if (tid == 0) {
            if (r > 0) G.rec_end[(int64_t)net * G.steps_max + (k - 2)] = (int32_t)s_rec_n;
            gen.g = 0;
            gen.G = nx_G;
            gen.lo = nx_lo;
            gen.part = 0;
            if (k + 1 <= G.steps_max) { nx_lo = G.grp_lo[k + 1]; nx_G = G.grp_n[k + 1]; }
        }
        const int32_t key0 = (int32_t)(k * 4);
        for (;;) {
            if (tid == 0) {
                int cnt = 0;
                bool done = false;
                while (cnt < kListCap) {
                    if (gen.part == 0) {
                        if (gen.nkey == key0 + gen.g) {
                            M.src[cnt++] = n + gen.nsrc;
                            ++gen.cur;
                            gen.nkey = INT_MAX;
                            if (gen.cur < S.n_in_spikes) {
                                gen.nkey = G.in_key[S.in_off + gen.cur];
                                gen.nsrc = G.in_src[S.in_off + gen.cur];
                            }
                            continue;
                        }
                        if (gen.g >= gen.G) { done = true; break; }
                        gen.part = 1;
                        gen.slot = (int)((gen.lo + gen.g) % R);
                        gen.a = 0;
                        gen.sm = M.sum[gen.slot * swc];
                        gen.m = 0;
                        continue;
                    }
                    if (gen.m) {
                        const int b = __ffs(gen.m) - 1;
                        gen.m &= gen.m - 1u;
                        M.src[cnt++] = gen.q * 32 + b;
                        continue;
                    }
                    if (gen.sm) {
                        const int b = __ffs(gen.sm) - 1;
                        gen.sm &= gen.sm - 1u;
                        gen.q = gen.a * 32 + b;
                        gen.m = M.ring[gen.slot * wc + gen.q];
                        continue;
                    }
                    if (++gen.a < swc) { gen.sm = M.sum[gen.slot * swc + gen.a]; continue; }
                    gen.part = 0;
                    ++gen.g;
                }
                s_S = cnt;
                s_more = done ? 0 : 1;
            }
            __syncthreads();
            const int Sn = s_S, more = s_more;
            if (Sn > 0) {
                if (warp == 0) {
                    int carry = 0;
                    for (int b = 0; b < Sn; b += 32) {
                        const int x = b + lane;
                        uint32_t lo = 0;
                        int fan = 0;
                        if (x < Sn) {
                            const int s = M.src[x];
                            lo = __ldg(optr + s);
                            fan = (int)(__ldg(optr + s + 1) - lo);
                        }
                        int incl = fan;
#pragma unroll
                        for (int o = 1; o < 32; o <<= 1) {
                            const int u = __shfl_up_sync(0xffffffffu, incl, o);
                            if (lane >= o) incl += u;
                        }
                        if (x < Sn) { M.off[x] = carry + incl - fan; M.base[x] = lo; }
                        carry += __shfl_sync(0xffffffffu, incl, 31);
                    }
                    if (lane == 0) M.off[Sn] = carry;
                }
                __syncthreads();
                const int total = M.off[Sn];
                for (int e0 = 0; e0 < total; e0 += kBatch * nt) {
                    uint16_t tq[kBatch];
                    float wq[kBatch];
                    int rk[kBatch];
                    bool inh[kBatch];
#pragma unroll
                    for (int q = 0; q < kBatch; ++q) {
                        const int e = e0 + q * nt + tid;
                        rk[q] = -1;
                        tq[q] = 0;
                        wq[q] = 0.0f;
                        inh[q] = false;
                        if (e < total) {
                            const int a = list_rank(M.off, Sn, e);
                            const uint32_t o = M.base[a] + (uint32_t)(e - M.off[a]);
                            tq[q] = __ldg(tg + o);
                            wq[q] = __ldg(ww + o);
                            const int s = M.src[a];
                            inh[q] = s >= n_exc && s < n;
                            rk[q] = a;
                        }
                    }
                    const int r_lo = list_rank(M.off, Sn, e0);
                    const int r_hi = list_rank(M.off, Sn, min(e0 + kBatch * nt, total) - 1);
                    for (int a = r_lo; a <= r_hi; ++a) {
#pragma unroll
                        for (int q = 0; q < kBatch; ++q)
                            if (rk[q] == a) {
                                float *g = inh[q] ? M.gI : M.gE;
                                g[tq[q]] += wq[q];
                            }
                        __syncthreads();
                    }
                }
                if (tid == 0) events += (unsigned long long)total;
            }
            if (!more) break;
            __syncthreads();
        }
        // -------------------------------------------------- 2. update, 3. spikes
        const int slot = (int)(k % R);
        for (int j = 0; j < nj; ++j) {
            {
                const int i = tid + j * nt;
                bool sp = false;
                if (i < n) {
                    float v = M.V[i], gE = M.gE[i], gI = M.gI[i];
                    int rr = M.rf[i];
                    int cls = 0, fi = 0;
                    float f = 1.0f;
                    if (rr >= 0 && rr < L.r_free) {
                        if (rr >= L.r_frac0) { cls = 2; fi = rr - L.r_frac0; f = L.frac[fi]; }
                        else cls = 1;
                    }
                    if (TRAJ) {
                        const int64_t x = (k - traj_k0 - 1) * G.n_total + so + i;
                        G.tV[x] = v;
                        G.tE[x] = gE;
                        G.tI[x] = gI;
                    }
                    sw_integrate<INTEG>(L, dt, v, gE, gI, cls, f);
                    if (rr >= 0) rr++;
                    if (v > L.v_thr) { v = L.e_leak; sp = true; rr = 0; }
                    if (TRAJ) G.tcode[(k - traj_k0 - 1) * G.n_total + so + i] = (uint8_t)(cls | (fi << 2) | (sp ? kCodeSpike : 0));
                    if (v != v) { v = L.e_leak; gE = 0.0f; gI = 0.0f; }
                    M.V[i] = v;
                    M.rf[i] = rr;
                    M.gE[i] = gE;
                    M.gI[i] = gI;
                }
                const unsigned m = __ballot_sync(0xffffffffu, sp);
                const int q = j * nwarps + warp;
                uint32_t base = 0;
                if (lane == 0) {
                    M.ring[slot * wc + q] = m;
                    if (m) {
                        atomicOr(&M.sum[slot * swc + (q >> 5)], 1u << (q & 31));
                        base = atomicAdd(&s_rec_n, (uint32_t)__popc(m));
                    }
                }
                if (m) {
                    base = __shfl_sync(0xffffffffu, base, 0);
                    if (sp) {
                        const uint32_t x = base + __popc(m & ((1u << lane) - 1u));
                        if ((int64_t)x < S.rec_cap) G.rec[S.rec_off + x] = (uint16_t)i;
                        else atomicOr(G.flags, FLAG_RECORD_OVERFLOW);
                    }
                }
            }
        }
        if (tid == 0) {
            // the slot written at step k+1 starts with an empty summary
            const int ns = (int)((k + 1) % R);
            for (int a = 0; a < swc; ++a) M.sum[ns * swc + a] = 0u;
        }
        __syncthreads();
        // observed membrane potentials after step k
        for (int m = tid; m < G.n_obs; m += nt)
            G.trace[((int64_t)net * G.steps_max + (k - 1)) * G.n_obs + m] = M.V[G.obs[(int64_t)net * G.n_obs + m]];
    }
    // save the network's state
    for (int i = tid; i < n; i += nt) {
        G.V[so + i] = M.V[i];
        G.refr[so + i] = M.rf[i];
        G.gE[so + i] = M.gE[i];
        G.gI[so + i] = M.gI[i];
    }
    for (int x = tid; x < R * wn; x += nt) {
        const int slot = x / wn, q = x - slot * wn;
        G.ring[S.ring_off + x] = M.ring[slot * wc + q];
    }
    for (int x = tid; x < R * swn; x += nt) {
        const int slot = x / swn, a = x - slot * swn;
        G.rsum[S.sum_off + x] = M.sum[slot * swc + a];
    }
    if (tid == 0) {
        if (nsteps > 0) G.rec_end[(int64_t)net * G.steps_max + (k0 + nsteps - 1)] = (int32_t)s_rec_n;
        G.rec_cnt[net] = s_rec_n;
        G.in_cursor[net] = gen.cur;
        G.events[net] += events;
    }
    __syncthreads();
}

template <int INTEG, bool TRAJ>
__global__ void __launch_bounds__(1024) k_sweep(SweepDev G, int nsteps, int max_n, int wc, int swc, int64_t traj_k0) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SweepSmem M;
    M.V = reinterpret_cast<float *>(smem_raw);
    M.gE = M.V + max_n;
    M.gI = M.gE + max_n;
    M.rf = reinterpret_cast<int32_t *>(M.gI + max_n);
    M.ring = reinterpret_cast<uint32_t *>(M.rf + max_n);
    M.sum = M.ring + G.R * wc;
    M.src = reinterpret_cast<int32_t *>(M.sum + G.R * swc);
    M.off = M.src + kListCap;
    M.base = reinterpret_cast<uint32_t *>(M.off + kListCap + 1);
    __shared__ int s_net;
    __shared__ SweepLif s_L;
    __shared__ SweepNet s_desc;
    const int64_t k0 = *G.step;
    for (;;) {
        if (threadIdx.x == 0) s_net = atomicAdd(G.queue, 1);
        __syncthreads();
        const int qi = s_net;
        if (qi >= G.n_nets) break;
        const int net = G.order[qi];
        {
            const int *src = reinterpret_cast<const int *>(G.nets + net);
            int *dst = reinterpret_cast<int *>(&s_desc);
            for (int x = threadIdx.x; x < (int)(sizeof(SweepNet) / sizeof(int)); x += blockDim.x) dst[x] = src[x];
        }
        __syncthreads();
        if (threadIdx.x == 0) s_L = s_desc.L;
        __syncthreads();
        sweep_network<INTEG, TRAJ>(G, M, s_desc, s_L, net, k0, nsteps, wc, swc, traj_k0);
    }
}

// After a chunk: advance the step counter and re-arm the network queue.
__global__ void k_sweep_advance(int64_t *step, int *queue, int nsteps) {
    *step += nsteps;
    *queue = 0;
}

}  // namespace

// ------------------------------------------------------------------- host --
namespace {

using SweepFn = void (*)(SweepDev, int, int, int, int, int64_t);

SweepFn sweep_fn(int integ, bool traj) {
    switch (integ) {
    case INTEG_EULER: return traj ? k_sweep<INTEG_EULER, true> : k_sweep<INTEG_EULER, false>;
    case INTEG_RK2: return traj ? k_sweep<INTEG_RK2, true> : k_sweep<INTEG_RK2, false>;
    default: return traj ? k_sweep<INTEG_RK4, true> : k_sweep<INTEG_RK4, false>;
    }
}

}  // namespace

namespace ebsw {

int enqueue_chunk(eb_sweep *h, int nsteps, cudaStream_t st, bool traj, int64_t traj_k0) {
    SweepFn f = sweep_fn(h->integ, traj);
    f<<<h->grid, h->block, h->smem, st>>>(h->G, nsteps, h->max_n, h->wc, h->swc, traj_k0);
    k_sweep_advance<<<1, 1, 0, st>>>(h->G.step, h->G.queue, nsteps);
    SK(cudaGetLastError());
    return EB_OK;
}

// The arrays that make up the dynamic state, in checkpoint order.
static void state_arrays(eb_sweep *h, void **ptr, size_t *bytes) {
    const size_t nt = (size_t)h->state_n, B = (size_t)h->n_nets;
    void *p[9] = {h->G.V, h->G.gE, h->G.gI, h->G.refr, h->G.ring, h->G.rsum, h->G.in_cursor, h->G.rec_cnt, h->G.events};
    size_t b[9] = {4 * nt, 4 * nt, 4 * nt, 4 * nt, 4 * (size_t)h->ring_words, 4 * (size_t)h->sum_words, 8 * B, 4 * B, 8 * B};
    for (int i = 0; i < 9; ++i) { ptr[i] = p[i]; bytes[i] = (b[i] + 255) / 256 * 256; }
    for (int i = 0; i < 9; ++i) bytes[i] = b[i] ? bytes[i] : 0;
}

size_t checkpoint_bytes(eb_sweep *h) {
    void *p[9];
    size_t b[9], t = 0;
    state_arrays(h, p, b);
    for (size_t x : b) t += x;
    return t;
}

int checkpoint_save(eb_sweep *h, int c, cudaStream_t st) {
    void *p[9];
    size_t b[9], off = 0;
    state_arrays(h, p, b);
    unsigned char *dst = (unsigned char *)h->ckpt[c];
    const size_t real[9] = {4 * (size_t)h->state_n, 4 * (size_t)h->state_n, 4 * (size_t)h->state_n, 4 * (size_t)h->state_n,
                            4 * (size_t)h->ring_words, 4 * (size_t)h->sum_words, 8 * (size_t)h->n_nets,
                            4 * (size_t)h->n_nets, 8 * (size_t)h->n_nets};
    for (int i = 0; i < 9; ++i) {
        if (real[i]) SK(cudaMemcpyAsync(dst + off, p[i], real[i], cudaMemcpyDeviceToDevice, st));
        off += b[i];
    }
    return EB_OK;
}

__global__ void k_sweep_set_step(int64_t *step, int *queue, int64_t v) {
    *step = v;
    *queue = 0;
}

int checkpoint_restore(eb_sweep *h, int c, int64_t step, cudaStream_t st) {
    void *p[9];
    size_t b[9], off = 0;
    state_arrays(h, p, b);
    const unsigned char *src = (const unsigned char *)h->ckpt[c];
    const size_t real[9] = {4 * (size_t)h->state_n, 4 * (size_t)h->state_n, 4 * (size_t)h->state_n, 4 * (size_t)h->state_n,
                            4 * (size_t)h->ring_words, 4 * (size_t)h->sum_words, 8 * (size_t)h->n_nets,
                            4 * (size_t)h->n_nets, 8 * (size_t)h->n_nets};
    for (int i = 0; i < 9; ++i) {
        if (real[i]) SK(cudaMemcpyAsync(p[i], src + off, real[i], cudaMemcpyDeviceToDevice, st));
        off += b[i];
    }
    k_sweep_set_step<<<1, 1, 0, st>>>(h->G.step, h->G.queue, step);
    SK(cudaGetLastError());
    return EB_OK;
}

}  // namespace ebsw

namespace {

// LIF parameters of a network from its 10 .cfg values (decay factors and the
// inverse capacitance computed like the plain path's finalize).
int fill_lif(eb_sweep *h, const float *lif_params, SweepLif &L);

// Precomputed refractory classes: the plain path's lif_deriv decides per call from
// l = refr * dt * 1000 (double); here the same comparisons run once per refr value.
int refractory_classes(float tau_ref, float dt_s, SweepLif &L) {
    const float dt_ms = dt_s * 1000.0f;
    L.r_frac0 = -1;
    for (int r = 0;; ++r) {
        const double l = ((double)r * (double)dt_s) * 1000.0;
        if (l > (double)tau_ref) {
            L.r_free = r;
            break;
        }
        if (l + (double)dt_ms > (double)tau_ref) {
            if (L.r_frac0 < 0) L.r_frac0 = r;
            if (r - L.r_frac0 >= kMaxFrac) return EB_ERR_UNSUPPORTED;
            L.frac[r - L.r_frac0] = (float)((l + (double)dt_ms - (double)tau_ref) / (double)dt_ms);
        }
        if (r > (1 << 24)) return EB_ERR_UNSUPPORTED;
    }
    if (L.r_frac0 < 0) L.r_frac0 = L.r_free;
    return EB_OK;
}

int fill_lif(eb_sweep *h, const float *lif_params, SweepLif &L) {
    const int en = L.en;
    memset(&L, 0, sizeof(L));
    L.en = en;
    L.e_exc = lif_params[0];
    L.e_inh = lif_params[1];
    L.e_leak = lif_params[2];
    L.v_thr = lif_params[3];
    L.g_leak = lif_params[8];
    L.inv_c_m = inv_double(lif_params[4]);
    const float dt_ms = h->dt * 1000.0f;
    const float el = (h->integ == INTEG_RK4) ? dt_ms * 0.5f : dt_ms;
    L.decay[0] = decay_factor(el, lif_params[5]);
    L.decay[1] = decay_factor(el, lif_params[6]);
    if (refractory_classes(lif_params[7], h->dt, L)) {
        set_error("refractory period %g ms unsupported at dt %g s", lif_params[7], h->dt);
        return EB_ERR_UNSUPPORTED;
    }
    return EB_OK;
}

}  // namespace

extern "C" {

int eb_sweep_create(int device, int n_networks, int integrator, float dt_s, float delay_s, uint64_t seed,
                    eb_sweep **out) {
    if (!out || n_networks <= 0 || n_networks > 65535 || integrator < INTEG_EULER || integrator > INTEG_RK4 || !(dt_s > 0) ||
        !(delay_s > 0)) {
        set_error("eb_sweep_create: bad argument (1..65535 networks, integrator Euler/RK2/RK4, dt > 0, delay > 0)");
        return EB_ERR_ARG;
    }
    SK(cudaSetDevice(device));
    eb_sweep *h = new eb_sweep();
    h->device = device;
    h->n_nets = n_networks;
    h->integ = integrator;
    h->dt = dt_s;
    h->delay = delay_s;
    h->seed = seed;
    h->nets.resize(n_networks);
    h->in_time.resize(n_networks);
    h->in_cell.resize(n_networks);
    h->xsrc.resize(n_networks);
    h->xtgt.resize(n_networks);
    h->xw.resize(n_networks);
    for (auto &s : h->nets) memset(&s, 0, sizeof(s));
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete h;
        set_error("stream: %s", cudaGetErrorString(e));
        return EB_ERR_CUDA;
    }
    *out = h;
    return EB_OK;
}

int eb_sweep_destroy(eb_sweep *h) {
    if (h) {
        cudaSetDevice(h->device);
        delete h;
    }
    return EB_OK;
}

int eb_sweep_set_network(eb_sweep *h, int i, int n, int n_in, int n_exc, const float *lif_params, float p,
                         float w_exc_max, float w_inh_max, float w_in_max) {
    if (!h || i < 0 || i >= h->n_nets || n <= 0 || n > kSweepMaxN || n_in < 0 || n + n_in > 65535 || n_exc < 0 ||
        n_exc > n || !lif_params || !(p >= 0.0f && p <= 1.0f)) {
        set_error("eb_sweep_set_network: bad argument (1 <= n <= %d, n + n_in <= 65535, 0 <= p <= 1)", kSweepMaxN);
        return EB_ERR_ARG;
    }
    if (h->built) { set_error("eb_sweep_set_network after eb_sweep_build"); return EB_ERR_STATE; }
    SweepNet &S = h->nets[i];
    S.n = n;
    S.n_in = n_in;
    S.n_exc = n_exc;
    S.wn = (n + 31) / 32;
    S.p = p;
    S.w_max[0] = w_exc_max;
    S.w_max[1] = w_inh_max;
    S.w_max[2] = w_in_max;
    for (int j = 0; j < 10; ++j) S.params[j] = lif_params[j];
    S.explicit_syn = 0;
    h->xsrc[i].clear();
    h->xtgt[i].clear();
    h->xw[i].clear();
    S.L.en = 0;
    const int rc = fill_lif(h, lif_params, S.L);
    if (rc) return rc;
    return EB_OK;
}

int eb_sweep_set_inputs(eb_sweep *h, int i, int64_t n, const float *time_s, const int32_t *cell) {
    if (!h || i < 0 || i >= h->n_nets || n < 0 || (n > 0 && (!time_s || !cell))) {
        set_error("eb_sweep_set_inputs: bad argument");
        return EB_ERR_ARG;
    }
    if (h->built) { set_error("eb_sweep_set_inputs after eb_sweep_build"); return EB_ERR_STATE; }
    for (int64_t q = 0; q < n; ++q)
        if (!(time_s[q] >= 0.0f)) { set_error("input spike %lld: negative or NaN time", (long long)q); return EB_ERR_ARG; }
    h->in_time[i].assign(time_s, time_s + n);
    h->in_cell[i].assign(cell, cell + n);
    return EB_OK;
}

int eb_sweep_set_synapses(eb_sweep *h, int i, int64_t m, const int32_t *src, const int32_t *tgt, const float *w) {
    if (!h || i < 0 || i >= h->n_nets || m < 0 || (m > 0 && (!src || !tgt || !w))) {
        set_error("eb_sweep_set_synapses: bad argument");
        return EB_ERR_ARG;
    }
    if (h->built) { set_error("eb_sweep_set_synapses after eb_sweep_build"); return EB_ERR_STATE; }
    SweepNet &S = h->nets[i];
    if (S.n <= 0) { set_error("eb_sweep_set_synapses: eb_sweep_set_network(%d) first", i); return EB_ERR_STATE; }
    for (int64_t k = 0; k < m; ++k)
        if (src[k] < 0 || src[k] >= S.n + S.n_in || tgt[k] < 0 || tgt[k] >= S.n) {
            set_error("eb_sweep_set_synapses: synapse %lld out of range", (long long)k);
            return EB_ERR_ARG;
        }
    h->xsrc[i].assign(src, src + m);
    h->xtgt[i].assign(tgt, tgt + m);
    h->xw[i].assign(w, w + m);
    S.explicit_syn = 1;
    return EB_OK;
}

int eb_sweep_build(eb_sweep *h, int64_t n_steps_max, float max_rate_hz) {
    if (!h || n_steps_max <= 0 || n_steps_max > (1 << 28) || !(max_rate_hz > 0)) {
        set_error("eb_sweep_build: bad argument");
        return EB_ERR_ARG;
    }
    if (h->built) { set_error("eb_sweep_build: already built"); return EB_ERR_STATE; }
    SK(cudaSetDevice(h->device));
    const int N = h->n_nets;
    for (int i = 0; i < N; ++i)
        if (h->nets[i].n <= 0) { set_error("eb_sweep_build: network %d not set", i); return EB_ERR_STATE; }
    // update times (the plain path's double accumulation) and the arrival step of
    // each source step: the first k with t_k > t_j + d
    const int64_t units = delay_units(h->delay);
    const double dd = (double)units * 0.0001;
    const int64_t T = n_steps_max + (int64_t)std::ceil(dd / (double)h->dt) + 16;
    std::vector<double> t(T + 1);
    t[0] = 0.0;
    for (int64_t k = 1; k <= T; ++k) t[k] = t[k - 1] + (double)h->dt;
    std::vector<int32_t> grp_lo(n_steps_max + 2, 0);
    std::vector<int8_t> grp_n(n_steps_max + 2, 0);
    h->h_arr_step.assign(n_steps_max + 1, INT32_MAX);
    int64_t dmax = 1;
    {
        int64_t ka = 2;
        for (int64_t j = 1; j <= n_steps_max; ++j) {
            const double a = t[j] + dd;
            if (ka < j + 1) ka = j + 1;
            while (ka <= T && t[ka] <= a) ++ka;
            if (ka > n_steps_max) break;
            h->h_arr_step[j] = (int32_t)ka;
            if (grp_n[ka] == 0) grp_lo[ka] = (int32_t)j;
            if (++grp_n[ka] > kMaxGroups) { set_error("eb_sweep_build: dt too small for the delay grid"); return EB_ERR_UNSUPPORTED; }
            dmax = std::max(dmax, ka - j);
        }
    }
    const int R = (int)dmax + 2;
    h->G.R = R;
    h->G.steps_max = (int)n_steps_max;
    h->G.dt_ms = h->dt * 1000.0f;
    h->G.integ = h->integ;
    // layout and input arrivals
    int64_t src_off = 0, state_off = 0, in_off = 0, ring_off = 0, sum_off = 0, rec_off = 0;
    std::vector<int32_t> in_key;
    std::vector<uint16_t> in_src;
    h->max_n = 0;
    for (int i = 0; i < N; ++i) {
        SweepNet &S = h->nets[i];
        S.src_off = src_off;
        src_off += S.n + S.n_in + 1;
        S.state_off = state_off;
        state_off += S.n;
        S.ring_off = ring_off;
        ring_off += (int64_t)R * S.wn;
        S.sum_off = sum_off;
        sum_off += (int64_t)R * ((S.wn + 31) / 32);
        S.rec_off = rec_off;
        S.rec_cap = (int64_t)std::ceil((double)S.n * (double)n_steps_max * (double)h->dt * (double)max_rate_hz) + 64;
        rec_off += S.rec_cap;
        h->max_n = std::max(h->max_n, S.n);
        // input spikes: arrival a = t_in + d reaches the first step with t_k > a;
        // phase = arriving source steps with a_j <= a (their spikes come first)
        struct Rec { int32_t key; float time; int32_t cell; };
        std::vector<Rec> recs;
        recs.reserve(h->in_time[i].size());
        for (size_t q = 0; q < h->in_time[i].size(); ++q) {
            const int32_t c = h->in_cell[i][q];
            if (c < 0 || c >= S.n_in) { set_error("network %d: input cell %d out of range", i, c); return EB_ERR_ARG; }
            const double a = (double)h->in_time[i][q] + dd;
            const int64_t ka = std::upper_bound(t.begin() + 1, t.end(), a) - t.begin();
            if (ka > n_steps_max) continue;
            int phase = 0;
            for (int g = 0; g < grp_n[ka]; ++g)
                if (t[grp_lo[ka] + g] + dd <= a) phase = g + 1;
            recs.push_back({(int32_t)(ka * 4 + phase), h->in_time[i][q], c});
        }
        std::stable_sort(recs.begin(), recs.end(), [](const Rec &x, const Rec &y) {
            if (x.key != y.key) return x.key < y.key;
            if (x.time != y.time) return x.time < y.time;
            return x.cell < y.cell;
        });
        S.in_off = in_off;
        S.n_in_spikes = (int64_t)recs.size();
        for (const Rec &x : recs) {
            in_key.push_back(x.key);
            in_src.push_back((uint16_t)x.cell);
        }
        in_off += (int64_t)recs.size();
    }
    h->state_n = state_off;
    h->ring_words = ring_off;
    h->sum_words = sum_off;
    h->h_in_key = in_key;
    h->G.n_total = state_off;
    int rc;
    SweepNet *d_nets;
    if ((rc = h->upload((void **)&d_nets, h->nets.data(), sizeof(SweepNet) * N))) return rc;
    h->d_nets = d_nets;
    h->G.nets = d_nets;
    h->G.n_nets = N;
    // connectivity: count per source, scan on the host, fill
    uint32_t *d_optr;
    if ((rc = h->upload((void **)&d_optr, nullptr, sizeof(uint32_t) * (size_t)src_off))) return rc;
    SK(cudaMemsetAsync(d_optr, 0, sizeof(uint32_t) * (size_t)src_off, h->stream));
    k_sweep_count<<<dim3(512, N), 256, 0, h->stream>>>(d_nets, h->seed, d_optr);
    SK(cudaGetLastError());
    std::vector<uint32_t> cnt(src_off);
    SK(cudaMemcpyAsync(cnt.data(), d_optr, sizeof(uint32_t) * (size_t)src_off, cudaMemcpyDeviceToHost, h->stream));
    SK(cudaStreamSynchronize(h->stream));
    // explicit networks: synapses sorted by (source, target), the reference's order
    // for one delay (qsort_inters, src/spike/Network.cpp:45-68), ties by caller order
    std::vector<std::vector<int64_t>> xord(N);
    for (int i = 0; i < N; ++i) {
        if (!h->nets[i].explicit_syn) continue;
        const SweepNet &S = h->nets[i];
        auto &o = xord[i];
        o.resize(h->xsrc[i].size());
        for (size_t k = 0; k < o.size(); ++k) o[k] = (int64_t)k;
        const auto &xs = h->xsrc[i], &xt = h->xtgt[i];
        std::stable_sort(o.begin(), o.end(), [&](int64_t a, int64_t b) {
            return xs[a] != xs[b] ? xs[a] < xs[b] : xt[a] < xt[b];
        });
        for (size_t k = 1; k < o.size(); ++k)
            if (xs[o[k]] == xs[o[k - 1]] && xt[o[k]] == xt[o[k - 1]]) {
                set_error("network %d: two synapses from %d to %d (one per pair in a sweep network)", i, xs[o[k]], xt[o[k]]);
                return EB_ERR_UNSUPPORTED;
            }
        for (int s = 0; s < S.n + S.n_in; ++s) cnt[S.src_off + s] = 0;
        for (size_t k = 0; k < o.size(); ++k) cnt[S.src_off + xs[k]]++;
    }
    int64_t syn_off = 0;
    for (int i = 0; i < N; ++i) {
        SweepNet &S = h->nets[i];
        S.syn_off = syn_off;
        uint64_t acc = 0, n_e = 0, n_i = 0;
        for (int s = 0; s < S.n + S.n_in; ++s) {
            const uint32_t c = cnt[S.src_off + s];
            cnt[S.src_off + s] = (uint32_t)acc;
            acc += c;
            if (s >= S.n_exc && s < S.n) n_i += c; else n_e += c;
        }
        if (acc > 0xffffffffull) { set_error("network %d: too many synapses", i); return EB_ERR_UNSUPPORTED; }
        cnt[S.src_off + S.n + S.n_in] = (uint32_t)acc;
        syn_off += (int64_t)acc;
        // conductance types present among the network's synapses
        S.L.en = (n_e ? 1 : 0) | (n_i ? 2 : 0);
    }
    h->total_syn = syn_off;
    SK(cudaMemcpy(d_nets, h->nets.data(), sizeof(SweepNet) * N, cudaMemcpyHostToDevice));
    SK(cudaMemcpy(d_optr, cnt.data(), sizeof(uint32_t) * (size_t)src_off, cudaMemcpyHostToDevice));
    h->G.optr = d_optr;
    uint16_t *d_tgt;
    float *d_w;
    if ((rc = h->upload((void **)&d_tgt, nullptr, sizeof(uint16_t) * (size_t)syn_off))) return rc;
    if ((rc = h->upload((void **)&d_w, nullptr, sizeof(float) * (size_t)syn_off))) return rc;
    h->G.tgt = d_tgt;
    h->G.w = d_w;
    k_sweep_fill<<<dim3(64, N), 256, 0, h->stream>>>(d_nets, d_optr, h->seed, d_tgt, d_w);
    SK(cudaGetLastError());
    // explicit networks' targets and weights, and the sweep -> caller synapse order
    {
        std::vector<int64_t> perm(syn_off);
        std::vector<uint16_t> xt;
        std::vector<float> xw;
        for (int i = 0; i < N; ++i) {
            const SweepNet &S = h->nets[i];
            const int64_t mi = (i + 1 < N ? h->nets[i + 1].syn_off : syn_off) - S.syn_off;
            if (!S.explicit_syn) {
                for (int64_t k = 0; k < mi; ++k) perm[S.syn_off + k] = S.syn_off + k;
                continue;
            }
            const auto &o = xord[i];
            xt.resize(o.size());
            xw.resize(o.size());
            for (size_t k = 0; k < o.size(); ++k) {
                xt[k] = (uint16_t)h->xtgt[i][o[k]];
                xw[k] = h->xw[i][o[k]];
                perm[S.syn_off + (int64_t)k] = S.syn_off + o[k];
            }
            if (!o.empty()) {
                SK(cudaMemcpyAsync(d_tgt + S.syn_off, xt.data(), sizeof(uint16_t) * o.size(), cudaMemcpyHostToDevice, h->stream));
                SK(cudaMemcpyAsync(d_w + S.syn_off, xw.data(), sizeof(float) * o.size(), cudaMemcpyHostToDevice, h->stream));
                SK(cudaStreamSynchronize(h->stream));
            }
        }
        if ((rc = h->upload((void **)&h->perm, perm.data(), sizeof(int64_t) * perm.size()))) return rc;
    }
    // state and tables
    h->v_init.assign(state_off, 0.0f);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < h->nets[i].n; ++j) h->v_init[h->nets[i].state_off + j] = h->nets[i].L.e_leak;
    if ((rc = h->upload((void **)&h->G.V, nullptr, sizeof(float) * (size_t)state_off))) return rc;
    if ((rc = h->upload((void **)&h->G.gE, nullptr, sizeof(float) * (size_t)state_off))) return rc;
    if ((rc = h->upload((void **)&h->G.gI, nullptr, sizeof(float) * (size_t)state_off))) return rc;
    if ((rc = h->upload((void **)&h->G.refr, nullptr, sizeof(int32_t) * (size_t)state_off))) return rc;
    if ((rc = h->upload((void **)&h->G.ring, nullptr, sizeof(uint32_t) * (size_t)ring_off))) return rc;
    if ((rc = h->upload((void **)&h->G.rsum, nullptr, sizeof(uint32_t) * (size_t)sum_off))) return rc;
    if ((rc = h->upload((void **)&h->G.grp_lo, grp_lo.data(), sizeof(int32_t) * grp_lo.size()))) return rc;
    if ((rc = h->upload((void **)&h->G.grp_n, grp_n.data(), sizeof(int8_t) * grp_n.size()))) return rc;
    if ((rc = h->upload((void **)&h->G.in_key, in_key.data(), sizeof(int32_t) * in_key.size()))) return rc;
    if ((rc = h->upload((void **)&h->G.in_src, in_src.data(), sizeof(uint16_t) * in_src.size()))) return rc;
    if ((rc = h->upload((void **)&h->G.in_cursor, nullptr, sizeof(int64_t) * N))) return rc;
    if ((rc = h->upload((void **)&h->G.rec, nullptr, sizeof(uint16_t) * (size_t)rec_off))) return rc;
    if ((rc = h->upload((void **)&h->G.rec_end, nullptr, sizeof(int32_t) * (size_t)N * n_steps_max))) return rc;
    if ((rc = h->upload((void **)&h->G.rec_cnt, nullptr, sizeof(uint32_t) * N))) return rc;
    if ((rc = h->upload((void **)&h->G.events, nullptr, sizeof(unsigned long long) * N))) return rc;
    if ((rc = h->upload((void **)&h->G.flags, nullptr, sizeof(uint32_t)))) return rc;
    if ((rc = h->upload((void **)&h->G.queue, nullptr, sizeof(int)))) return rc;
    if ((rc = h->upload((void **)&h->G.step, nullptr, sizeof(int64_t)))) return rc;
    if ((rc = h->upload((void **)&h->d_arr_step, h->h_arr_step.data(), sizeof(int32_t) * h->h_arr_step.size()))) return rc;
    std::vector<int32_t> order(N);
    for (int i = 0; i < N; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return h->nets[a].n > h->nets[b].n; });
    if ((rc = h->upload((void **)&h->G.order, order.data(), sizeof(int32_t) * N))) return rc;
    SK(cudaStreamSynchronize(h->stream));
    h->built = true;
    if ((rc = eb_sweep_reset(h))) return rc;
    return eb_sweep_configure(h, 0, 0);
}

int eb_sweep_reset(eb_sweep *h) {
    if (!h || !h->built) { set_error("eb_sweep_reset: sweep not built"); return EB_ERR_STATE; }
    SK(cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    const size_t ns = (size_t)h->state_n;
    SK(cudaMemcpyAsync(h->G.V, h->v_init.data(), sizeof(float) * ns, cudaMemcpyHostToDevice, st));
    SK(cudaMemsetAsync(h->G.gE, 0, sizeof(float) * ns, st));
    SK(cudaMemsetAsync(h->G.gI, 0, sizeof(float) * ns, st));
    SK(cudaMemsetAsync(h->G.refr, 0xff, sizeof(int32_t) * ns, st));  // -1: never spiked
    SK(cudaMemsetAsync(h->G.ring, 0, sizeof(uint32_t) * (size_t)h->ring_words, st));
    SK(cudaMemsetAsync(h->G.rsum, 0, sizeof(uint32_t) * (size_t)h->sum_words, st));
    SK(cudaMemsetAsync(h->G.in_cursor, 0, sizeof(int64_t) * h->n_nets, st));
    SK(cudaMemsetAsync(h->G.rec_cnt, 0, sizeof(uint32_t) * h->n_nets, st));
    SK(cudaMemsetAsync(h->G.rec_end, 0, sizeof(int32_t) * (size_t)h->n_nets * h->G.steps_max, st));
    SK(cudaMemsetAsync(h->G.events, 0, sizeof(unsigned long long) * h->n_nets, st));
    SK(cudaMemsetAsync(h->G.flags, 0, sizeof(uint32_t), st));
    SK(cudaMemsetAsync(h->G.queue, 0, sizeof(int), st));
    SK(cudaMemsetAsync(h->G.step, 0, sizeof(int64_t), st));
    SK(cudaStreamSynchronize(st));
    h->steps_done = 0;
    h->needs_reset = false;
    h->ckpt_upto = h->ckpt_every > 0 ? 0 : -1;
    return EB_OK;
}

int eb_sweep_configure(eb_sweep *h, int block, int steps_per_launch) {
    if (!h || !h->built) { set_error("eb_sweep_configure: sweep not built"); return EB_ERR_STATE; }
    int nb = block ? block : h->block;
    if (nb != 128 && nb != 256 && nb != 512 && nb != 1024) { set_error("block must be 128, 256, 512 or 1024"); return EB_ERR_ARG; }
    if (steps_per_launch < 0) { set_error("steps_per_launch < 0"); return EB_ERR_ARG; }
    const int npt = (h->max_n + nb - 1) / nb;  // neurons per thread
    const int wc = npt * nb / 32;
    const int swc = (wc + 31) / 32;
    const size_t smem = 16 * (size_t)h->max_n + sizeof(uint32_t) * (size_t)h->G.R * (wc + swc) +
                        sizeof(int32_t) * (3 * (size_t)kListCap + 1);
    SweepFn f = sweep_fn(h->integ, false);
    SK(cudaSetDevice(h->device));
    if (smem > 48 * 1024) {
        for (bool traj : {false, true}) {
            cudaError_t e = cudaFuncSetAttribute((const void *)sweep_fn(h->integ, traj),
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) {
                set_error("sweep kernel: %zu bytes of shared memory unavailable (%s)", smem, cudaGetErrorString(e));
                return EB_ERR_UNSUPPORTED;
            }
        }
    }
    int nsm = 0, occ = 0;
    SK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
    SK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, f, nb, smem));
    if (occ < 1) {
        set_error("sweep kernel does not fit (block %d, %zu bytes of shared memory)", nb, smem);
        return EB_ERR_UNSUPPORTED;
    }
    h->block = nb;
    h->npt = npt;
    h->wc = wc;
    h->swc = swc;
    h->smem = smem;
    h->grid = std::min(occ * nsm, h->n_nets);
    if (steps_per_launch) h->steps_per_launch = steps_per_launch;
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
        h->graph_chunks = 0;
    }
    return EB_OK;
}

int eb_sweep_run_async(eb_sweep *h, int64_t n_steps) {
    if (!h || !h->built) { set_error("eb_sweep_run: sweep not built"); return EB_ERR_STATE; }
    if (h->needs_reset) { set_error("eb_sweep_run: the adjoint left the sweep mid-run; eb_sweep_reset first"); return EB_ERR_STATE; }
    if (n_steps < 0 || h->steps_done + n_steps > h->G.steps_max) {
        set_error("eb_sweep_run: %lld steps exceed the %d built for", (long long)(h->steps_done + n_steps), h->G.steps_max);
        return EB_ERR_ARG;
    }
    SK(cudaSetDevice(h->device));
    if (h->ckpt_every > 0) {
        // chunks aligned to the checkpoint interval, the state saved before each
        const int E = h->ckpt_every;
        if (h->steps_done % E) { set_error("eb_sweep_run: checkpointed runs start at a multiple of %d steps", E); return EB_ERR_STATE; }
        const bool from0 = h->ckpt_upto == h->steps_done;
        int64_t done = 0;
        while (done < n_steps) {
            const int64_t k = h->steps_done + done;
            const int len = (int)std::min<int64_t>(E, n_steps - done);
            int rc = checkpoint_save(h, (int)(k / E), h->stream);
            if (!rc) rc = enqueue_chunk(h, len, h->stream);
            if (rc) return rc;
            done += len;
        }
        h->steps_done += n_steps;
        h->ckpt_upto = from0 ? h->steps_done : -1;
        return EB_OK;
    }
    const int spl = h->steps_per_launch;
    const int chunks = (int)(n_steps / spl);
    if (chunks > 0) {
        // the multi-step loop as one CUDA graph: chunks x (sweep kernel, advance)
        if (!h->graph || h->graph_chunks != chunks) {
            if (h->graph) cudaGraphExecDestroy(h->graph);
            h->graph = nullptr;
            cudaGraph_t g;
            SK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
            int rc = EB_OK;
            for (int c = 0; c < chunks && rc == EB_OK; ++c) rc = enqueue_chunk(h, spl, h->stream);
            cudaError_t e = cudaStreamEndCapture(h->stream, &g);
            if (rc) return rc;
            SK(e);
            e = cudaGraphInstantiate(&h->graph, g, 0);
            cudaGraphDestroy(g);
            SK(e);
            h->graph_chunks = chunks;
        }
        SK(cudaGraphLaunch(h->graph, h->stream));
    }
    const int rem = (int)(n_steps - (int64_t)chunks * spl);
    if (rem > 0) {
        int rc = enqueue_chunk(h, rem, h->stream);
        if (rc) return rc;
    }
    h->steps_done += n_steps;
    return EB_OK;
}

int eb_sweep_sync(eb_sweep *h) {
    if (!h || !h->built) { set_error("eb_sweep_sync: sweep not built"); return EB_ERR_STATE; }
    SK(cudaSetDevice(h->device));
    SK(cudaStreamSynchronize(h->stream));
    uint32_t f = 0;
    SK(cudaMemcpy(&f, h->G.flags, sizeof(f), cudaMemcpyDeviceToHost));
    if (f & FLAG_RECORD_OVERFLOW) { set_error("sweep: spike record overflow (raise max_rate_hz)"); return EB_ERR_OVERFLOW; }
    return EB_OK;
}

int eb_sweep_run(eb_sweep *h, int64_t n_steps) {
    int rc = eb_sweep_run_async(h, n_steps);
    if (rc) return rc;
    return eb_sweep_sync(h);
}

// Times `trial_steps` steps from the initial state for each launch configuration
// (threads per CTA, hence neurons per thread; steps per launch) and keeps the
// fastest.  Leaves the sweep reset to its initial state.
int eb_sweep_autotune(eb_sweep *h, int64_t trial_steps, int *best_block, int *best_spl, float *best_ms) {
    if (!h || !h->built || trial_steps <= 0 || trial_steps > h->G.steps_max) {
        set_error("eb_sweep_autotune: sweep not built or bad trial length");
        return EB_ERR_ARG;
    }
    SK(cudaSetDevice(h->device));
    cudaEvent_t e0, e1;
    SK(cudaEventCreate(&e0));
    SK(cudaEventCreate(&e1));
    const int blocks[4] = {128, 256, 512, 1024};
    const int64_t spls[2] = {std::max<int64_t>(1, trial_steps / 4), trial_steps};
    float best = 0;
    int bb = 0, bs = 0;
    int rc = EB_OK;
    bool warmed = false;
    for (int b : blocks) {
        for (int64_t s : spls) {
            if ((rc = eb_sweep_configure(h, b, (int)s))) {
                if (rc == EB_ERR_ARG || rc == EB_ERR_UNSUPPORTED) { rc = EB_OK; continue; }
                break;
            }
            for (int rep = warmed ? 1 : 0; rep < 2; ++rep) {
                if ((rc = eb_sweep_reset(h))) break;
                cudaEventRecord(e0, h->stream);
                if ((rc = eb_sweep_run_async(h, trial_steps))) break;
                cudaEventRecord(e1, h->stream);
                if ((rc = eb_sweep_sync(h))) break;
            }
            warmed = true;
            if (rc) break;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (!bb || ms < best) { best = ms; bb = b; bs = (int)s; }
        }
        if (rc) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (!bb) { set_error("eb_sweep_autotune: no launch configuration fits"); return EB_ERR_UNSUPPORTED; }
    if ((rc = eb_sweep_configure(h, bb, bs))) return rc;
    if ((rc = eb_sweep_reset(h))) return rc;
    if (best_block) *best_block = bb;
    if (best_spl) *best_spl = bs;
    if (best_ms) *best_ms = best;
    return EB_OK;
}

int eb_sweep_get_spikes(eb_sweep *h, int i, int64_t cap, int64_t *n, int32_t *step, int32_t *cell) {
    if (!h || !h->built || i < 0 || i >= h->n_nets || !n || cap < 0) { set_error("eb_sweep_get_spikes: bad argument"); return EB_ERR_ARG; }
    SK(cudaSetDevice(h->device));
    SK(cudaStreamSynchronize(h->stream));
    const SweepNet &S = h->nets[i];
    const int64_t ns = h->steps_done;
    std::vector<int32_t> end(ns);
    if (ns) SK(cudaMemcpy(end.data(), h->G.rec_end + (int64_t)i * h->G.steps_max, sizeof(int32_t) * ns, cudaMemcpyDeviceToHost));
    const int64_t cnt = ns ? (int64_t)(uint32_t)end[ns - 1] : 0;
    *n = cnt;
    if (cnt > S.rec_cap) { set_error("network %d: spike record overflowed (raise max_rate_hz)", i); return EB_ERR_OVERFLOW; }
    if (cnt > cap) { set_error("eb_sweep_get_spikes: buffer holds %lld of %lld spikes", (long long)cap, (long long)cnt); return EB_ERR_OVERFLOW; }
    std::vector<uint16_t> buf(cnt);
    if (cnt) SK(cudaMemcpy(buf.data(), h->G.rec + S.rec_off, sizeof(uint16_t) * cnt, cudaMemcpyDeviceToHost));
    int64_t b = 0;
    for (int64_t k = 0; k < ns; ++k) {
        const int64_t e = (uint32_t)end[k];
        std::sort(buf.begin() + b, buf.begin() + e);  // within a step the record order is arbitrary
        for (int64_t q = b; q < e; ++q) {
            if (step) step[q] = (int32_t)(k + 1);
            if (cell) cell[q] = buf[q];
        }
        b = e;
    }
    return EB_OK;
}

int eb_sweep_spike_counts(eb_sweep *h, int64_t *counts) {
    if (!h || !h->built || !counts) { set_error("eb_sweep_spike_counts: bad argument"); return EB_ERR_ARG; }
    SK(cudaSetDevice(h->device));
    SK(cudaStreamSynchronize(h->stream));
    std::vector<uint32_t> c(h->n_nets);
    SK(cudaMemcpy(c.data(), h->G.rec_cnt, sizeof(uint32_t) * h->n_nets, cudaMemcpyDeviceToHost));
    for (int i = 0; i < h->n_nets; ++i) counts[i] = c[i];
    return EB_OK;
}

int eb_sweep_get_synapses(eb_sweep *h, int i, int64_t cap, int64_t *m, int32_t *src, int32_t *tgt, float *w) {
    if (!h || !h->built || i < 0 || i >= h->n_nets || !m || cap < 0) { set_error("eb_sweep_get_synapses: bad argument"); return EB_ERR_ARG; }
    SK(cudaSetDevice(h->device));
    SK(cudaStreamSynchronize(h->stream));
    const SweepNet &S = h->nets[i];
    const int ns = S.n + S.n_in;
    std::vector<uint32_t> optr(ns + 1);
    SK(cudaMemcpy(optr.data(), h->G.optr + S.src_off, sizeof(uint32_t) * (ns + 1), cudaMemcpyDeviceToHost));
    const int64_t mm = optr[ns];
    *m = mm;
    if (mm > cap) { set_error("eb_sweep_get_synapses: buffer holds %lld of %lld synapses", (long long)cap, (long long)mm); return EB_ERR_OVERFLOW; }
    std::vector<uint16_t> t(mm);
    if (mm) {
        SK(cudaMemcpy(t.data(), h->G.tgt + S.syn_off, sizeof(uint16_t) * mm, cudaMemcpyDeviceToHost));
        if (w) SK(cudaMemcpy(w, h->G.w + S.syn_off, sizeof(float) * mm, cudaMemcpyDeviceToHost));
    }
    for (int s = 0; s < ns; ++s)
        for (int64_t o = optr[s]; o < (int64_t)optr[s + 1]; ++o) {
            if (src) src[o] = s;
            if (tgt) tgt[o] = t[o];
        }
    return EB_OK;
}

int eb_sweep_get_state(eb_sweep *h, int i, int var, float *out) {
    if (!h || !h->built || i < 0 || i >= h->n_nets || var < 0 || var > 2 || !out) { set_error("eb_sweep_get_state: bad argument"); return EB_ERR_ARG; }
    SK(cudaSetDevice(h->device));
    SK(cudaStreamSynchronize(h->stream));
    const float *src = var == 0 ? h->G.V : (var == 1 ? h->G.gE : h->G.gI);
    SK(cudaMemcpy(out, src + h->nets[i].state_off, sizeof(float) * h->nets[i].n, cudaMemcpyDeviceToHost));
    return EB_OK;
}

int eb_sweep_info(eb_sweep *h, int64_t *synapses, int64_t *device_bytes, int64_t *events, int *block,
                  int *steps_per_launch, int *grid) {
    if (!h) { set_error("eb_sweep_info: null handle"); return EB_ERR_ARG; }
    if (synapses) *synapses = h->total_syn;
    if (device_bytes) *device_bytes = h->dev_bytes;
    if (events) {
        *events = 0;
        if (h->built) {
            SK(cudaSetDevice(h->device));
            SK(cudaStreamSynchronize(h->stream));
            std::vector<unsigned long long> ev(h->n_nets);
            SK(cudaMemcpy(ev.data(), h->G.events, sizeof(unsigned long long) * h->n_nets, cudaMemcpyDeviceToHost));
            for (auto v : ev) *events += (int64_t)v;
        }
    }
    if (block) *block = h->block;
    if (steps_per_launch) *steps_per_launch = h->steps_per_launch;
    if (grid) *grid = h->grid;
    return EB_OK;
}

int eb_sweep_stream(eb_sweep *h, void **stream) {
    if (!h || !stream) { set_error("eb_sweep_stream: bad argument"); return EB_ERR_ARG; }
    *stream = (void *)h->stream;
    return EB_OK;
}

int eb_sweep_set_params(eb_sweep *h, int i, const float *lif_params) {
    if (!h || i < 0 || i >= h->n_nets || !lif_params || h->nets[i].n <= 0) { set_error("eb_sweep_set_params: bad argument"); return EB_ERR_ARG; }
    SweepNet &S = h->nets[i];
    SweepLif L = S.L;
    int rc = fill_lif(h, lif_params, L);
    if (rc) return rc;
    S.L = L;
    for (int j = 0; j < 10; ++j) S.params[j] = lif_params[j];
    if (h->built) {
        SK(cudaSetDevice(h->device));
        SK(cudaStreamSynchronize(h->stream));
        SK(cudaMemcpy(h->d_nets + i, &S, sizeof(SweepNet), cudaMemcpyHostToDevice));
        for (int j = 0; j < S.n; ++j) h->v_init[S.state_off + j] = L.e_leak;
    }
    return EB_OK;
}

namespace {
__global__ void k_perm_gather(const int64_t *perm, int64_t m, const float *src, float *dst) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < m; p += (int64_t)gridDim.x * blockDim.x)
        dst[p] = src[perm[p]];
}
__global__ void k_perm_scatter(const int64_t *perm, int64_t m, const float *src, float *dst) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < m; p += (int64_t)gridDim.x * blockDim.x)
        dst[perm[p]] = src[p];
}
}  // namespace

static int weights_io(eb_sweep *h, float *buf, int on_device, int to_sweep) {
    if (!h || !h->built || !buf) { set_error("eb_sweep weights: sweep not built or null buffer"); return EB_ERR_ARG; }
    SK(cudaSetDevice(h->device));
    const int64_t m = h->total_syn;
    if (!m) return EB_OK;
    float *dev = buf;
    float *tmp = nullptr;
    if (!on_device) {
        SK(cudaMallocAsync((void **)&tmp, sizeof(float) * m, h->stream));
        dev = tmp;
        if (to_sweep) SK(cudaMemcpyAsync(tmp, buf, sizeof(float) * m, cudaMemcpyHostToDevice, h->stream));
    }
    float *w = const_cast<float *>(h->G.w);
    if (to_sweep) k_perm_gather<<<592, 256, 0, h->stream>>>(h->perm, m, dev, w);
    else k_perm_scatter<<<592, 256, 0, h->stream>>>(h->perm, m, w, dev);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && !on_device && !to_sweep) e = cudaMemcpyAsync(buf, tmp, sizeof(float) * m, cudaMemcpyDeviceToHost, h->stream);
    if (tmp) cudaFreeAsync(tmp, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) { set_error("eb_sweep weights: %s", cudaGetErrorString(e)); return EB_ERR_CUDA; }
    return EB_OK;
}

int eb_sweep_set_weights(eb_sweep *h, const float *w, int on_device) {
    return weights_io(h, const_cast<float *>(w), on_device, 1);
}

int eb_sweep_get_weights(eb_sweep *h, float *w, int on_device) { return weights_io(h, w, on_device, 0); }

int eb_sweep_set_observed(eb_sweep *h, int m, const int32_t *idx) {
    if (!h || !h->built || m < 0 || (m > 0 && !idx)) { set_error("eb_sweep_set_observed: sweep not built or bad argument"); return EB_ERR_ARG; }
    for (int i = 0; i < h->n_nets; ++i)
        for (int q = 0; q < m; ++q)
            if (idx[(int64_t)i * m + q] < 0 || idx[(int64_t)i * m + q] >= h->nets[i].n) {
                set_error("eb_sweep_set_observed: network %d index %d out of range", i, idx[(int64_t)i * m + q]);
                return EB_ERR_ARG;
            }
    if (m <= h->G.n_obs && m > 0) {
        SK(cudaMemcpy((void *)h->G.obs, idx, sizeof(int32_t) * (size_t)h->n_nets * m, cudaMemcpyHostToDevice));
    } else if (m > 0) {
        int rc;
        int32_t *d_obs;
        float *d_trace;
        if ((rc = h->upload((void **)&d_obs, idx, sizeof(int32_t) * (size_t)h->n_nets * m))) return rc;
        if ((rc = h->dalloc((void **)&d_trace, sizeof(float) * (size_t)h->n_nets * h->G.steps_max * m))) return rc;
        h->G.obs = d_obs;
        h->G.trace = d_trace;
    }
    h->G.n_obs = m;
    h->h_obs.assign(idx, idx + (size_t)h->n_nets * m);
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
        h->graph_chunks = 0;
    }
    return EB_OK;
}

int eb_sweep_get_trace(eb_sweep *h, float *out, int on_device) {
    if (!h || !h->built || !out) { set_error("eb_sweep_get_trace: bad argument"); return EB_ERR_ARG; }
    const int m = h->G.n_obs;
    if (!m || !h->steps_done) return EB_OK;
    SK(cudaSetDevice(h->device));
    const size_t row = sizeof(float) * (size_t)h->steps_done * m;
    const size_t pitch = sizeof(float) * (size_t)h->G.steps_max * m;
    SK(cudaMemcpy2DAsync(out, row, h->G.trace, pitch, row, h->n_nets,
                         on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->stream));
    SK(cudaStreamSynchronize(h->stream));
    return EB_OK;
}

int eb_sweep_set_checkpoints(eb_sweep *h, int every) {
    if (!h || !h->built || every < 0) { set_error("eb_sweep_set_checkpoints: sweep not built or bad interval"); return EB_ERR_ARG; }
    if (every == 0) { h->ckpt_every = 0; return EB_OK; }
    if (every > 255) { set_error("eb_sweep_set_checkpoints: at most 255 steps between checkpoints"); return EB_ERR_ARG; }
    SK(cudaSetDevice(h->device));
    const int n = (int)((h->G.steps_max + every - 1) / every);
    const size_t b = checkpoint_bytes(h);
    while ((int)h->ckpt.size() < n) {
        void *p;
        int rc = h->dalloc(&p, b);
        if (rc) return rc;
        h->ckpt.push_back(p);
    }
    h->ckpt_every = every;
    h->n_ckpt = n;
    h->ckpt_upto = h->steps_done == 0 ? 0 : -1;
    return EB_OK;
}

}  // extern "C"
