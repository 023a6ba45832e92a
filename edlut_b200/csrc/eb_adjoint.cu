// Adjoint of the batched sweep: gradients of a loss on observed membrane traces
// with respect to each network's g_leak, E_leak, tau_AMPA, tau_GABA and every
// synaptic weight, for the forward computed by the sweep kernel (the method's
// own time stepping, unchanged).
//
// The forward is a discrete map per step k: deliveries (g += w of each arriving
// synapse), one integrator step of (V, gE, gI), the threshold test and the reset
// V <- E_leak.  A spike is stamped at the update time t_k and delivered at
// t_k + d, so the spike pattern is piecewise constant in the parameters: the
// exact derivative of the forward carries no spike-time terms, and the jump
// condition at a threshold crossing is the reset map itself (the adjoint of V is
// cut, its value goes to E_leak).  Between spikes neurons interact only through
// spikes, so the adjoint is neuron-local:
//   lambda_{k-1} = J_k^T lambda_k + dL/dx_{k-1}
// with J_k the Jacobian of the integrator step (Euler / RK2 / RK4 stages
// reversed), and dL/dw of a synapse = sum over its source's spikes of the
// adjoint of the target's conductance at the arrival step.
//
// Memory: the forward saves the full state every K steps (eb_sweep_set_checkpoints);
// the backward walks the segments last to first: restore the checkpoint,
// recompute the segment with the trajectory-recording forward kernel (the
// integration inputs of every neuron-step), run the per-neuron adjoint over the
// segment (k_adj_neuron), then the weight gradients of the spikes arriving in the
// segment (k_adj_wgrad, per source: a deterministic sum over its spikes).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "eb_sweep.h"

using namespace eb;
using namespace ebsw;

namespace {

constexpr int kInstCap = 4096;  // spike instances per weight-gradient pass

// Adjoint of one derivative evaluation D(V, gE, gI) (sw_deriv): lk = dL/dD.
__device__ __forceinline__ void d_deriv(const SweepLif &L, float V, float gE, float gI, int cls, float f, float lk,
                                        float &lV, float &lE, float &lI, float &pGL, float &pEL) {
    if (cls == 1) return;
    const float s = (cls == 2 ? f : 1.0f) * L.inv_c_m * lk;
    float dV = -L.g_leak;
    if (L.en & 1) { dV -= gE; lE += s * (L.e_exc - V); }
    if (L.en & 2) { dV -= gI; lI += s * (L.e_inh - V); }
    lV += s * dV;
    pGL += s * (L.e_leak - V);
    pEL += s * L.g_leak;
}

// Adjoint of sw_decay (g' = a g, or 0 below 1e-9): lEo, lIo = dL/dg'.
__device__ __forceinline__ void d_decay(const SweepLif &L, float gE, float gI, float lEo, float lIo, float &lE,
                                        float &lI, float &pAE, float &pAI) {
    const float limit = 1e-9;
    if (L.en & 1) {
        if (!(gE < limit)) { lE += lEo * L.decay[0]; pAE += lEo * gE; }
    } else {
        lE += lEo;
    }
    if (L.en & 2) {
        if (!(gI < limit)) { lI += lIo * L.decay[1]; pAI += lIo * gI; }
    } else {
        lI += lIo;
    }
}

// Reverse of one integrator step (sw_integrate) at inputs (V, gE, gI): given the
// adjoints of its outputs (lVo for V before the reset, lEo, lIo for the decayed
// conductances) returns the adjoints of its inputs and adds the parameter
// partials (g_leak, E_leak, AMPA and GABA decay factors).
template <int INTEG>
__device__ __forceinline__ void d_integrate(const SweepLif &L, float dt, float V, float gE, float gI, int cls, float f,
                                            float lVo, float lEo, float lIo, float &lV, float &lE, float &lI,
                                            float &pGL, float &pEL, float &pAE, float &pAI) {
    lV = 0.0f;
    lE = 0.0f;
    lI = 0.0f;
    if (INTEG == INTEG_EULER) {
        // V' = V + dt k1, g' = decay(g)
        lV = lVo;
        d_deriv(L, V, gE, gI, cls, f, lVo * dt, lV, lE, lI, pGL, pEL);
        d_decay(L, gE, gI, lEo, lIo, lE, lI, pAE, pAI);
    } else if (INTEG == INTEG_RK2) {
        // V1 = V + k1 dt, g2 = decay(g), k2 = D(V1, g2), V' = V1 + (k2 - k1) dt / 2
        const float k1 = sw_deriv(L, V, gE, gI, cls, f);
        const float V1 = V + k1 * dt;
        float gE2 = gE, gI2 = gI;
        sw_decay(L, gE2, gI2);
        const float lk2 = lVo * dt * 0.5f;
        float lV1 = lVo, lE2 = lEo, lI2 = lIo;
        d_deriv(L, V1, gE2, gI2, cls, f, lk2, lV1, lE2, lI2, pGL, pEL);
        const float lk1 = -lk2 + lV1 * dt;
        lV = lV1;
        d_deriv(L, V, gE, gI, cls, f, lk1, lV, lE, lI, pGL, pEL);
        d_decay(L, gE, gI, lE2, lI2, lE, lI, pAE, pAI);
    } else {
        // a1 = V + k1 h/2, gA = decay(g), k2 = D(a1, gA), a2 = V + k2 h/2, k3 = D(a2, gA),
        // a3 = V + k3 h, gB = decay(gA), k4 = D(a3, gB), V' = V + (k1 + 2 (k2 + k3) + k4) h/6, g' = gB
        const float h05 = dt * 0.5f;
        const float h016 = dt * 0.166666666667f;
        const float k1 = sw_deriv(L, V, gE, gI, cls, f);
        const float a1 = V + k1 * h05;
        float gAE = gE, gAI = gI;
        sw_decay(L, gAE, gAI);
        const float k2 = sw_deriv(L, a1, gAE, gAI, cls, f);
        const float a2 = V + k2 * h05;
        const float k3 = sw_deriv(L, a2, gAE, gAI, cls, f);
        const float a3 = V + k3 * dt;
        float gBE = gAE, gBI = gAI;
        sw_decay(L, gBE, gBI);
        lV = lVo;
        float lk1 = lVo * h016;
        const float lk4 = lk1;
        float lBE = lEo, lBI = lIo, la3 = 0.0f;
        d_deriv(L, a3, gBE, gBI, cls, f, lk4, la3, lBE, lBI, pGL, pEL);
        lV += la3;
        const float lk3 = 2.0f * h016 * lVo + la3 * dt;
        float lAE = 0.0f, lAI = 0.0f;
        d_decay(L, gAE, gAI, lBE, lBI, lAE, lAI, pAE, pAI);
        float la2 = 0.0f;
        d_deriv(L, a2, gAE, gAI, cls, f, lk3, la2, lAE, lAI, pGL, pEL);
        lV += la2;
        const float lk2 = 2.0f * h016 * lVo + la2 * h05;
        float la1 = 0.0f;
        d_deriv(L, a1, gAE, gAI, cls, f, lk2, la1, lAE, lAI, pGL, pEL);
        lV += la1;
        lk1 += la1 * h05;
        d_decay(L, gE, gI, lAE, lAI, lE, lI, pAE, pAI);
        d_deriv(L, V, gE, gI, cls, f, lk1, lV, lE, lI, pGL, pEL);
    }
}

__device__ __forceinline__ float frac_of(const SweepLif &L, int fi) {
    return fi == 0 ? L.frac[0] : fi == 1 ? L.frac[1] : fi == 2 ? L.frac[2] : L.frac[3];
}

// Per-neuron adjoint over one segment of `len` steps after step k_lo, backward.
// Carries (lambda_V, lambda_gE, lambda_gI) across segments in lam*, accumulates
// the parameter partials in gacc (double, per neuron) and writes the adjoint of
// each step's post-arrival conductances to muE / muI for the weight gradients.
template <int INTEG>
__global__ void __launch_bounds__(256) k_adj_neuron(SweepDev G, const SweepNet *nets, int64_t k_lo, int len,
                                                     int64_t n_steps, const float *gtrace, const int32_t *obs_slot,
                                                     float *lamV, float *lamE, float *lamI, double *gacc, float *muE,
                                                     float *muI, int first_seg) {
    const int net = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = nets[net].n;
    if (i >= n) return;
    const SweepLif L = nets[net].L;
    const int64_t Nt = G.n_total;
    const int64_t gi = nets[net].state_off + i;
    const int m = obs_slot[gi];
    const float dt = G.dt_ms;
    float lV = lamV[gi], lE = lamE[gi], lI = lamI[gi];
    double aGL = 0.0, aEL = 0.0, aAE = 0.0, aAI = 0.0;
    for (int kk = len - 1; kk >= 0; --kk) {
        const int64_t x = (int64_t)kk * Nt + gi;
        if (m >= 0) lV += gtrace[((int64_t)net * n_steps + (k_lo + kk)) * G.n_obs + m];
        const int code = G.tcode[x];
        const float V = G.tV[x], gE = G.tE[x], gI = G.tI[x];
        const int cls = code & 3;
        const float f = cls == 2 ? frac_of(L, (code >> 2) & 3) : 1.0f;
        float pGL = 0.0f, pEL = 0.0f, pAE = 0.0f, pAI = 0.0f;
        if (code & kCodeSpike) {  // V_k = E_leak: the jump cuts lambda_V
            aEL += (double)lV;
            lV = 0.0f;
        }
        float nV, nE, nI;
        d_integrate<INTEG>(L, dt, V, gE, gI, cls, f, lV, lE, lI, nV, nE, nI, pGL, pEL, pAE, pAI);
        lV = nV;
        lE = nE;
        lI = nI;
        muE[x] = lE;
        muI[x] = lI;
        aGL += (double)pGL;
        aEL += (double)pEL;
        aAE += (double)pAE;
        aAI += (double)pAI;
    }
    if (first_seg) aEL += (double)lV;  // V_0 = E_leak
    lamV[gi] = lV;
    lamE[gi] = lE;
    lamI[gi] = lI;
    gacc[0 * Nt + gi] += aGL;
    gacc[1 * Nt + gi] += aEL;
    gacc[2 * Nt + gi] += aAE;
    gacc[3 * Nt + gi] += aAI;
}

// First index in [lo, hi) of keys[] with keys[i] >= v.
__device__ int64_t lower_bound_key(const int32_t *keys, int64_t lo, int64_t hi, int32_t v) {
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (keys[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Weight gradients of the spikes arriving in the segment (steps k_lo+1 .. k_lo+len):
// internal spikes of source steps [j_a, j_b] and input spikes with arrival keys in
// the segment.  Block (network, part) takes the sources of its part, sorts their
// (source, step) instances in shared memory and gives each source to one warp,
// which adds, per synapse, the sum over the source's instances (ascending step)
// of the target's conductance adjoint at the arrival step.
__global__ void __launch_bounds__(256) k_adj_wgrad(SweepDev G, const SweepNet *nets, const int32_t *arr_step,
                                                    int64_t k_lo, int len, int j_a, int j_b, const float *muE,
                                                    const float *muI, float *gw, uint32_t *flags) {
    __shared__ uint32_t keys[kInstCap];
    __shared__ int runs[kInstCap];
    __shared__ int s_cnt, s_runs;
    __shared__ int64_t s_rs, s_re, s_ilo, s_ihi;
    const int net = blockIdx.x;
    const SweepNet &S = nets[net];
    const int nsrc = S.n + S.n_in;
    const int p_lo = (int)((int64_t)blockIdx.y * nsrc / gridDim.y);
    const int p_hi = (int)((int64_t)(blockIdx.y + 1) * nsrc / gridDim.y);
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    const int64_t Nt = G.n_total;
    const int32_t *rec_end = G.rec_end + (int64_t)net * G.steps_max;
    if (tid == 0) {
        s_rs = j_a >= 2 ? rec_end[j_a - 2] : 0;
        s_re = j_b >= j_a ? rec_end[j_b - 1] : s_rs;
        const int32_t *ik = G.in_key + S.in_off;
        s_ilo = lower_bound_key(ik, 0, S.n_in_spikes, (int32_t)(4 * (k_lo + 1)));
        s_ihi = lower_bound_key(ik, s_ilo, S.n_in_spikes, (int32_t)(4 * (k_lo + len + 1)));
    }
    __syncthreads();
    const int64_t rs = s_rs, re = s_re, ilo = s_ilo, ihi = s_ihi;
    if (re <= rs && ihi <= ilo) return;
    const uint16_t *rec = G.rec + S.rec_off;
    int lo = p_lo;
    while (lo < p_hi) {
        int hi = p_hi, cnt = 0;
        for (;;) {  // narrow the source range until its instances fit
            if (tid == 0) s_cnt = 0;
            __syncthreads();
            int c = 0;
            for (int64_t p = rs + tid; p < re; p += nt) {
                const int s = rec[p];
                c += (s >= lo && s < hi);
            }
            for (int64_t q = ilo + tid; q < ihi; q += nt) {
                const int s = S.n + G.in_src[S.in_off + q];
                c += (s >= lo && s < hi);
            }
            if (c) atomicAdd(&s_cnt, c);
            __syncthreads();
            cnt = s_cnt;
            __syncthreads();
            if (cnt <= kInstCap || hi - lo <= 1) break;
            hi = lo + (hi - lo) / 2;
        }
        if (cnt > kInstCap) {
            if (tid == 0) atomicOr(flags, FLAG_BUCKET_OVERFLOW);
            return;
        }
        if (cnt > 0) {
            // collect (source << 8 | step in segment)
            if (tid == 0) s_cnt = 0;
            __syncthreads();
            for (int j = j_a + warp; j <= j_b; j += nwarps) {
                const int64_t b = j >= 2 ? rec_end[j - 2] : 0, e = rec_end[j - 1];
                const int kk = arr_step[j] - (int)k_lo - 1;
                for (int64_t p = b + lane; p < e; p += 32) {
                    const int s = rec[p];
                    if (s >= lo && s < hi) keys[atomicAdd(&s_cnt, 1)] = ((uint32_t)s << 8) | (uint32_t)kk;
                }
            }
            for (int64_t q = ilo + tid; q < ihi; q += nt) {
                const int s = S.n + G.in_src[S.in_off + q];
                if (s >= lo && s < hi) {
                    const int kk = G.in_key[S.in_off + q] / 4 - (int)k_lo - 1;
                    keys[atomicAdd(&s_cnt, 1)] = ((uint32_t)s << 8) | (uint32_t)kk;
                }
            }
            __syncthreads();
            // bitonic sort of the keys (padded to a power of two)
            int np = 1;
            while (np < cnt) np <<= 1;
            for (int x = cnt + tid; x < np; x += nt) keys[x] = 0xffffffffu;
            __syncthreads();
            for (int size = 2; size <= np; size <<= 1)
                for (int stride = size >> 1; stride > 0; stride >>= 1) {
                    for (int x = tid; x < np; x += nt) {
                        const int y = x ^ stride;
                        if (y > x) {
                            const uint32_t a = keys[x], b = keys[y];
                            const bool up = (x & size) == 0;
                            if ((a > b) == up) { keys[x] = b; keys[y] = a; }
                        }
                    }
                    __syncthreads();
                }
            // runs of one source
            if (tid == 0) s_runs = 0;
            __syncthreads();
            for (int x = tid; x < cnt; x += nt)
                if (x == 0 || (keys[x] >> 8) != (keys[x - 1] >> 8)) runs[atomicAdd(&s_runs, 1)] = x;
            __syncthreads();
            const int nr = s_runs;
            for (int r = warp; r < nr; r += nwarps) {
                const int a = runs[r];
                const uint32_t src = keys[a] >> 8;
                int b = a + 1;
                while (b < cnt && (keys[b] >> 8) == src) ++b;
                const bool inh = (int)src >= S.n_exc && (int)src < S.n;
                const float *mu = inh ? muI : muE;
                const uint32_t o0 = G.optr[S.src_off + src], o1 = G.optr[S.src_off + src + 1];
                for (uint32_t o = o0 + lane; o < o1; o += 32) {
                    const int64_t t = S.state_off + G.tgt[S.syn_off + o];
                    float acc = 0.0f;
                    for (int q = a; q < b; ++q) acc += mu[(int64_t)(keys[q] & 0xffu) * Nt + t];
                    gw[S.syn_off + o] += acc;
                }
            }
            __syncthreads();
        }
        lo = hi;
    }
}

// Per-network sums of the per-neuron partials, in a fixed order.
__global__ void k_adj_reduce(const SweepNet *nets, int64_t Nt, const double *gacc, double *out) {
    __shared__ double sh[256];
    const SweepNet &S = nets[blockIdx.x];
    for (int c = 0; c < 4; ++c) {
        double a = 0.0;
        for (int i = threadIdx.x; i < S.n; i += blockDim.x) a += gacc[c * Nt + S.state_off + i];
        sh[threadIdx.x] = a;
        __syncthreads();
        for (int st = blockDim.x >> 1; st > 0; st >>= 1) {
            if ((int)threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[blockIdx.x * 4 + c] = sh[0];
        __syncthreads();
    }
}

__global__ void k_perm_scatter_grad(const int64_t *perm, int64_t m, const float *src, float *dst) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < m; p += (int64_t)gridDim.x * blockDim.x)
        dst[perm[p]] = src[p];
}

using AdjFn = void (*)(SweepDev, const SweepNet *, int64_t, int, int64_t, const float *, const int32_t *, float *,
                       float *, float *, double *, float *, float *, int);

AdjFn adj_fn(int integ) {
    switch (integ) {
    case INTEG_EULER: return k_adj_neuron<INTEG_EULER>;
    case INTEG_RK2: return k_adj_neuron<INTEG_RK2>;
    default: return k_adj_neuron<INTEG_RK4>;
    }
}

int adj_alloc(eb_sweep *h, void **p, size_t b) { return h->dalloc(p, b); }

}  // namespace

extern "C" int eb_sweep_adjoint(eb_sweep *h, const float *grad_trace, int gt_on_device, float *grad_w,
                                int gw_on_device, double *grad_params) {
    if (!h || !h->built) { set_error("eb_sweep_adjoint: sweep not built"); return EB_ERR_STATE; }
    if (h->ckpt_every <= 0 || h->ckpt_upto != h->steps_done || h->steps_done <= 0 || h->needs_reset) {
        set_error("eb_sweep_adjoint: needs a checkpointed run from step 0 (eb_sweep_set_checkpoints, eb_sweep_reset, eb_sweep_run)");
        return EB_ERR_STATE;
    }
    if (h->G.n_obs <= 0 || !grad_trace) { set_error("eb_sweep_adjoint: no observed neurons or no trace gradient"); return EB_ERR_ARG; }
    SK(cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    const int E = h->ckpt_every;
    const int64_t S = h->steps_done, Nt = h->state_n;
    const int nseg = (int)((S + E - 1) / E);
    int rc;
    // scratch, allocated once for the checkpoint interval
    if (h->traj_steps < E) {
        if ((rc = adj_alloc(h, (void **)&h->G.tV, sizeof(float) * (size_t)E * Nt))) return rc;
        if ((rc = adj_alloc(h, (void **)&h->G.tE, sizeof(float) * (size_t)E * Nt))) return rc;
        if ((rc = adj_alloc(h, (void **)&h->G.tI, sizeof(float) * (size_t)E * Nt))) return rc;
        if ((rc = adj_alloc(h, (void **)&h->G.tcode, (size_t)E * Nt))) return rc;
        if ((rc = adj_alloc(h, (void **)&h->muE, sizeof(float) * (size_t)E * Nt))) return rc;
        if ((rc = adj_alloc(h, (void **)&h->muI, sizeof(float) * (size_t)E * Nt))) return rc;
        h->traj_steps = E;
    }
    if (!h->lamV) {
        if ((rc = adj_alloc(h, (void **)&h->lamV, sizeof(float) * (size_t)Nt))) return rc;
        if ((rc = adj_alloc(h, (void **)&h->lamE, sizeof(float) * (size_t)Nt))) return rc;
        if ((rc = adj_alloc(h, (void **)&h->lamI, sizeof(float) * (size_t)Nt))) return rc;
        if ((rc = adj_alloc(h, (void **)&h->gacc, sizeof(double) * 4 * (size_t)Nt))) return rc;
        if ((rc = adj_alloc(h, (void **)&h->gw_sorted, sizeof(float) * (size_t)std::max<int64_t>(1, h->total_syn)))) return rc;
        if ((rc = adj_alloc(h, (void **)&h->obs_slot, sizeof(int32_t) * (size_t)Nt))) return rc;
        if ((rc = adj_alloc(h, (void **)&h->red_out, sizeof(double) * 4 * (size_t)h->n_nets))) return rc;
    }
    // observed slot of every neuron (-1: not observed)
    {
        std::vector<int32_t> slot(Nt, -1);
        const int m = h->G.n_obs;
        for (int i = 0; i < h->n_nets; ++i)
            for (int q = 0; q < m; ++q) slot[h->nets[i].state_off + h->h_obs[(size_t)i * m + q]] = q;
        SK(cudaMemcpyAsync(h->obs_slot, slot.data(), sizeof(int32_t) * Nt, cudaMemcpyHostToDevice, st));
        SK(cudaStreamSynchronize(st));
    }
    const float *gt = grad_trace;
    float *gt_tmp = nullptr;
    const size_t gt_n = (size_t)h->n_nets * S * h->G.n_obs;
    if (!gt_on_device) {
        SK(cudaMallocAsync((void **)&gt_tmp, sizeof(float) * gt_n, st));
        SK(cudaMemcpyAsync(gt_tmp, grad_trace, sizeof(float) * gt_n, cudaMemcpyHostToDevice, st));
        gt = gt_tmp;
    }
    SK(cudaMemsetAsync(h->lamV, 0, sizeof(float) * Nt, st));
    SK(cudaMemsetAsync(h->lamE, 0, sizeof(float) * Nt, st));
    SK(cudaMemsetAsync(h->lamI, 0, sizeof(float) * Nt, st));
    SK(cudaMemsetAsync(h->gacc, 0, sizeof(double) * 4 * Nt, st));
    SK(cudaMemsetAsync(h->gw_sorted, 0, sizeof(float) * (size_t)std::max<int64_t>(1, h->total_syn), st));
    SK(cudaMemsetAsync(h->G.flags, 0, sizeof(uint32_t), st));
    const AdjFn fa = adj_fn(h->integ);
    const dim3 ga((h->max_n + 255) / 256, h->n_nets);
    const int parts = std::max(1, (2 * 148 + h->n_nets - 1) / h->n_nets);
    const std::vector<int32_t> &arr = h->h_arr_step;
    for (int s = nseg - 1; s >= 0; --s) {
        const int64_t k_lo = (int64_t)s * E;
        const int len = (int)std::min<int64_t>(E, S - k_lo);
        if ((rc = checkpoint_restore(h, s, k_lo, st))) break;
        if ((rc = enqueue_chunk(h, len, st, true, k_lo))) break;
        fa<<<ga, 256, 0, st>>>(h->G, h->d_nets, k_lo, len, S, gt, h->obs_slot, h->lamV, h->lamE, h->lamI, h->gacc,
                               h->muE, h->muI, s == 0 ? 1 : 0);
        // source steps whose spikes arrive in the segment
        const int32_t k1 = (int32_t)(k_lo + 1), k2 = (int32_t)(k_lo + len);
        int j_a = (int)(std::lower_bound(arr.begin() + 1, arr.end(), k1) - arr.begin());
        int j_b = (int)(std::upper_bound(arr.begin() + 1, arr.end(), k2) - arr.begin()) - 1;
        k_adj_wgrad<<<dim3(h->n_nets, parts), 256, 0, st>>>(h->G, h->d_nets, h->d_arr_step, k_lo, len, j_a, j_b,
                                                            h->muE, h->muI, h->gw_sorted, h->G.flags);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { set_error("adjoint kernels: %s", cudaGetErrorString(e)); rc = EB_ERR_CUDA; break; }
    }
    if (gt_tmp) cudaFreeAsync(gt_tmp, st);
    h->needs_reset = true;
    if (rc) return rc;
    k_adj_reduce<<<h->n_nets, 256, 0, st>>>(h->d_nets, Nt, h->gacc, h->red_out);
    SK(cudaGetLastError());
    if (grad_w && h->total_syn) {
        float *dst = grad_w, *tmp = nullptr;
        if (!gw_on_device) {
            SK(cudaMallocAsync((void **)&tmp, sizeof(float) * h->total_syn, st));
            dst = tmp;
        }
        k_perm_scatter_grad<<<592, 256, 0, st>>>(h->perm, h->total_syn, h->gw_sorted, dst);
        SK(cudaGetLastError());
        if (tmp) {
            SK(cudaMemcpyAsync(grad_w, tmp, sizeof(float) * h->total_syn, cudaMemcpyDeviceToHost, st));
            SK(cudaFreeAsync(tmp, st));
        }
    }
    std::vector<double> red(4 * (size_t)h->n_nets);
    SK(cudaMemcpyAsync(red.data(), h->red_out, sizeof(double) * red.size(), cudaMemcpyDeviceToHost, st));
    uint32_t flags = 0;
    SK(cudaMemcpyAsync(&flags, h->G.flags, sizeof(flags), cudaMemcpyDeviceToHost, st));
    SK(cudaStreamSynchronize(st));
    if (flags) { set_error("eb_sweep_adjoint: a source spiked more than %d times in one segment", kInstCap); return EB_ERR_OVERFLOW; }
    // d(decay)/d(tau) = decay * el / tau^2 with decay = exp(-el / tau)
    const double el = (h->integ == INTEG_RK4) ? (double)(h->dt * 1000.0f * 0.5f) : (double)(h->dt * 1000.0f);
    if (grad_params)
        for (int i = 0; i < h->n_nets; ++i) {
            const SweepNet &Sn = h->nets[i];
            const double te = Sn.params[5], ti = Sn.params[6];
            grad_params[4 * i + 0] = red[4 * i + 0];
            grad_params[4 * i + 1] = red[4 * i + 1];
            grad_params[4 * i + 2] = red[4 * i + 2] * (double)Sn.L.decay[0] * el / (te * te);
            grad_params[4 * i + 3] = red[4 * i + 3] * (double)Sn.L.decay[1] * el / (ti * ti);
        }
    return EB_OK;
}
