// Device-side neuron models and integrators of the time-driven hot path.
//
// One thread (or one warp lane) owns one neuron; the integrator stages live in
// registers.  The arithmetic follows the reference CPU models operation by
// operation (same float/double promotions, same lookup tables computed on the
// host, no FMA contraction: the library is compiled with --fmad=false), so a
// neuron update here produces the same float32 bits as the reference:
//   LIF  src/neuron_model/LIFTimeDrivenModel.cpp:160-242
//   AdEx src/neuron_model/AdExTimeDrivenModel.cpp:157-235
//   HH   src/neuron_model/HHTimeDrivenModel.cpp:188-276, rate table HHTimeDrivenModel.h:372-441
//   Euler include/integration_method/Euler.h:123-146, RK2 RK2.h:133-165,
//   RK4 RK4.h:167-231, BDFn BDFn.h:288-420 (Jacobian :704-724, inverse :735-797).
#pragma once
#include <cstdint>
#include "eb_types.h"

namespace eb {

constexpr float kExptMin = -20.0f;
constexpr float kExptMax = 20.0f;
constexpr float kHHMinV = -90.0f;

// ExponentialTable::GetResult (include/simulation/ExponentialTable.h:92-103).
__device__ __forceinline__ float expt(const PopDev &P, float v) {
    if (v >= kExptMin && v <= kExptMax) {
        int pos = (int)((v - kExptMin) * P.expt_aux);
        return __ldg(P.exp_table + pos);
    }
    if (v > kExptMax) return (float)exp((double)v);
    return 0.0f;
}

__device__ __forceinline__ float nmda_inf(const PopDev &P, float v, float e_inh) {
    int pos = (int)((v - e_inh) * P.nmda_aux);
    if (pos < 0) pos = 0; else if (pos > kNmdaTable - 1) pos = kNmdaTable - 1;
    return __ldg(P.nmda_table + pos);
}

// Enabled conductance types of a population (bit 0 AMPA, 1 GABA, 2 NMDA): the
// template value when a kernel is specialised for it (EN >= 0), else P.en.
template <int EN>
__device__ __forceinline__ int en_mask(const PopDev &P) { return EN >= 0 ? EN : P.en; }

// -------------------------------------------------------------------- LIF --
// Refractory state of one update: the reference's derivative decides from
// l = LastSpikeTime (ms) against tau_ref on every call; the decision only depends
// on the update count since the last spike, so it is taken once per update with
// the same double arithmetic and the derivative calls apply it.
struct Refr {
    int mode;    // 0: free (full derivative), 1: partial (fraction * full), 2: refractory (0)
    float frac;  // fraction of mode 1
};

// refr = updates since the last spike (-1: never spiked, LastSpikeTime >= 100 s).
// LastSpikeTime = refr * dt exactly, because every partial sum of the reference's
// double accumulation is exact.
__device__ __forceinline__ Refr lif_refr(const PopDev &P, int refr) {
    Refr r{0, 1.0f};
    if (refr < 0) return r;
    const double tref = (double)P.p[7];
    const double l = ((double)refr * (double)P.dt_s) * 1000.0;
    if (l > tref) return r;
    if (l + (double)P.dt_ms > tref) {
        r.mode = 1;
        r.frac = (float)((l + (double)P.dt_ms - tref) / (double)P.dt_ms);
    } else {
        r.mode = 2;
    }
    return r;
}

// x = {V, gE, gI, gNMDA}
template <int EN = -1>
__device__ __forceinline__ void lif_deriv(const PopDev &P, const float *x, float *dx, Refr rf) {
    const float *p = P.p;  // e_exc e_inh e_leak v_thr c_m tau_exc tau_inh tau_ref g_leak tau_nmda
    const int en = en_mask<EN>(P);
    float current = 0.0f;
    if (en & 1) current += x[1] * (p[0] - x[0]);
    if (en & 2) current += x[2] * (p[1] - x[0]);
    if (en & 4) current += x[3] * nmda_inf(P, x[0], p[1]) * (p[0] - x[0]);
    const float full = (current + p[8] * (p[2] - x[0])) * P.inv_c_m;
    dx[0] = rf.mode == 0 ? full : rf.mode == 1 ? rf.frac * full : 0.0f;
}

// ------------------------------------------------------------------- AdEx --
// p = a b thr_slo_fac v_thr tau_w e_exc e_inh e_reset e_leak g_leak c_m tau_exc tau_inh tau_nmda
// x = {V, w, gE, gI, gNMDA}
template <int EN = -1>
__device__ __forceinline__ void adex_deriv(const PopDev &P, const float *x, float *dx) {
    const float *p = P.p;
    const float a = p[0], slope = p[2], vthr = p[3], eexc = p[5], einh = p[6], eleak = p[8], gl = p[9];
    const int en = en_mask<EN>(P);
    // P.adex_vmax = vthr + 6 * slope and P.adex_glslope = gl * slope: the same float
    // operations, evaluated once on the host
    if (x[0] <= P.adex_vmax) {
        float current = 0.0f;
        if (en & 1) current += x[2] * (eexc - x[0]);
        if (en & 2) current += x[3] * (einh - x[0]);
        if (en & 4) current += x[4] * nmda_inf(P, x[0], einh) * (eexc - x[0]);
        dx[0] = (gl * (eleak - x[0]) + P.adex_glslope * expt(P, (x[0] - vthr) * P.inv_slope) - x[1] + current) * P.inv_c_m;
        dx[1] = (a * (x[0] - eleak) - x[1]) * P.inv_tau_w;
    } else if (x[0] <= 0.0f) {
        const float Vm = vthr + 6 * slope;
        float current = 0.0f;
        if (en & 1) current += x[2] * (eexc - Vm);
        if (en & 2) current += x[3] * (einh - Vm);
        if (en & 4) current += x[4] * nmda_inf(P, Vm, einh) * (eexc - Vm);
        dx[0] = (gl * (eleak - Vm) + gl * slope * expt(P, (Vm - vthr) * P.inv_slope) - x[1] + current) * P.inv_c_m;
        dx[1] = (a * (x[0] - eleak) - x[1]) * P.inv_tau_w;
    } else {
        dx[0] = 0.0f;
        dx[1] = 0.0f;
    }
}

// --------------------------------------------------------------------- HH --
// Partial results of one HH derivative evaluation: the rates at V and the partial
// sums of dV/dt, left to right as the reference adds them: s0 = current +
// gl (eleak - V), a3 = gna m m m, sA = s0 + a3 h (ena - V), B = gkd n n n n (ek - V).
struct HHParts {
    float am, bm, ah, bh, an, bn;
    float s0, a3, sA, B;
};

// p = e_exc e_inh e_leak g_leak c_m v_thr tau_exc tau_inh tau_nmda g_na g_kd e_na e_k
// x = {V, m, h, n, gE, gI, gNMDA}.  The clamps write the state passed in, as the
// reference does (HHTimeDrivenModel.cpp:197-222).
template <int EN = -1>
__device__ __forceinline__ void hh_deriv(const PopDev &P, float *x, float *dx, HHParts &R) {
    const int en = en_mask<EN>(P);
    const float *p = P.p;
    const float eexc = p[0], einh = p[1], eleak = p[2], gl = p[3], gna = p[9], gkd = p[10], ena = p[11], ek = p[12];
    if (x[0] < ek) x[0] = ek;
    if (x[0] > ena - 1.0f) x[0] = ena - 1.0f;
    if (x[1] < 0) x[1] = 0.0f;
    if (x[1] > 1) x[1] = 1.0f;
    if (x[2] < 0) x[2] = 0.0f;
    if (x[2] > 1) x[2] = 1.0f;
    if (x[3] < 0) x[3] = 0.0f;
    if ((double)x[3] > 0.72) x[3] = 0.72f;
    const float V = x[0], m = x[1], h = x[2], n = x[3];
    int pos = (int)((V - kHHMinV) * P.hh_aux);
    if (pos < 0) pos = 0; else if (pos > kHHTable - 1) pos = kHHTable - 1;
    const float *r = P.hh_table + (size_t)pos * 6;
    const float am = __ldg(r + 0), bm = __ldg(r + 1), ah = __ldg(r + 2), bh = __ldg(r + 3), an = __ldg(r + 4), bn = __ldg(r + 5);
    float current = 0.0f;
    if (en & 1) current += x[4] * (eexc - x[0]);
    if (en & 2) current += x[5] * (einh - x[0]);
    if (en & 4) current += x[6] * nmda_inf(P, x[0], einh) * (eexc - x[0]);
    // (current + gl (eleak - V) + gna m m m h (ena - V) + gkd n n n n (ek - V)) / c_m
    const float s0 = current + gl * (eleak - V);
    const float a3 = gna * m * m * m;
    const float sA = s0 + a3 * h * (ena - V);
    const float B = gkd * n * n * n * n * (ek - V);
    dx[0] = (sA + B) * P.inv_c_m;
    dx[1] = (am * (1.0f - m) - bm * m);
    dx[2] = (ah * (1.0f - h) - bh * h);
    dx[3] = (an * (1.0f - n) - bn * n);
    R = HHParts{am, bm, ah, bh, an, bn, s0, a3, sA, B};
}

template <int EN = -1>
__device__ __forceinline__ void hh_deriv(const PopDev &P, float *x, float *dx) {
    HHParts R;
    hh_deriv<EN>(P, x, dx, R);
}

// Columns m, h, n of the BDF Jacobian, (f(x) - f(x - eps e_j)) / eps, where x was
// clamped by the evaluation that gave f(x) = fx and R.  Displacing one gate leaves
// V, hence the rates, and the other gates' derivatives unchanged: their
// differences are exactly zero, and dV/dt only needs its displaced term.  The
// displaced gate is clamped as the full evaluation would clamp it, so every entry
// is the full evaluation's bit for bit.
__device__ __forceinline__ void hh_gate_columns(const PopDev &P, const float *x, const float *fx, const HHParts &R,
                                                float eps, float inv_eps, float *jac) {
    const float *p = P.p;
    const float gna = p[9], gkd = p[10], ena = p[11], ek = p[12];
    const float V = x[0], m = x[1], h = x[2], n = x[3];
    float m2 = m - eps;
    if (m2 < 0) m2 = 0.0f;
    if (m2 > 1) m2 = 1.0f;
    const float dm0 = (R.s0 + gna * m2 * m2 * m2 * h * (ena - V) + R.B) * P.inv_c_m;
    const float dm1 = R.am * (1.0f - m2) - R.bm * m2;
    float h2 = h - eps;
    if (h2 < 0) h2 = 0.0f;
    if (h2 > 1) h2 = 1.0f;
    const float dh0 = (R.s0 + R.a3 * h2 * (ena - V) + R.B) * P.inv_c_m;
    const float dh2 = R.ah * (1.0f - h2) - R.bh * h2;
    float n2 = n - eps;
    if (n2 < 0) n2 = 0.0f;
    if ((double)n2 > 0.72) n2 = 0.72f;
    const float dn0 = (R.sA + gkd * n2 * n2 * n2 * n2 * (ek - V)) * P.inv_c_m;
    const float dn3 = R.an * (1.0f - n2) - R.bn * n2;
    jac[0 * 4 + 1] = (fx[0] - dm0) * inv_eps;
    jac[1 * 4 + 1] = (fx[1] - dm1) * inv_eps;
    jac[2 * 4 + 1] = 0.0f;
    jac[3 * 4 + 1] = 0.0f;
    jac[0 * 4 + 2] = (fx[0] - dh0) * inv_eps;
    jac[1 * 4 + 2] = 0.0f;
    jac[2 * 4 + 2] = (fx[2] - dh2) * inv_eps;
    jac[3 * 4 + 2] = 0.0f;
    jac[0 * 4 + 3] = (fx[0] - dn0) * inv_eps;
    jac[1 * 4 + 3] = 0.0f;
    jac[2 * 4 + 3] = 0.0f;
    jac[3 * 4 + 3] = (fx[3] - dn3) * inv_eps;
}

template <int KIND> struct Model;
template <> struct Model<KIND_LIF> {
    static constexpr int ND = 1, NV = 4;
    template <int EN = -1>
    __device__ static void deriv(const PopDev &P, float *x, float *dx, Refr rf) { lif_deriv<EN>(P, x, dx, rf); }
};
template <> struct Model<KIND_ADEX> {
    static constexpr int ND = 2, NV = 5;
    template <int EN = -1>
    __device__ static void deriv(const PopDev &P, float *x, float *dx, Refr) { adex_deriv<EN>(P, x, dx); }
};
template <> struct Model<KIND_HH> {
    static constexpr int ND = 4, NV = 7;
    template <int EN = -1>
    __device__ static void deriv(const PopDev &P, float *x, float *dx, Refr) { hh_deriv<EN>(P, x, dx); }
};

// EvaluateTimeDependentEquation: g <- 0 below 1e-9, else g * factor (enabled types only).
template <int ND, int EN = -1>
__device__ __forceinline__ void decay(const PopDev &P, float *x) {
    const float limit = 1e-9;
    const int en = en_mask<EN>(P);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (!(en & (1 << c))) continue;
        if (x[ND + c] < limit) x[ND + c] = 0.0f;
        else x[ND + c] *= P.decay[c];
    }
}

// Gauss-Jordan inverse with the reference's zero-pivot row swap (BDFn.h:735-797).
template <int N>
__device__ __forceinline__ bool invermat(const float *a, float *ainv) {
    if constexpr (N == 1) {
        ainv[0] = 1.0f / a[0];
        return true;
    }
    float la[N * N], li[N * N];
#pragma unroll
    for (int i = 0; i < N * N; ++i) { la[i] = a[i]; li[i] = 0.0f; }
#pragma unroll
    for (int i = 0; i < N; ++i) li[i * N + i] = 1.0f;
#pragma unroll
    for (int s = 0; s < N; ++s) {
        float el = la[s * N + s];
        if (el == 0) {
            bool found = false;
#pragma unroll
            for (int r = s + 1; r < N; ++r) {
                if (found) break;
                el = la[r * N + s];
                if (el != 0) {
#pragma unroll
                    for (int c = 0; c < N; ++c) {
                        float v = la[r * N + c]; la[r * N + c] = la[s * N + c]; la[s * N + c] = v;
                        v = li[r * N + c]; li[r * N + c] = li[s * N + c]; li[s * N + c] = v;
                    }
                    found = true;
                } else if (r == N - 1) {
                    return false;
                }
            }
        }
        const float inv = 1.0f / el;
#pragma unroll
        for (int c = 0; c < N; ++c) { la[s * N + c] *= inv; li[s * N + c] *= inv; }
#pragma unroll
        for (int r = 0; r < N; ++r) {
            if (r == s) continue;
            const float coef = -la[r * N + s];
#pragma unroll
            for (int c = 0; c < N; ++c) {
                la[r * N + c] += la[s * N + c] * coef;
                li[r * N + c] += li[s * N + c] * coef;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < N * N; ++i) ainv[i] = li[i];
    return true;
}

// Per-neuron BDF history, SoA in global memory: D[q][v][n], P[q][v][n].
struct BdfRef {
    float *D, *Pv;
    int64_t stride;  // population size
    int64_t i;
    __device__ float &d(int q, int v, int nd) const { return D[((int64_t)q * nd + v) * stride + i]; }
    __device__ float &pv(int q, int v, int nd) const { return Pv[((int64_t)q * nd + v) * stride + i]; }
};

// One integration step of one neuron.  x holds all NV state variables.  Returns
// false only if the BDF Newton matrix was singular.
template <int KIND, int INTEG, int EN = -1>
__device__ __forceinline__ bool integrate(const PopDev &P, float *x, int refr, int &bdf_state, const BdfRef &H) {
    using M = Model<KIND>;
    constexpr int ND = M::ND, NV = M::NV;
    const float dt = P.dt_ms;
    float k1[NV], k2[NV], k3[NV], k4[NV], aux[NV];
    const Refr rf = (KIND == KIND_LIF) ? lif_refr(P, refr) : Refr{0, 1.0f};
    if (INTEG == INTEG_EULER) {
        M::template deriv<EN>(P, x, k1, rf);
#pragma unroll
        for (int j = 0; j < ND; ++j) x[j] += dt * k1[j];
        decay<ND, EN>(P, x);
    } else if (INTEG == INTEG_RK2) {
        M::template deriv<EN>(P, x, k1, rf);
#pragma unroll
        for (int j = 0; j < ND; ++j) x[j] += k1[j] * dt;
        decay<ND, EN>(P, x);
        M::template deriv<EN>(P, x, k2, rf);
#pragma unroll
        for (int j = 0; j < ND; ++j) x[j] += (-k1[j] + k2[j]) * dt * 0.5f;
    } else if (INTEG == INTEG_RK4) {
        const float h05 = dt * 0.5f;
        const float h016 = dt * 0.166666666667f;
        M::template deriv<EN>(P, x, k1, rf);
#pragma unroll
        for (int j = 0; j < ND; ++j) aux[j] = x[j] + k1[j] * h05;
#pragma unroll
        for (int j = ND; j < NV; ++j) aux[j] = x[j];
        decay<ND, EN>(P, aux);
        M::template deriv<EN>(P, aux, k2, rf);
#pragma unroll
        for (int j = 0; j < ND; ++j) aux[j] = x[j] + k2[j] * h05;
        M::template deriv<EN>(P, aux, k3, rf);
#pragma unroll
        for (int j = 0; j < ND; ++j) aux[j] = x[j] + k3[j] * dt;
        decay<ND, EN>(P, aux);
        M::template deriv<EN>(P, aux, k4, rf);
#pragma unroll
        for (int j = 0; j < ND; ++j) x[j] += (k1[j] + 2.0f * (k2[j] + k3[j]) + k4[j]) * h016;
#pragma unroll
        for (int j = ND; j < NV; ++j) x[j] = aux[j];
    } else {  // BDFn
        int st = bdf_state;
        float pr[NV], p1[ND], c[ND], jac[ND * ND], J[ND * ND], iJ[ND * ND];
        if (st == 0) {
            M::template deriv<EN>(P, x, aux, rf);
#pragma unroll
            for (int j = 0; j < ND; ++j) pr[j] = x[j] + dt * aux[j];
        } else {
#pragma unroll
            for (int j = 0; j < ND; ++j) {
                pr[j] = x[j];
                for (int q = 0; q < st; ++q) pr[j] += H.d(q, j, ND);
            }
        }
#pragma unroll
        for (int j = ND; j < NV; ++j) pr[j] = x[j];
        decay<ND, EN>(P, pr);
        const float *co = P.bdf_coef[st];
        float hist[6][ND];
        for (int q = 1; q < st; ++q)
#pragma unroll
            for (int j = 0; j < ND; ++j) hist[q - 1][j] = H.pv(q - 1, j, ND);
        float epsi = 1.0f;
        int k = 0;
        const float eps_j = dt * 0.1f;
        const float inv_eps = 1.0f / eps_j;
        HHParts R;
        while (epsi > 1e-6 && k < 10) {
            if constexpr (KIND == KIND_HH) hh_deriv<EN>(P, pr, aux, R);
            else M::template deriv<EN>(P, pr, aux, rf);
#pragma unroll
            for (int j = 0; j < ND; ++j) {
                c[j] = co[0] * dt * aux[j] + co[1] * x[j];
                for (int q = 1; q < st; ++q) c[j] += co[q + 1] * hist[q - 1][j];
            }
            // Jacobian: one-sided difference at eps = 0.1 dt (BDFn.h:704-724).  Its
            // base point is f(pr), already in aux: deriv clamps its argument in
            // place before evaluating (HH) and clamping twice changes nothing, so
            // evaluating it again would give the same values bit for bit.
            if constexpr (KIND == KIND_HH) {
                float tmp[NV], neg[NV];
#pragma unroll
                for (int v = 0; v < NV; ++v) tmp[v] = pr[v];
                tmp[0] -= eps_j;
                M::template deriv<EN>(P, tmp, neg, rf);
#pragma unroll
                for (int z = 0; z < ND; ++z) jac[z * ND] = (aux[z] - neg[z]) * inv_eps;
                hh_gate_columns(P, pr, aux, R, eps_j, inv_eps, jac);
            } else {
                float tmp[NV], neg[NV];
                const float *pos = aux;
#pragma unroll
                for (int j = 0; j < ND; ++j) {
#pragma unroll
                    for (int v = 0; v < NV; ++v) tmp[v] = pr[v];
                    tmp[j] -= eps_j;
                    M::template deriv<EN>(P, tmp, neg, rf);
#pragma unroll
                    for (int z = 0; z < ND; ++z) jac[z * ND + j] = (pos[z] - neg[z]) * inv_eps;
                }
            }
#pragma unroll
            for (int z = 0; z < ND; ++z)
#pragma unroll
                for (int t = 0; t < ND; ++t) {
                    J[z * ND + t] = co[0] * dt * jac[z * ND + t];
                    if (z == t) J[z * ND + t] -= 1;
                }
            if (!invermat<ND>(J, iJ)) return false;
#pragma unroll
            for (int z = 0; z < ND; ++z) {
                float a = 0.0f;
#pragma unroll
                for (int t = 0; t < ND; ++t) a += iJ[z * ND + t] * (pr[t] - c[t]);
                p1[z] = a + pr[z];
            }
            float mx = 0.0f;
#pragma unroll
            for (int z = 0; z < ND; ++z) {
                float d = fabsf(p1[z] - pr[z]);
                if (d > mx) mx = d;
            }
#pragma unroll
            for (int z = 0; z < ND; ++z) pr[z] = p1[z];
            epsi = mx;
            k++;
        }
        if (st < P.bdf_order) st++;
        bdf_state = st;
#pragma unroll
        for (int j = 0; j < ND; ++j) {
            float dq[7];
            for (int q = 0; q < st; ++q) dq[q] = H.d(q, j, ND);
            for (int q = st - 1; q > 0; --q) dq[q] = -dq[q - 1];
            dq[0] = pr[j] - x[j];
            for (int q = 1; q < st; ++q) dq[q] += dq[q - 1];
            for (int q = 0; q < st; ++q) H.d(q, j, ND) = dq[q];
        }
        if (st > 1) {
            for (int q = st - 2; q > 0; --q)
#pragma unroll
                for (int j = 0; j < ND; ++j) H.pv(q, j, ND) = hist[q - 1][j];
#pragma unroll
            for (int j = 0; j < ND; ++j) H.pv(0, j, ND) = x[j];
        }
#pragma unroll
        for (int j = 0; j < ND; ++j) x[j] = pr[j];
        decay<ND, EN>(P, x);
    }
    return true;
}

// EvaluateSpikeCondition of the three models.  Returns true on a spike; sets
// reset when the model restarts its integrator history (LIF, AdEx; not HH).
template <int KIND>
__device__ __forceinline__ bool spike_condition(const PopDev &P, float *x, float prevV, bool &reset) {
    reset = false;
    if (KIND == KIND_LIF) {
        if (x[0] > P.p[3]) { x[0] = P.p[2]; reset = true; return true; }
    } else if (KIND == KIND_ADEX) {
        if (x[0] > 0.0f) { x[0] = P.p[7]; x[1] += P.p[1]; reset = true; return true; }
    } else {
        if (x[0] > -30.0f && prevV < -30.0f) return true;
    }
    return false;
}

}  // namespace eb
