/* TEST INFRASTRUCTURE ONLY -- part of the CPU oracle (see edlut_oracle.c).
 *
 * Per-neuron model and integrator arithmetic, written once and instantiated
 * twice by edlut_oracle.c:
 *   R=float  (ORACLE_F32=1): mirrors the reference CPU twins operation by
 *            operation, including their lookup tables and mixed float/double
 *            promotions, so results are bit-identical to the reference;
 *   R=double (ORACLE_F32=0): the same equations in FP64 with exact exp(),
 *            the error yardstick.
 * Every function cites the reference code it restates (paths relative to the
 * reference's Kernel/ directory).
 */

/* ---------------------------------------------------------------- tables -- */
/* ExponentialTable::GetResult, include/simulation/ExponentialTable.h:92-103. */
static R SFX(expt)(R v) {
#if ORACLE_F32
    if (v >= EXPT_MIN && v <= EXPT_MAX) {
        int pos = (int)((v - EXPT_MIN) * EXPT_AUX);
        return g_exptable[pos];
    }
    if (v > EXPT_MAX) return (float)exp((double)v);
    return 0.0f;
#else
    return exp(v);
#endif
}

/* HH channel rates: table in HHTimeDrivenModel.h:372-441 (f32) or closed form (f64). */
static void SFX(hh_rates)(const eo_popstate *ps, R V, R out[6]) {
#if ORACLE_F32
    int pos = (int)((V - HH_MIN_V) * HH_AUX);
    if (pos < 0) pos = 0; else if (pos > HH_TABLE - 1) pos = HH_TABLE - 1;
    const float *t = ps->hh_table + (size_t)pos * 6;
    for (int i = 0; i < 6; ++i) out[i] = t[i];
#else
    double vt = ps->p[5];
    double x = 13.0 - V + vt;
    out[0] = (x == 0.0) ? 1.28 : 0.32 * x / (exp(x * 0.25) - 1.0);
    x = V - vt - 40.0;
    out[1] = (x == 0.0) ? 1.4 : 0.28 * x / (exp(x * 0.2) - 1.0);
    out[2] = 0.128 * exp((17.0 - V + vt) / 18.0);
    out[3] = 4.0 / (1.0 + exp((40.0 - V + vt) * 0.2));
    x = 15.0 - V + vt;
    out[4] = (x == 0.0) ? 0.16 : 0.032 * x / (exp(x * 0.2) - 1.0);
    out[5] = 0.5 * exp((10.0 - V + vt) * 0.025);
#endif
}

/* NMDA gating 1/(1+exp(-0.062 V) 1.2/3.57): table LIFTimeDrivenModel.cpp:26-50 (f32). */
static R SFX(nmda)(const eo_popstate *ps, R V, float e_exc, float e_inh) {
#if ORACLE_F32
    int pos = (int)((V - e_inh) * ps->nmda_aux);
    if (pos < 0) pos = 0; else if (pos > NMDA_TABLE - 1) pos = NMDA_TABLE - 1;
    return ps->nmda_table[pos];
#else
    (void)ps; (void)e_exc; (void)e_inh;
    return 1.0 / (1.0 + exp(-0.062 * V) * (1.2 / 3.57));
#endif
}

/* ---------------------------------------------------------- derivatives -- */
/* LIFTimeDrivenModel::EvaluateDifferentialEquation, LIFTimeDrivenModel.cpp:172-205.
 * x = {V, gE, gI, gNMDA, I_ext}; lst = LastSpikeTime (double seconds). */
static void SFX(lif_deriv)(const eo_popstate *ps, R *x, R *dx, double lst, float elapsed) {
    const float *p = ps->p;  /* e_exc e_inh e_leak v_thr c_m tau_exc tau_inh tau_ref g_leak tau_nmda */
    R current = 0.0f;
    if (ps->en[0]) current += x[1] * ((R)p[0] - x[0]);
    if (ps->en[1]) current += x[2] * ((R)p[1] - x[0]);
    if (ps->en[2]) current += x[3] * SFX(nmda)(ps, x[0], p[0], p[1]) * ((R)p[0] - x[0]);
    current += x[4];
    double l = lst * 1000.0;  /* GetLastSpikeTime * GetTimeScale() (float 1000) */
    R gl = p[8];
    R invc = ORACLE_F32 ? (R)ps->inv_c_m : (R)(1.0 / (double)p[4]);
    if (l > (double)p[7]) {
        dx[0] = (current + gl * ((R)p[2] - x[0])) * invc;
    } else if (l + (double)elapsed > (double)p[7]) {
        R fraction = (R)((l + (double)elapsed - (double)p[7]) / (double)elapsed);
        dx[0] = fraction * ((current + gl * ((R)p[2] - x[0])) * invc);
    } else {
        dx[0] = 0;
    }
}

/* AdExTimeDrivenModel::EvaluateDifferentialEquation, AdExTimeDrivenModel.cpp:170-213.
 * p = a b thr_slo_fac v_thr tau_w e_exc e_inh e_reset e_leak g_leak c_m tau_exc tau_inh tau_nmda
 * x = {V, w, gE, gI, gNMDA, I_ext}. */
static void SFX(adex_deriv)(const eo_popstate *ps, R *x, R *dx, double lst, float elapsed) {
    (void)lst; (void)elapsed;
    const float *p = ps->p;
    R a = p[0], slope = p[2], vthr = p[3], eexc = p[5], einh = p[6], eleak = p[8], gl = p[9];
    R inv_slope = ORACLE_F32 ? (R)ps->inv_thr_slo_fac : (R)(1.0 / (double)p[2]);
    R inv_tw = ORACLE_F32 ? (R)ps->inv_tau_w : (R)(1.0 / (double)p[4]);
    R invc = ORACLE_F32 ? (R)ps->inv_c_m : (R)(1.0 / (double)p[10]);
    R vcap = vthr + 6 * slope;
    if (x[0] <= vcap) {
        R current = 0.0f;
        if (ps->en[0]) current += x[2] * (eexc - x[0]);
        if (ps->en[1]) current += x[3] * (einh - x[0]);
        if (ps->en[2]) current += x[4] * SFX(nmda)(ps, x[0], p[5], p[6]) * (eexc - x[0]);
        current += x[5];
        dx[0] = (gl * (eleak - x[0]) + gl * slope * SFX(expt)((x[0] - vthr) * inv_slope) - x[1] + current) * invc;
        dx[1] = (a * (x[0] - eleak) - x[1]) * inv_tw;
    } else if (x[0] <= 0.0f) {
        R Vm = vthr + 6 * slope;
        R current = 0.0f;
        if (ps->en[0]) current += x[2] * (eexc - Vm);
        if (ps->en[1]) current += x[3] * (einh - Vm);
        if (ps->en[2]) current += x[4] * SFX(nmda)(ps, Vm, p[5], p[6]) * (eexc - Vm);
        current += x[5];
        dx[0] = (gl * (eleak - Vm) + gl * slope * SFX(expt)((Vm - vthr) * inv_slope) - x[1] + current) * invc;
        dx[1] = (a * (x[0] - eleak) - x[1]) * inv_tw;
    } else {
        dx[0] = 0;
        dx[1] = 0;
    }
}

/* HHTimeDrivenModel::EvaluateDifferentialEquation, HHTimeDrivenModel.cpp:196-255.
 * The clamps write the state that is passed in.
 * p = e_exc e_inh e_leak g_leak c_m v_thr tau_exc tau_inh tau_nmda g_na g_kd e_na e_k
 * x = {V, m, h, n, gE, gI, gNMDA, I_ext}. */
static void SFX(hh_deriv)(const eo_popstate *ps, R *x, R *dx, double lst, float elapsed) {
    (void)lst; (void)elapsed;
    const float *p = ps->p;
    R eexc = p[0], einh = p[1], eleak = p[2], gl = p[3], gna = p[9], gkd = p[10], ena = p[11], ek = p[12];
    R invc = ORACLE_F32 ? (R)ps->inv_c_m : (R)(1.0 / (double)p[4]);
    if (x[0] < ek) x[0] = ek;
    if (x[0] > ena - 1.0f) x[0] = ena - 1.0f;
    if (x[1] < 0) x[1] = 0.0f;
    if (x[1] > 1) x[1] = 1.0f;
    if (x[2] < 0) x[2] = 0.0f;
    if (x[2] > 1) x[2] = 1.0f;
    if (x[3] < 0) x[3] = 0.0f;
    if (x[3] > 0.72) x[3] = 0.72f;
    R V = x[0], m = x[1], h = x[2], n = x[3];
    R r[6];
    SFX(hh_rates)(ps, V, r);
    R current = 0.0f;
    if (ps->en[0]) current += x[4] * (eexc - x[0]);
    if (ps->en[1]) current += x[5] * (einh - x[0]);
    if (ps->en[2]) current += x[6] * SFX(nmda)(ps, x[0], p[0], p[1]) * (eexc - x[0]);
    current += x[7];
    dx[0] = (current + gl * (eleak - V) + gna * m * m * m * h * (ena - V) + gkd * n * n * n * n * (ek - V)) * invc;
    dx[1] = (r[0] * (1.0f - m) - r[1] * m);
    dx[2] = (r[2] * (1.0f - h) - r[3] * h);
    dx[3] = (r[4] * (1.0f - n) - r[5] * n);
}

static void SFX(deriv)(const eo_popstate *ps, R *x, R *dx, double lst, float elapsed) {
    switch (ps->kind) {
    case EO_LIF: SFX(lif_deriv)(ps, x, dx, lst, elapsed); break;
    case EO_ADEX: SFX(adex_deriv)(ps, x, dx, lst, elapsed); break;
    default: SFX(hh_deriv)(ps, x, dx, lst, elapsed); break;
    }
}

/* EvaluateTimeDependentEquation of the three models (e.g. LIFTimeDrivenModel.cpp:207-242):
 * g <- 0 below 1e-9, else g * factor, for the enabled conductance types only. */
static void SFX(decay)(const eo_popstate *ps, R *x, int half) {
    const float limit = 1e-9;
    int nd = ps->ndiff;
    for (int c = 0; c < 3; ++c) {
        if (!ps->en[c]) continue;
        R f = ORACLE_F32 ? (R)ps->decay_f32[half][c] : (R)ps->decay_f64[half][c];
        if (x[nd + c] < limit) x[nd + c] = 0.0f;
        else x[nd + c] *= f;
    }
}

/* EvaluateSpikeCondition: LIF LIFTimeDrivenModel.cpp:160-170, AdEx AdExTimeDrivenModel.cpp:157-168,
 * HH HHTimeDrivenModel.cpp:188-194.  Returns 1 on spike; *reset_bdf set when the integrator
 * state must restart (LIF/AdEx call resetState, HH does not). */
static int SFX(spike)(const eo_popstate *ps, R *x, R prevV, int *reset_bdf) {
    const float *p = ps->p;
    *reset_bdf = 0;
    if (ps->kind == EO_LIF) {
        if (x[0] > (R)p[3]) { x[0] = p[2]; *reset_bdf = 1; return 1; }
    } else if (ps->kind == EO_ADEX) {
        if (x[0] > 0.0f) { x[0] = p[7]; x[1] += (R)p[1]; *reset_bdf = 1; return 1; }
    } else {
        if (x[0] > -30.0f && prevV < -30.0f) return 1;
    }
    return 0;
}

/* ---------------------------------------------------------- integrators -- */
/* Gauss-Jordan inverse with zero-pivot row swap, BDFn.h:735-797. Returns 0 if singular. */
static int SFX(invermat)(int n, const R *a, R *ainv) {
    if (n == 1) { ainv[0] = 1.0f / a[0]; return 1; }
    R la[EO_MAXV * EO_MAXV], li[EO_MAXV * EO_MAXV];
    for (int i = 0; i < n * n; ++i) { la[i] = a[i]; li[i] = 0.0f; }
    for (int i = 0; i < n; ++i) li[i * n + i] = 1.0f;
    for (int s = 0; s < n; ++s) {
        R el = la[s * n + s];
        if (el == 0) {
            for (int r = s + 1; r < n; ++r) {
                el = la[r * n + s];
                if (el != 0) {
                    for (int c = 0; c < n; ++c) {
                        R v = la[r * n + c]; la[r * n + c] = la[s * n + c]; la[s * n + c] = v;
                        v = li[r * n + c]; li[r * n + c] = li[s * n + c]; li[s * n + c] = v;
                    }
                    break;
                }
                if (r == n - 1) return 0;
            }
        }
        R inv = 1.0f / el;
        for (int c = 0; c < n; ++c) { la[s * n + c] *= inv; li[s * n + c] *= inv; }
        for (int r = 0; r < n; ++r) {
            if (r == s) continue;
            R coef = -la[r * n + s];
            for (int c = 0; c < n; ++c) {
                la[r * n + c] += la[s * n + c] * coef;
                li[r * n + c] += li[s * n + c] * coef;
            }
        }
    }
    for (int i = 0; i < n * n; ++i) ainv[i] = li[i];
    return 1;
}

/* One-sided numerical Jacobian, BDFn.h:704-724 (epsilon = 0.1 dt). */
static void SFX(jacobian)(const eo_popstate *ps, const R *x, R *jac, double lst) {
    int nd = ps->ndiff, nv = ps->nvars;
    float dt = ps->dt_ms;
    R epsi = ORACLE_F32 ? (R)(dt * 0.1f) : (R)((double)dt * 0.1);
    R inv_epsi = 1.0f / epsi;
    R tmp[EO_MAXV], pos[EO_MAXV], neg[EO_MAXV];
    memcpy(tmp, x, sizeof(R) * nv);
    SFX(deriv)(ps, tmp, pos, lst, dt);
    for (int j = 0; j < nd; ++j) {
        memcpy(tmp, x, sizeof(R) * nv);
        tmp[j] -= epsi;
        SFX(deriv)(ps, tmp, neg, lst, dt);
        for (int z = 0; z < nd; ++z) jac[z * nd + j] = (pos[z] - neg[z]) * inv_epsi;
    }
}

/* Advance one neuron by one step.  Euler: Euler.h:123-146; RK2: RK2.h:133-165;
 * RK4: RK4.h:167-231; BDFn: BDFn.h:288-420.  Returns 1 if it spiked. */
static int SFX(step_neuron)(eo_popstate *ps, int64_t i, R *x, double *lst) {
    int nd = ps->ndiff, nv = ps->nvars;
    float dt = ps->dt_ms;
    R prevV = x[0];
    R k1[EO_MAXV], k2[EO_MAXV], k3[EO_MAXV], k4[EO_MAXV], aux[EO_MAXV];
    if (ps->integ == EO_EULER) {
        SFX(deriv)(ps, x, k1, *lst, dt);
        for (int j = 0; j < nd; ++j) x[j] += dt * k1[j];
        SFX(decay)(ps, x, 0);
    } else if (ps->integ == EO_RK2) {
        SFX(deriv)(ps, x, k1, *lst, dt);
        for (int j = 0; j < nd; ++j) x[j] += k1[j] * dt;
        SFX(decay)(ps, x, 0);
        SFX(deriv)(ps, x, k2, *lst, dt);
        for (int j = 0; j < nd; ++j) x[j] += (-k1[j] + k2[j]) * dt * 0.5f;
    } else if (ps->integ == EO_RK4) {
        R h05 = ORACLE_F32 ? (R)(dt * 0.5f) : (R)((double)dt * 0.5);
        R h016 = ORACLE_F32 ? (R)(dt * 0.166666666667f) : (R)((double)dt / 6.0);
        SFX(deriv)(ps, x, k1, *lst, dt);
        for (int j = 0; j < nd; ++j) aux[j] = x[j] + k1[j] * h05;
        for (int j = nd; j < nv; ++j) aux[j] = x[j];
        SFX(decay)(ps, aux, 0);
        SFX(deriv)(ps, aux, k2, *lst, dt);
        for (int j = 0; j < nd; ++j) aux[j] = x[j] + k2[j] * h05;
        SFX(deriv)(ps, aux, k3, *lst, dt);
        for (int j = 0; j < nd; ++j) aux[j] = x[j] + k3[j] * dt;
        SFX(decay)(ps, aux, 0);
        SFX(deriv)(ps, aux, k4, *lst, dt);
        for (int j = 0; j < nd; ++j) x[j] += (k1[j] + 2.0f * (k2[j] + k3[j]) + k4[j]) * h016;
        for (int j = nd; j < nv; ++j) x[j] = aux[j];
    } else {
        /* BDFn */
        int st = ps->bdf_state[i];
        R *Dm = (R *)ps->SFX(bdf_D);   /* [order][n][nd] */
        R *Pm = (R *)ps->SFX(bdf_P);   /* [order-1][n][nd] */
        int64_t N = ps->n;
        R p[EO_MAXV], p1[EO_MAXV], c[EO_MAXV], jac[EO_MAXV * EO_MAXV], J[EO_MAXV * EO_MAXV], iJ[EO_MAXV * EO_MAXV];
#define DD(ii, jj) Dm[((size_t)(ii) * N + i) * nd + (jj)]
#define PP(ii, jj) Pm[((size_t)(ii) * N + i) * nd + (jj)]
        if (st == 0) {
            SFX(deriv)(ps, x, aux, *lst, dt);
            for (int j = 0; j < nd; ++j) p[j] = x[j] + dt * aux[j];
        } else {
            for (int j = 0; j < nd; ++j) {
                p[j] = x[j];
                for (int q = 0; q < st; ++q) p[j] += DD(q, j);
            }
        }
        for (int j = nd; j < nv; ++j) p[j] = x[j];
        SFX(decay)(ps, p, 0);
        const float *co = ps->bdf_coef[st];
        R epsi = 1.0f;
        int k = 0;
        while (epsi > 1e-6 && k < 10) {
            SFX(deriv)(ps, p, aux, *lst, dt);
            for (int j = 0; j < nd; ++j) {
                c[j] = ORACLE_F32 ? (R)(co[0] * dt) * aux[j] + (R)co[1] * x[j]
                                  : (R)co[0] * (R)dt * aux[j] + (R)co[1] * x[j];
                for (int q = 1; q < st; ++q) c[j] += (R)co[q + 1] * PP(q - 1, j);
            }
            SFX(jacobian)(ps, p, jac, *lst);
            for (int z = 0; z < nd; ++z)
                for (int t = 0; t < nd; ++t) {
                    J[z * nd + t] = ORACLE_F32 ? (R)(co[0] * dt) * jac[z * nd + t]
                                               : (R)co[0] * (R)dt * jac[z * nd + t];
                    if (z == t) J[z * nd + t] -= 1;
                }
            if (!SFX(invermat)(nd, J, iJ)) return -1;
            for (int z = 0; z < nd; ++z) {
                R a = 0.0f;
                for (int t = 0; t < nd; ++t) a += iJ[z * nd + t] * (p[t] - c[t]);
                p1[z] = a + p[z];
            }
            R mx = 0.0f;
            for (int z = 0; z < nd; ++z) {
                R d = fabs(p1[z] - p[z]);
                if (d > mx) mx = d;
            }
            memcpy(p, p1, sizeof(R) * nd);
            epsi = mx;
            k++;
        }
        if (st < ps->bdf_order) st++;
        ps->bdf_state[i] = st;
        for (int j = 0; j < nd; ++j) {
            for (int q = st - 1; q > 0; --q) DD(q, j) = -DD(q - 1, j);
            DD(0, j) = p[j] - x[j];
            for (int q = 1; q < st; ++q) DD(q, j) += DD(q - 1, j);
        }
        if (st > 1) {
            for (int q = st - 2; q > 0; --q)
                for (int j = 0; j < nd; ++j) PP(q, j) = PP(q - 1, j);
            for (int j = 0; j < nd; ++j) PP(0, j) = x[j];
        }
        for (int j = 0; j < nd; ++j) x[j] = p[j];
        SFX(decay)(ps, x, 0);
#undef DD
#undef PP
    }
    *lst += (double)ps->dt_s;
    int reset_bdf = 0;
    int s = SFX(spike)(ps, x, prevV, &reset_bdf);
    if (s) {
        *lst = 0.0;
        if (reset_bdf && ps->integ == EO_BDF) ps->bdf_state[i] = 0;
    }
    return s;
}
