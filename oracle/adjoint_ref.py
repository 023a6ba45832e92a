"""FP64 reference adjoint of the time-driven LIF network -- test infrastructure.

Only the tests and the benchmark's checks import this module; it is never on the
product path.  It checks the GPU adjoint of the batched sweep (which has no
counterpart in the reference) in two independent ways:

* :func:`adjoint_fp64` -- the discrete adjoint of the FP64 forward of the C
  oracle (``edlut_oracle.c`` with fp64=1: the reference's LIF update and RK
  integrators, src/neuron_model/LIFTimeDrivenModel.cpp:160-242,
  include/integration_method/Euler.h:123-146, RK2.h:133-165, RK4.h:167-231, in
  double precision), restated here with numpy.  The forward trajectory comes from
  the oracle's full FP64 trace; the post-arrival conductances are rebuilt from its
  spikes with the reference's delivery rule (arrival at the first update time
  after t_spike + d, include/simulation/Event.h:37).
* :func:`finite_difference` -- FP64 central differences of the same loss through
  two oracle runs, with the denominator taken from the float32 values the forward
  actually receives.

The loss is any function of the observed membrane traces; callers pass dL/dtrace.
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as O


def _time_grid(dt: float, n: int) -> np.ndarray:
    t = np.zeros(n + 1)
    for k in range(1, n + 1):
        t[k] = t[k - 1] + float(np.float32(dt))
    return t


def _units(d: float) -> int:
    f = np.floor(float(np.float32(d)) * (1.0 / 0.0001) + 0.0001 * 0.5)
    return 1 if f <= 0 else int(f)


def trajectory_fp64(net, in_times, in_cells, nsteps: int):
    """FP64 forward of a one-population LIF network (layer 0 LIF, further layers
    inputs): per step k = 1..nsteps the integration inputs (V_in, gE_in, gI_in), the
    refractory class and fraction, the spike flag, and the state after the step."""
    lif = net.layers[0]
    n = lif.n
    p = lif.full_params()
    dt = float(np.float32(lif.dt))
    r = O.run(net, in_times, in_cells, nsteps, fp64=True, trace=(nsteps, 0, n))
    tr = r["trace"]  # [steps, n, 8]: V, gE, gI, ...
    sp_step, sp_cell = r["spike_step"], r["spike_cell"]
    spiked = np.zeros((nsteps + 1, n), bool)
    m = sp_cell < n
    spiked[sp_step[m], sp_cell[m]] = True
    # arrivals: internal spike at step j reaches the first k > j with t_k > t_j + d;
    # an input spike at time t reaches the first k with t_k > t + d
    t = _time_grid(dt, nsteps + 64)
    src = np.asarray(net.src)
    tgt = np.asarray(net.tgt)
    w = np.asarray(net.weight, np.float64)
    st = np.asarray(net.stype)
    dunits = np.array([_units(d) for d in np.asarray(net.delay, np.float32)])
    if len(set(dunits.tolist())) > 1:
        raise ValueError("one delay per network")
    dd = float(dunits[0]) * 0.0001
    arr_E = np.zeros((nsteps + 2, n))
    arr_I = np.zeros((nsteps + 2, n))
    by_src = {}
    for k in range(len(src)):
        by_src.setdefault(int(src[k]), []).append(k)
    syn_arrivals = [[] for _ in range(len(src))]  # arrival steps per synapse

    def deliver(s, ka):
        for q in by_src.get(s, ()):
            (arr_I if st[q] == 1 else arr_E)[ka, tgt[q]] += w[q]
            syn_arrivals[q].append(ka)

    for j, c in zip(sp_step[m], sp_cell[m]):
        a = t[j] + dd
        ka = int(np.searchsorted(t, a, side="right"))
        if ka <= nsteps:
            deliver(int(c), ka)
    for tin, c in zip(np.asarray(in_times, np.float32), np.asarray(in_cells)):
        a = float(tin) + dd
        ka = max(1, int(np.searchsorted(t, a, side="right")))
        if ka <= nsteps:
            deliver(int(c), ka)
    V_post = np.concatenate([np.full((1, n), float(np.float32(p["e_leak"]))), tr[:, :, 0]])
    gE_post = np.concatenate([np.zeros((1, n)), tr[:, :, 1]])
    gI_post = np.concatenate([np.zeros((1, n)), tr[:, :, 2]])
    V_in = V_post[:-1]
    gE_in = gE_post[:-1] + arr_E[1:nsteps + 1]
    gI_in = gI_post[:-1] + arr_I[1:nsteps + 1]
    # refractory class at step k from the steps since the last spike
    dt_ms = float(np.float32(np.float32(dt) * np.float32(1000.0)))
    tau_ref = float(np.float32(p["tau_ref"]))
    cls = np.zeros((nsteps, n), np.int8)
    frac = np.ones((nsteps, n))
    last = np.full(n, -1, np.int64)
    for k in range(1, nsteps + 1):
        rr = np.where(last >= 0, k - 1 - last, -1)
        l = (rr.astype(np.float64) * dt) * 1000.0
        free = (rr < 0) | (l > tau_ref)
        part = ~free & (l + dt_ms > tau_ref)
        cls[k - 1] = np.where(free, 0, np.where(part, 2, 1))
        frac[k - 1] = np.where(part, (l + dt_ms - tau_ref) / dt_ms, 1.0)
        last = np.where(spiked[k], k, last)
    en = [bool((st == 0).any()), bool((st == 1).any())]
    return dict(V_in=V_in, gE_in=gE_in, gI_in=gI_in, cls=cls, frac=frac, spiked=spiked[1:nsteps + 1],
                V_post=V_post[1:], syn_arrivals=syn_arrivals, en=en, params=p, dt_ms=dt_ms,
                integrator=lif.integrator, spikes=(sp_step, sp_cell))


def adjoint_fp64(traj, obs, grad_trace):
    """Discrete adjoint of the FP64 forward.  obs: observed neurons [m]; grad_trace:
    dL/dV_obs [steps, m].  Returns (grad_params [g_leak, e_leak, tau_exc, tau_inh],
    grad_w per synapse in the network description's order)."""
    p = traj["params"]
    Ee, Ei, EL = float(np.float32(p["e_exc"])), float(np.float32(p["e_inh"])), float(np.float32(p["e_leak"]))
    gL = float(np.float32(p["g_leak"]))
    invc = 1.0 / float(np.float32(p["c_m"]))
    tE, tI = float(np.float32(p["tau_exc"])), float(np.float32(p["tau_inh"]))
    h = traj["dt_ms"]
    integ = traj["integrator"]
    el = h * 0.5 if integ == "RK4" else h
    aE, aI = np.exp(-el / tE), np.exp(-el / tI)
    en1, en2 = traj["en"]
    lim = float(np.float32(1e-9))
    nsteps, n = traj["V_in"].shape
    lV = np.zeros(n)
    lE = np.zeros(n)
    lI = np.zeros(n)
    G = np.zeros(4)  # g_leak, e_leak, d aE, d aI
    muE = np.zeros((nsteps, n))
    muI = np.zeros((nsteps, n))

    def D(V, gE, gI, c, f):
        cur = (gE * (Ee - V) if en1 else 0.0) + (gI * (Ei - V) if en2 else 0.0)
        full = (cur + gL * (EL - V)) * invc
        return np.where(c == 1, 0.0, np.where(c == 2, f * full, full))

    def dD(V, gE, gI, c, f, lk, acc):
        s = np.where(c == 1, 0.0, np.where(c == 2, f, 1.0)) * invc * lk
        dV = -gL - (gE if en1 else 0.0) - (gI if en2 else 0.0)
        acc[0] += s * (EL - V)
        acc[1] += s * gL
        return s * dV, (s * (Ee - V) if en1 else 0.0 * s), (s * (Ei - V) if en2 else 0.0 * s)

    def decay(gE, gI):
        return (np.where(gE < lim, 0.0, gE * aE) if en1 else gE), (np.where(gI < lim, 0.0, gI * aI) if en2 else gI)

    def d_decay(gE, gI, lEo, lIo, acc):
        if en1:
            on = ~(gE < lim)
            lE_ = np.where(on, lEo * aE, 0.0)
            acc[2] += np.where(on, lEo * gE, 0.0)
        else:
            lE_ = lEo
        if en2:
            on = ~(gI < lim)
            lI_ = np.where(on, lIo * aI, 0.0)
            acc[3] += np.where(on, lIo * gI, 0.0)
        else:
            lI_ = lIo
        return lE_, lI_

    for k in range(nsteps, 0, -1):
        x = k - 1
        lV = lV.copy()
        lV[obs] += grad_trace[x]
        V, gE, gI = traj["V_in"][x], traj["gE_in"][x], traj["gI_in"][x]
        c, f = traj["cls"][x], traj["frac"][x]
        acc = [np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)]
        sp = traj["spiked"][x]
        acc[1] += np.where(sp, lV, 0.0)
        lVo = np.where(sp, 0.0, lV)
        if integ == "Euler":
            a, b, cc = dD(V, gE, gI, c, f, lVo * h, acc)
            nV = lVo + a
            dE, dI = d_decay(gE, gI, lE, lI, acc)
            nE, nI = b + dE, cc + dI
        elif integ == "RK2":
            k1 = D(V, gE, gI, c, f)
            V1 = V + k1 * h
            gE2, gI2 = decay(gE, gI)
            lk2 = lVo * h * 0.5
            a, b, cc = dD(V1, gE2, gI2, c, f, lk2, acc)
            lV1, lE2, lI2 = lVo + a, lE + b, lI + cc
            lk1 = -lk2 + lV1 * h
            a, b, cc = dD(V, gE, gI, c, f, lk1, acc)
            dE, dI = d_decay(gE, gI, lE2, lI2, acc)
            nV, nE, nI = lV1 + a, b + dE, cc + dI
        else:  # RK4
            h05, h016 = h * 0.5, h / 6.0
            k1 = D(V, gE, gI, c, f)
            a1 = V + k1 * h05
            gAE, gAI = decay(gE, gI)
            k2 = D(a1, gAE, gAI, c, f)
            a2 = V + k2 * h05
            k3 = D(a2, gAE, gAI, c, f)
            a3 = V + k3 * h
            gBE, gBI = decay(gAE, gAI)
            nV = lVo.copy()
            lk1 = lVo * h016
            a, b, cc = dD(a3, gBE, gBI, c, f, lk1, acc)
            nV += a
            lBE, lBI = lE + b, lI + cc
            lk3 = 2.0 * h016 * lVo + a * h
            lAE, lAI = d_decay(gAE, gAI, lBE, lBI, acc)
            a, b, cc = dD(a2, gAE, gAI, c, f, lk3, acc)
            nV += a
            lAE, lAI = lAE + b, lAI + cc
            lk2 = 2.0 * h016 * lVo + a * h05
            a, b, cc = dD(a1, gAE, gAI, c, f, lk2, acc)
            nV += a
            lAE, lAI = lAE + b, lAI + cc
            lk1 = lk1 + a * h05
            dE, dI = d_decay(gE, gI, lAE, lAI, acc)
            a, b, cc = dD(V, gE, gI, c, f, lk1, acc)
            nV, nE, nI = nV + a, dE + b, dI + cc
        lV, lE, lI = nV, nE, nI
        muE[x], muI[x] = lE, lI
        for q in range(4):
            G[q] += acc[q].sum()
    G[1] += lV.sum()  # V_0 = E_leak
    grad = np.array([G[0], G[1], G[2] * aE * el / tE ** 2, G[3] * aI * el / tI ** 2])
    return grad, muE, muI


def weight_grad(net, traj, muE, muI):
    """dL/dw per synapse: the sum over its arrivals of the target's conductance adjoint."""
    tgt = np.asarray(net.tgt)
    st = np.asarray(net.stype)
    gw = np.zeros(len(tgt))
    for q, arrs in enumerate(traj["syn_arrivals"]):
        mu = muI if st[q] == 1 else muE
        for ka in arrs:
            gw[q] += mu[ka - 1, tgt[q]]
    return gw


def finite_difference(net, in_times, in_cells, nsteps: int, loss, what, rel: float = 1e-6):
    """Central FP64 difference of loss(trace [steps, n]) through the oracle.
    what = ("param", name) or ("weight", synapse index).  The perturbed value is a
    float32 (what the forward receives); the denominator is the float32 difference.
    Returns (derivative, spike trains identical at +/- and at the base)."""
    import copy
    base = O.run(net, in_times, in_cells, nsteps, fp64=True)
    outs = []
    for sgn in (1, -1):
        nb = copy.deepcopy(net)
        if what[0] == "param":
            v0 = nb.layers[0].full_params()[what[1]]
            v = float(np.float32(v0 * (1 + sgn * rel)))
            nb.layers[0].params = dict(nb.layers[0].params)
            nb.layers[0].params[what[1]] = v
        else:
            q = what[1]
            v0 = float(nb.weight[q])
            v = np.float32(v0 * (1 + sgn * rel) if v0 != 0 else sgn * rel)
            nb.weight = np.array(nb.weight, np.float32)
            nb.weight[q] = v
            nb.max_weight = np.maximum(np.asarray(nb.max_weight, np.float32), nb.weight)
            v = float(v)
        n = nb.layers[0].n
        r = O.run(nb, in_times, in_cells, nsteps, fp64=True, trace=(nsteps, 0, n))
        same = np.array_equal(r["spike_step"], base["spike_step"]) and np.array_equal(r["spike_cell"], base["spike_cell"])
        outs.append((v, loss(r["trace"][:, :, 0]), same))
    (vp, lp, sp), (vm, lm, sm) = outs
    return (lp - lm) / (vp - vm), sp and sm
