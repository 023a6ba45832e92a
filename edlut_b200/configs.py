"""Seeded synthetic networks with the shapes of the five benchmark workloads.

No dataset is involved: every network, weight and input spike comes from
``numpy.random.default_rng(seed)``.  Each builder takes a ``scale`` so the same
construction yields the full-size workload for the benchmark and a reduced copy
the CPU oracle finishes in seconds for the parity tests.

* :func:`lif_recurrent`     1,000 conductance LIF (800 E / 200 I), p=0.1, 100 Poisson inputs
                            at 10 Hz, 1 ms delays, Euler dt=0.1 ms.
* :func:`cerebellar_layer`  AdEx granule layer (in-degree 4 from Poisson mossy fibres at
                            5-50 Hz) feeding LIF Purkinje cells through plastic (STDP)
                            synapses; RK4 dt=0.1 ms.
* :func:`hh_network`        Hodgkin-Huxley neurons, in-degree 100, delays 1-5 ms, one
                            200 Hz Poisson drive each; BDF order 2 at dt=0.05 ms.
* :func:`sweep_networks`    many independent LIF networks of uneven size (log-uniform)
                            with per-network g_leak / E_leak / weight scale; RK2.
"""
from __future__ import annotations

import numpy as np

from .network import Layer, NetworkDescription, poisson_input_times

# LIF parameters for the recurrent workload (the benchmark description fixes
# E_exc 0, E_inh -80, E_L -65, v_thr -50, tau_ref 1 ms, tau_AMPA 0.5 ms,
# tau_GABA 10 ms and leaves C_m / g_L to the builder; these put the network in
# the 5-30 Hz range).
LIF_C1 = dict(e_exc=0.0, e_inh=-80.0, e_leak=-65.0, v_thr=-50.0, c_m=2.0, tau_exc=0.5,
              tau_inh=10.0, tau_ref=1.0, g_leak=0.2, tau_nmda=20.0)


def lif_recurrent(seed: int = 1, n: int = 1000, n_inputs: int = 100, p: float = 0.1,
                  rate_hz: float = 10.0, t_end: float = 1.0, dt: float = 1e-4,
                  integrator: str = "Euler", model: str = "LIFTimeDrivenModel",
                  params: dict | None = None, w_exc_max: float = 0.5, w_inh_max: float = 2.0,
                  delay: float = 1e-3, bdf_order: int = 2):
    """Recurrent E/I LIF network driven by Poisson inputs.

    Neurons 0..n_inputs-1 are ``InputSpikeNeuronModel`` (their spikes come from the
    returned input list); n_inputs.. are one LIF layer whose first 80% project
    excitatory (type 0) and last 20% inhibitory (type 1) synapses.
    Returns (NetworkDescription, input_times, input_cells).
    """
    rng = np.random.default_rng(seed)
    net = NetworkDescription()
    inp = net.add_layer(Layer(n_inputs, "InputSpikeNeuronModel", output=0))
    lif = net.add_layer(Layer(n, model, dict(params or LIF_C1), integrator=integrator, dt=dt,
                              bdf_order=bdf_order, name="lif"))
    n_exc = int(round(0.8 * n))
    sources = np.arange(n_inputs + n)
    mask = rng.random((len(sources), n)) < p
    s_idx, t_idx = np.nonzero(mask)
    src = sources[s_idx]
    tgt = lif.start + t_idx
    inh = src >= lif.start + n_exc
    stype = np.where(inh, 1, 0).astype(np.int32)
    wmax = np.where(inh, w_inh_max, w_exc_max).astype(np.float32)
    w = (rng.random(len(src)) * wmax).astype(np.float32)
    net.add_synapses(src, tgt, delay, stype, w, wmax, -1)
    times, cells = poisson_input_times(rng, n_inputs, rate_hz, t_end, dt)
    return net, times, cells + inp.start


def cerebellar_layer(seed: int = 1, n_granule: int = 250_000, n_mossy: int = 5_000,
                     n_purkinje: int = 200, pf_per_purkinje: int = 50_000,
                     t_end: float = 1.0, dt: float = 1e-4, integrator: str = "RK4",
                     w_mf: float = 4.0, w_pf: float = 0.05, w_pf_max: float = 0.1,
                     stdp=(1e-3, 0.020, 1.05e-3, 0.020), delay: float = 1e-3,
                     granule_params: dict | None = None, purkinje_params: dict | None = None):
    """Granule (AdEx) layer with in-degree 4 from Poisson mossy fibres at U[5,50] Hz,
    and Purkinje (LIF) cells each receiving ``pf_per_purkinje`` granule synapses
    drawn without replacement, all plastic under additive STDP.
    Returns (NetworkDescription, input_times, input_cells)."""
    rng = np.random.default_rng(seed)
    net = NetworkDescription()
    mf = net.add_layer(Layer(n_mossy, "InputSpikeNeuronModel", output=0))
    grc = net.add_layer(Layer(n_granule, "AdExTimeDrivenModel", dict(granule_params or {}),
                              integrator=integrator, dt=dt, name="granule"))
    pc = net.add_layer(Layer(n_purkinje, "LIFTimeDrivenModel",
                             dict(purkinje_params or dict(c_m=100.0, g_leak=5.0, tau_exc=2.0)),
                             integrator=integrator, dt=dt, name="purkinje"))
    net.rules.append(("STDP", list(stdp)))
    # mossy fibre -> granule: in-degree exactly 4
    src = rng.integers(0, n_mossy, size=(n_granule, 4)) + mf.start
    tgt = np.repeat(np.arange(n_granule) + grc.start, 4)
    net.add_synapses(src.ravel(), tgt, delay, 0, w_mf, w_mf, -1)
    # granule -> Purkinje: pf_per_purkinje distinct granules per Purkinje cell
    k = min(pf_per_purkinje, n_granule)
    srcs = np.empty((n_purkinje, k), np.int64)
    for j in range(n_purkinje):
        srcs[j] = rng.choice(n_granule, size=k, replace=False)
    srcs += grc.start
    tgts = np.repeat(np.arange(n_purkinje) + pc.start, k)
    wpf = (rng.random(n_purkinje * k) * 2 * w_pf).astype(np.float32)
    net.add_synapses(srcs.ravel(), tgts, delay, 0, np.minimum(wpf, w_pf_max), w_pf_max, 0)
    rates = rng.uniform(5.0, 50.0, n_mossy)
    times, cells = poisson_input_times(rng, n_mossy, rates, t_end, dt)
    return net, times, cells + mf.start


def hh_network(seed: int = 1, n: int = 100_000, indeg: int = 100, t_end: float = 0.5,
               dt: float = 5e-5, drive_hz: float = 200.0, w_exc: float = 3.0,
               w_inh: float = 12.0, w_drive: float = 30.0, bdf_order: int = 2,
               integrator: str = "BDF", params: dict | None = None, unique_times: bool = True):
    """Hodgkin-Huxley network: fixed in-degree from uniformly random sources (80% of
    sources excitatory), integer delays of 1-5 ms, one Poisson drive per neuron at
    ``drive_hz`` through a 1 ms excitatory synapse.
    Returns (NetworkDescription, input_times, input_cells)."""
    rng = np.random.default_rng(seed)
    net = NetworkDescription()
    drv = net.add_layer(Layer(n, "InputSpikeNeuronModel", output=0))
    hh = net.add_layer(Layer(n, "HHTimeDrivenModel", dict(params or {}), integrator=integrator,
                             dt=dt, bdf_order=bdf_order, name="hh"))
    n_exc = int(round(0.8 * n))
    src = rng.integers(0, n, size=(n, indeg))
    tgt = np.repeat(np.arange(n), indeg)
    src = src.ravel()
    inh = src >= n_exc
    delay = rng.integers(1, 6, size=len(src)).astype(np.float32) * np.float32(1e-3)
    net.add_synapses(src + hh.start, tgt + hh.start, delay, inh.astype(np.int32),
                     np.where(inh, w_inh, w_exc), np.where(inh, w_inh, w_exc), -1)
    net.add_synapses(np.arange(n) + drv.start, np.arange(n) + hh.start, 1e-3, 0, w_drive,
                     w_drive, -1)
    times, cells = poisson_input_times(rng, n, drive_hz, t_end, dt, unique=unique_times)
    return net, times, cells + drv.start


def sweep_sizes(seed: int = 1, n_networks: int = 4096, n_min: int = 500, n_max: int = 5000):
    """Network sizes log-uniform in [n_min, n_max]."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_networks)).astype(np.int64)


def sweep_networks(seed: int = 1, n_networks: int = 4096, n_min: int = 500, n_max: int = 5000,
                   t_end: float = 1.0, dt: float = 1e-4, n_inputs: int = 100, rate_hz: float = 10.0,
                   p: float = 0.1, variation: float = 0.3, base: dict | None = None,
                   w_exc_max: float = 0.5, w_inh_max: float = 2.0, w_in_max: float = 0.5,
                   ref_size: int = 1000):
    """Specifications of the batched parameter sweep: ``n_networks`` independent
    LIF networks (80% E / 20% I) with sizes log-uniform in [n_min, n_max], each
    with its own Poisson seed for ``n_inputs`` inputs at ``rate_hz``.

    Per network, with s_x ~ U[1 - variation, 1 + variation]:
      * g_leak = base g_leak * s_g;
      * E_leak = v_thr - (v_thr - base E_leak) * s_e -- the variation applies to the
        leak's 15 mV distance below threshold, so every network stays excitable
        rather than firing tonically (E_leak above v_thr);
      * weight scale s_w on every weight range; recurrent ranges are also scaled by
        ref_size / n so that each neuron's mean recurrent drive matches the
        1,000-neuron recurrent workload at every size.
    Returns a list of dicts with keys n, n_exc, n_in, params, p, w_exc_max,
    w_inh_max, w_in_max, times, cells (cells are input indices 0..n_in-1)."""
    sizes = sweep_sizes(seed, n_networks, n_min, n_max)
    rng = np.random.default_rng([seed, 0x5EED])
    lo, hi = 1.0 - variation, 1.0 + variation
    s_g = rng.uniform(lo, hi, n_networks)
    s_e = rng.uniform(lo, hi, n_networks)
    s_w = rng.uniform(lo, hi, n_networks)
    b = dict(base or LIF_C1)
    specs = []
    for i, n in enumerate(sizes):
        n = int(n)
        prm = dict(b)
        prm["g_leak"] = float(np.float32(b["g_leak"] * s_g[i]))
        prm["e_leak"] = float(np.float32(b["v_thr"] - (b["v_thr"] - b["e_leak"]) * s_e[i]))
        rec_scale = s_w[i] * ref_size / n
        irng = np.random.default_rng([seed, 1, i])
        times, cells = poisson_input_times(irng, n_inputs, rate_hz, t_end, dt)
        specs.append(dict(n=n, n_exc=int(round(0.8 * n)), n_in=n_inputs, params=prm, p=p,
                          w_exc_max=float(np.float32(w_exc_max * rec_scale)),
                          w_inh_max=float(np.float32(w_inh_max * rec_scale)),
                          w_in_max=float(np.float32(w_in_max * s_w[i])),
                          times=times, cells=cells.astype(np.int32)))
    return specs


# Per-model synaptic weight ranges that give moderate firing in parity_network.
_PARITY_W = {
    "LIFTimeDrivenModel": dict(w_in=0.5, w_exc=0.5, w_inh=2.0),
    "AdExTimeDrivenModel": dict(w_in=6.0, w_exc=2.0, w_inh=4.0),
    "HHTimeDrivenModel": dict(w_in=40.0, w_exc=10.0, w_inh=20.0),
}


def parity_network(model: str = "LIFTimeDrivenModel", integrator: str = "Euler", seed: int = 1,
                   n: int = 200, n_inputs: int = 40, p: float = 0.1, rate_hz: float = 20.0,
                   t_end: float = 0.2, dt: float = 1e-4, bdf_order: int = 2, stdp: bool = False,
                   delays=(1e-3,), params: dict | None = None, weights: dict | None = None):
    """Small recurrent E/I network of one model, for step-level parity against the
    reference: Poisson inputs, p-connectivity, one or several delays, optional STDP on
    the excitatory recurrent synapses.  Returns (NetworkDescription, in_times, in_cells)."""
    rng = np.random.default_rng(seed)
    w = dict(_PARITY_W[model.replace("_GPU", "")])
    w.update(weights or {})
    net = NetworkDescription()
    inp = net.add_layer(Layer(n_inputs, "InputSpikeNeuronModel", output=0))
    pop = net.add_layer(Layer(n, model, dict(params or {}), integrator=integrator, dt=dt,
                              bdf_order=bdf_order, name="pop"))
    if stdp:
        net.rules.append(("STDP", [0.05 * w["w_exc"], 0.020, 0.0525 * w["w_exc"], 0.020]))
    n_exc = int(round(0.8 * n))
    # input -> population (dense-ish so every neuron is driven)
    m_in = rng.random((n_inputs, n)) < max(p, 0.25)
    s, t = np.nonzero(m_in)
    net.add_synapses(s + inp.start, t + pop.start, delays[0], 0,
                     (rng.random(len(s)) * w["w_in"]).astype(np.float32), w["w_in"], -1)
    mr = rng.random((n, n)) < p
    s, t = np.nonzero(mr)
    inh = s >= n_exc
    d = np.asarray(delays, np.float32)[rng.integers(0, len(delays), len(s))]
    wmax = np.where(inh, w["w_inh"], w["w_exc"]).astype(np.float32)
    ww = (rng.random(len(s)) * wmax).astype(np.float32)
    rule = np.where(inh | (not stdp), -1, 0).astype(np.int32)
    net.add_synapses(s + pop.start, t + pop.start, d, inh.astype(np.int32), ww, wmax, rule)
    times, cells = poisson_input_times(rng, n_inputs, rate_hz, t_end, dt)
    return net, times, cells + inp.start


def wide_fanin_network(seed: int = 1, n_relay: int = 3000, n_target: int = 4, n_repeat: int = 2,
                       n_direct: int = 40, bursts=(60, 200, 400, 512, 520, 800, 2000, 3000),
                       gap_steps: int = 40, dt: float = 1e-4):
    """Arrival-count coverage network for the block-per-neuron update: ``n_relay``
    LIF relays, each driven by its own input, fire in bursts of the given sizes (half
    of a burst one step after the other half), and project with delays 0.9 or 1.0 ms
    onto ``n_target`` LIF targets (RK4, STDP) and ``n_repeat`` LIF targets (Euler,
    STDP) that also receive ``n_direct`` inputs, some of which fire twice within one
    step.  A burst of B relays delivers about B/2 arrivals in one step (the two
    halves meet) and B/4 in the steps either side, so the defaults reach every
    arrival-count regime of the update (tens, up to 256, up to 1024, beyond).
    Returns (NetworkDescription, input_times, input_cells)."""
    rng = np.random.default_rng(seed)
    net = NetworkDescription()
    inp = net.add_layer(Layer(n_relay + n_direct, "InputSpikeNeuronModel", output=0))
    rel = net.add_layer(Layer(n_relay, "LIFTimeDrivenModel", dict(LIF_C1), integrator="RK2", dt=dt, name="relay"))
    tgt = net.add_layer(Layer(n_target, "LIFTimeDrivenModel", dict(LIF_C1), integrator="RK4", dt=dt, name="target"))
    rep = net.add_layer(Layer(n_repeat, "LIFTimeDrivenModel", dict(LIF_C1), integrator="Euler", dt=dt,
                              name="repeat"))
    w_max = 0.2
    net.rules.append(("STDP", [0.05 * w_max, 0.020, 0.0525 * w_max, 0.020]))
    # input j -> relay j: one spike of the relay per input spike
    net.add_synapses(np.arange(n_relay) + inp.start, np.arange(n_relay) + rel.start, 1e-4, 0, 8.0, 8.0, -1)
    for layer in (tgt, rep):
        s = np.repeat(np.arange(n_relay), len(layer))
        t = np.tile(np.arange(len(layer)), n_relay)
        d = np.where(rng.random(len(s)) < 0.5, 0.9e-3, 1.0e-3).astype(np.float32)
        w = (rng.random(len(s)) * w_max).astype(np.float32)
        net.add_synapses(s + rel.start, t + layer.start, d, 0, w, np.float32(1.25 * w_max), 0)
    s = np.repeat(np.arange(n_direct), n_repeat)
    t = np.tile(np.arange(n_repeat), n_direct)
    net.add_synapses(s + n_relay + inp.start, t + rep.start, 1e-3, 0,
                     (rng.random(len(s)) * w_max).astype(np.float32), np.float32(1.25 * w_max), 0)
    times, cells = [], []
    for b, size in enumerate(bursts):
        step = 20 + gap_steps * b
        who = rng.choice(n_relay, size=min(size, n_relay), replace=False)
        half = len(who) // 2
        times.append(np.full(half, (step + 0.5) * dt))
        times.append(np.full(len(who) - half, (step + 1.5) * dt))
        cells.append(who)
    t_end = (20 + gap_steps * len(bursts)) * dt
    dt_in, dc_in = poisson_input_times(rng, n_direct, 200.0, t_end, dt)
    times.append(dt_in)
    cells.append(dc_in + n_relay)
    # doublets: a direct input firing twice inside one step
    for _ in range(12):
        j = int(rng.integers(0, n_direct))
        k = int(rng.integers(10, int(t_end / dt) - 10))
        times.append(np.array([(k + 0.2) * dt, (k + 0.7) * dt]))
        cells.append(np.array([j + n_relay, j + n_relay]))
    times = np.concatenate(times)
    cells = np.concatenate(cells).astype(np.int64)
    o = np.lexsort((cells, times))
    return net, times[o], cells[o] + inp.start


# Parameters the adjoint differentiates, in the order of its gradient rows.
ADJOINT_PARAMS = ("g_leak", "e_leak", "tau_exc", "tau_inh")


def adjoint_networks(seed: int = 1, n_networks: int = 64, n: int = 10_000, indeg: int = 100,
                     n_inputs: int = 100, in_indeg: int = 10, rate_hz: float = 10.0, t_end: float = 0.5,
                     dt: float = 1e-4, w_exc_max: float = 0.5, w_inh_max: float = 2.0,
                     w_in_max: float = 0.5, base: dict | None = None, tau_exc: float | None = None):
    """Networks of the adjoint-fitting workload: ``n_networks`` LIF networks of ``n``
    neurons (80% E / 20% I), each neuron with exactly ``indeg`` recurrent inputs drawn
    without replacement (the 1,000-neuron recurrent workload's in-degree, so its weight
    ranges carry over) and ``in_indeg`` inputs from ``n_inputs`` Poisson sources at
    ``rate_hz`` (per-network seeds).  Parameters are the recurrent workload's (AMPA
    tau 0.5 ms; ``tau_exc`` overrides it -- longer AMPA time constants at this drive
    make the explicit integrators unstable at C_m = 2).  Returns specs
    for :meth:`edlut_b200.sweep.Sweep.from_specs` with explicit ``src``, ``tgt``, ``w``
    (sources 0..n-1 recurrent, n.. inputs)."""
    b = dict(base or LIF_C1)
    if tau_exc is not None:
        b["tau_exc"] = tau_exc
    specs = []
    n_exc = int(round(0.8 * n))
    for i in range(n_networks):
        rng = np.random.default_rng([seed, 2, i])
        # recurrent: per target `indeg` distinct sources
        src_r = _distinct_rows(rng, n, n, indeg)
        tgt_r = np.repeat(np.arange(n), indeg)
        src_r = src_r.reshape(-1)
        inh = (src_r >= n_exc)
        w_r = rng.random(len(src_r)) * np.where(inh, w_inh_max, w_exc_max)
        src_i = _distinct_rows(rng, n, n_inputs, in_indeg).reshape(-1) + n
        tgt_i = np.repeat(np.arange(n), in_indeg)
        w_i = rng.random(len(src_i)) * w_in_max
        times, cells = poisson_input_times(rng, n_inputs, rate_hz, t_end, dt)
        specs.append(dict(n=n, n_exc=n_exc, n_in=n_inputs, params=dict(b),
                          src=np.concatenate([src_r, src_i]).astype(np.int32),
                          tgt=np.concatenate([tgt_r, tgt_i]).astype(np.int32),
                          w=np.concatenate([w_r, w_i]).astype(np.float32),
                          times=times, cells=cells.astype(np.int32)))
    return specs


def _distinct_rows(rng, rows: int, n: int, k: int) -> np.ndarray:
    """rows x k draws without replacement from range(n): the first k distinct values of
    an i.i.d. stream per row (a uniform random subset), vectorised."""
    out = np.empty((rows, k), np.int64)
    todo = np.arange(rows)
    extra = 8 + k // 4
    while len(todo):
        m = k + extra
        draw = rng.integers(0, n, size=(len(todo), m))
        order = np.argsort(draw, axis=1, kind="stable")
        srt = np.take_along_axis(draw, order, 1)
        first = np.ones_like(srt, bool)
        first[:, 1:] = srt[:, 1:] != srt[:, :-1]
        keep = np.empty_like(first)
        np.put_along_axis(keep, order, first, 1)
        ok = keep.sum(1) >= k
        rank = np.cumsum(keep, 1)
        sel = keep & (rank <= k)
        good = todo[ok]
        out[good] = draw[ok][sel[ok]].reshape(-1, k)
        todo = todo[~ok]
        extra *= 2
    return out


def perturbed_params(base: dict, rng, spread: float = 0.3):
    """A parameter set with each of ADJOINT_PARAMS scaled by U[1 - spread, 1 + spread]
    (E_leak through its distance below threshold, which keeps it below v_thr)."""
    p = dict(base)
    for k in ADJOINT_PARAMS:
        s = rng.uniform(1 - spread, 1 + spread)
        if k == "e_leak":
            p[k] = float(np.float32(base["v_thr"] - (base["v_thr"] - base["e_leak"]) * s))
        else:
            p[k] = float(np.float32(base[k] * s))
    return p


def poisson_network(seed: int = 1, n: int = 150, generators=((40, 30.0), (30, 80.0)),
                    after=((20, 30.0),), p: float = 0.2, t_end: float = 0.2, dt: float = 1e-4,
                    integrator: str = "RK2", stdp: bool = True, w_in: float = 2.0,
                    w_exc: float = 0.5, w_inh: float = 2.0):
    """LIF population driven by PoissonGeneratorDeviceVector layers (the device
    generators replace input-spike lists).  ``generators`` are (size, frequency)
    layers before the LIF population and ``after`` layers after it; a layer whose
    frequency equals an earlier one's shares its model type, which decides the order
    its generators draw their seeds in.  Generator -> LIF synapses are plastic when
    ``stdp``.  Returns (NetworkDescription, [], [])."""
    rng = np.random.default_rng(seed)
    net = NetworkDescription()
    gens = []
    for i, (g, f) in enumerate(generators):
        gens.append(net.add_layer(Layer(g, "PoissonGeneratorDeviceVector", dict(frequency=f),
                                        name="poisson_%d" % i)))
    pop = net.add_layer(Layer(n, "LIFTimeDrivenModel", {}, integrator=integrator, dt=dt, name="lif"))
    for i, (g, f) in enumerate(after):
        gens.append(net.add_layer(Layer(g, "PoissonGeneratorDeviceVector", dict(frequency=f),
                                        name="poisson_after_%d" % i)))
    if stdp:
        net.rules.append(("STDP", [0.05 * w_in, 0.020, 0.0525 * w_in, 0.020]))
    for gl in gens:
        m = rng.random((len(gl), n)) < p
        s, t = np.nonzero(m)
        net.add_synapses(s + gl.start, t + pop.start, 1e-3, 0,
                         (rng.random(len(s)) * w_in).astype(np.float32), w_in, 0 if stdp else -1)
    n_exc = int(round(0.8 * n))
    mr = rng.random((n, n)) < 0.1
    s, t = np.nonzero(mr)
    inh = s >= n_exc
    wmax = np.where(inh, w_inh, w_exc).astype(np.float32)
    net.add_synapses(s + pop.start, t + pop.start, 1e-3, inh.astype(np.int32),
                     (rng.random(len(s)) * wmax).astype(np.float32), wmax, -1)
    return net, np.zeros(0, np.float32), np.zeros(0, np.int64)
