"""Network descriptions in EDLUT's own terms, and writers for its text formats.

A :class:`NetworkDescription` holds what an EDLUT network file and weights file
hold: neuron layers (model name + parameter file), learning rules, and synapses
(source, target, delay, type, max weight, learning-rule index, weight).  It can

* write the reference's file formats, so the same network runs unchanged in
  EDLUT and here:
    - network file  (parsed by ``Network::ParseNet``, ``src/spike/Network.cpp:422-645``)
    - weights file  (``src/spike/Network.cpp:647-690``)
    - neuron-model ``.cfg`` files (e.g. ``LIFTimeDrivenModel::ParseNeuronModel``,
      ``src/neuron_model/LIFTimeDrivenModel.cpp:448-540``) followed by the
      integration method (``include/integration_method/IntegrationMethod.h:300-318``,
      ``include/integration_method/BDFn.h:864-884``)
    - input-spike files (``FileInputSpikeDriver::LoadInputs``,
      ``src/communication/FileInputSpikeDriver.cpp:45-78``)
* be handed to :class:`edlut_b200.Simulation` directly (no text round trip).

Float values are written with 9 significant digits so that the reference's
``fscanf("%f")`` reads back the identical float32.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

# Parameter order of each model's .cfg file, exactly as its ParseNeuronModel reads it.
MODEL_PARAM_ORDER: Dict[str, List[str]] = {
    # src/neuron_model/LIFTimeDrivenModel.cpp:448-530
    "LIFTimeDrivenModel": ["e_exc", "e_inh", "e_leak", "v_thr", "c_m", "tau_exc",
                           "tau_inh", "tau_ref", "g_leak", "tau_nmda"],
    # src/neuron_model/AdExTimeDrivenModel.cpp (ParseNeuronModel)
    "AdExTimeDrivenModel": ["a", "b", "thr_slo_fac", "v_thr", "tau_w", "e_exc", "e_inh",
                            "e_reset", "e_leak", "g_leak", "c_m", "tau_exc", "tau_inh",
                            "tau_nmda"],
    # src/neuron_model/HHTimeDrivenModel.cpp (ParseNeuronModel)
    "HHTimeDrivenModel": ["e_exc", "e_inh", "e_leak", "g_leak", "c_m", "v_thr", "tau_exc",
                          "tau_inh", "tau_nmda", "g_na", "g_kd", "e_na", "e_k"],
    # src/neuron_model/PoissonGeneratorDeviceVector.cpp:175-200 (ParseNeuronModel)
    "PoissonGeneratorDeviceVector": ["frequency"],
}
# The *_GPU model names read the same parameter files in the same order.
for _n in list(MODEL_PARAM_ORDER):
    MODEL_PARAM_ORDER[_n + "_GPU"] = MODEL_PARAM_ORDER[_n]

# Defaults of each model (GetDefaultParameters of the CPU twins).
MODEL_DEFAULTS: Dict[str, Dict[str, float]] = {
    # src/neuron_model/LIFTimeDrivenModel.cpp:420-434
    "LIFTimeDrivenModel": dict(e_exc=0.0, e_inh=-80.0, e_leak=-65.0, v_thr=-50.0, c_m=2.0,
                               tau_exc=5.0, tau_inh=10.0, tau_ref=1.0, g_leak=0.2,
                               tau_nmda=20.0),
    # src/neuron_model/AdExTimeDrivenModel.cpp (GetDefaultParameters)
    "AdExTimeDrivenModel": dict(a=1.0, b=9.0, thr_slo_fac=2.0, v_thr=-50.0, tau_w=50.0,
                                e_exc=0.0, e_inh=-80.0, e_reset=-80.0, e_leak=-65.0,
                                g_leak=10.0, c_m=110.0, tau_exc=5.0, tau_inh=10.0,
                                tau_nmda=20.0),
    # src/neuron_model/HHTimeDrivenModel.cpp:491-505
    "HHTimeDrivenModel": dict(e_exc=0.0, e_inh=-80.0, e_leak=-65.0, g_leak=10.0, c_m=120.0,
                              v_thr=-52.0, tau_exc=5.0, tau_inh=10.0, tau_nmda=20.0,
                              g_na=20000.0, g_kd=6000.0, e_na=50.0, e_k=-90.0),
    # PoissonGeneratorDeviceVector::GetDefaultParameters (PoissonGeneratorDeviceVector.cpp:162-167)
    "PoissonGeneratorDeviceVector": dict(frequency=10.0),
}
for _n in list(MODEL_DEFAULTS):
    MODEL_DEFAULTS[_n + "_GPU"] = MODEL_DEFAULTS[_n]

INTEGRATORS = ("Euler", "RK2", "RK4", "BDF")
INPUT_MODELS = ("InputSpikeNeuronModel",)


def _f32(x: float) -> str:
    return "%.9g" % float(np.float32(x))


@dataclass
class Layer:
    """One layer line of the network file: ``n model param_file output log``."""
    n: int
    model: str
    params: Dict[str, float] = field(default_factory=dict)
    integrator: str = "Euler"
    dt: float = 1e-4
    bdf_order: int = 2
    output: int = 1
    log: int = 0
    name: Optional[str] = None  # parameter-file stem; derived when omitted

    def full_params(self) -> Dict[str, float]:
        p = dict(MODEL_DEFAULTS.get(self.model, {}))
        p.update(self.params)
        return p


@dataclass
class NetworkDescription:
    layers: List[Layer] = field(default_factory=list)
    # (name, [params in file order]); "STDP": max_LTP tau_LTP max_LTD tau_LTD
    rules: List[tuple] = field(default_factory=list)
    src: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    tgt: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    delay: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    stype: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    weight: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    max_weight: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    wchange: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))

    # ---- construction helpers -------------------------------------------------
    def add_layer(self, layer: Layer) -> range:
        start = self.n_neurons
        self.layers.append(layer)
        return range(start, start + layer.n)

    @property
    def n_neurons(self) -> int:
        return int(sum(l.n for l in self.layers))

    @property
    def n_synapses(self) -> int:
        return int(len(self.src))

    def add_synapses(self, src, tgt, delay, stype, weight, max_weight, wchange=-1):
        m = len(src)
        bc = lambda v, dt: np.broadcast_to(np.asarray(v, dt), (m,)).copy()
        self.src = np.concatenate([self.src, np.asarray(src, np.int64)])
        self.tgt = np.concatenate([self.tgt, np.asarray(tgt, np.int64)])
        self.delay = np.concatenate([self.delay, bc(delay, np.float32)])
        self.stype = np.concatenate([self.stype, bc(stype, np.int32)])
        self.weight = np.concatenate([self.weight, bc(weight, np.float32)])
        self.max_weight = np.concatenate([self.max_weight, bc(max_weight, np.float32)])
        self.wchange = np.concatenate([self.wchange, bc(wchange, np.int32)])

    def layer_of(self) -> np.ndarray:
        """Layer index of every neuron."""
        return np.repeat(np.arange(len(self.layers)), [l.n for l in self.layers])

    # ---- reference file formats ------------------------------------------------
    def _param_stem(self, i: int) -> str:
        l = self.layers[i]
        return l.name or ("layer%d_%s" % (i, l.model))

    def write_model_cfg(self, path_stem: str, layer: Layer) -> None:
        base = layer.model
        order = MODEL_PARAM_ORDER[base]
        p = layer.full_params()
        with open(path_stem + ".cfg", "w") as f:
            f.write("// %s parameters (one value per line, EDLUT .cfg layout)\n" % base)
            for k in order:
                f.write("// %s\n%s\n" % (k, _f32(p[k])))
            if base == "PoissonGeneratorDeviceVector":  # a device: no integration method
                return
            f.write("// integration method\n%s\n" % layer.integrator)
            if layer.integrator == "BDF":
                f.write("// BDF order\n%d\n" % layer.bdf_order)
            f.write("// integration step (s)\n%s\n" % _f32(layer.dt))

    def write_files(self, directory: str, stem: str = "net") -> tuple:
        """Write network, weights and model files; returns (netfile, weightsfile).

        Each synapse gets its own block line (``src 1 tgt 1 1 delay 0 type maxw rule``),
        which keeps the reference's original synapse index equal to ours.
        """
        os.makedirs(directory, exist_ok=True)
        for i, l in enumerate(self.layers):
            if l.model in MODEL_PARAM_ORDER:
                self.write_model_cfg(os.path.join(directory, self._param_stem(i)), l)
        netf = os.path.join(directory, stem + "_net.cfg")
        wf = os.path.join(directory, stem + "_weights.cfg")
        with open(netf, "w") as f:
            f.write("// network written by edlut_b200.network\n")
            f.write("%d\n%d\n" % (len(self.layers), self.n_neurons))
            for i, l in enumerate(self.layers):
                pf = self._param_stem(i) if l.model in MODEL_PARAM_ORDER else "Null"
                f.write("%d %s %s %d %d\n" % (l.n, l.model, pf, l.output, l.log))
            f.write("%d\n" % len(self.rules))
            for name, params in self.rules:
                f.write("%s %s\n" % (name, " ".join(_f32(v) for v in params)))
            f.write("%d\n" % self.n_synapses)
            # the line after "src 1 tgt 1 1" is shared by every synapse with the same
            # delay, type, max weight and rule: format each distinct one once
            cols = [np.unique(a, return_inverse=True) for a in
                    (self.delay.astype(np.float32), self.stype, self.max_weight.astype(np.float32), self.wchange)]
            key = np.zeros(self.n_synapses, np.int64)
            for u, inv in cols:
                key = key * len(u) + inv.reshape(-1)
            ukey, code = np.unique(key, return_inverse=True)
            tails = []
            for k in ukey.tolist():
                idx = []
                for u, _ in reversed(cols):
                    idx.append(k % len(u))
                    k //= len(u)
                (d, ty, mw, wc) = (cols[j][0][i] for j, i in enumerate(reversed(idx)))
                tails.append(" %s 0 %d %s %d\n" % (_f32(d), int(ty), _f32(mw), int(wc)))
            for lo in range(0, self.n_synapses, 1 << 20):
                hi = min(self.n_synapses, lo + (1 << 20))
                f.writelines(["%d 1 %d 1 1%s" % (s, t, tails[c]) for s, t, c in
                              zip(self.src[lo:hi].tolist(), self.tgt[lo:hi].tolist(),
                                  code.reshape(-1)[lo:hi].tolist())])
        with open(wf, "w") as f:
            w32 = self.weight.astype(np.float32)
            for lo in range(0, len(w32), 1 << 20):
                f.writelines(["1 %s\n" % v for v in np.char.mod("%.9g", w32[lo:lo + (1 << 20)].astype(np.float64)).tolist()])
        return netf, wf


def write_input_spikes(path: str, times: Sequence[float], cells: Sequence[int]) -> None:
    """Input-spike file: count, then ``time 1 0 cell 1`` per spike (times as float32)."""
    times = np.asarray(times, np.float32)
    cells = np.asarray(cells, np.int64)
    with open(path, "w") as f:
        f.write("%d\n" % len(times))
        f.writelines("%s 1 0 %d 1\n" % (_f32(t), c) for t, c in zip(times.tolist(), cells.tolist()))


def poisson_input_times(rng: np.random.Generator, n_inputs: int, rate_hz, t_end: float,
                        dt: float = 1e-4, t_start: float = 0.0, unique: bool = True) -> tuple:
    """Seeded Poisson spike lists for ``n_inputs`` input neurons, as (times, cells).

    Each input spikes in a step of length ``dt`` with probability rate*dt (at most
    once per step), drawn as geometric gaps between spike steps.  Times are float32
    and placed strictly inside a step window (10%..90% of the way between two update
    times) so that no input event coincides with a neuron update; every time is
    unique, so the reference's order of events at equal time stamps never matters
    (``unique=False`` skips that step, for throughput runs whose inputs are too dense
    for unique float32 times).  Sorted by time.
    """
    rate = np.broadcast_to(np.asarray(rate_hz, np.float64), (n_inputs,))
    k0 = int(round(t_start / dt))
    nsteps = int(round(t_end / dt)) - k0
    p = np.clip(rate * dt, 0.0, 1.0)
    mean = p * nsteps
    cap = int(np.max(mean + 8.0 * np.sqrt(mean + 1.0) + 8.0)) if n_inputs else 0
    steps_all, cells_all = [], []
    for lo in range(0, n_inputs, 4096):
        hi = min(n_inputs, lo + 4096)
        pp = np.maximum(p[lo:hi], 1e-300)
        gaps = rng.geometric(pp[:, None], size=(hi - lo, cap))
        st = np.cumsum(gaps, axis=1) - 1
        ok = st < nsteps
        ok &= (p[lo:hi] > 0)[:, None]
        r, c = np.nonzero(ok)
        steps_all.append(st[r, c] + k0)
        cells_all.append(r + lo)
    step = np.concatenate(steps_all) if steps_all else np.zeros(0, np.int64)
    cell = np.concatenate(cells_all) if cells_all else np.zeros(0, np.int64)
    frac = 0.1 + 0.8 * rng.random(len(step))
    times = ((step + frac) * dt).astype(np.float32)
    order = np.lexsort((cell, times))
    times, cell = times[order], cell[order]
    # make float32 times unique (nudge collisions up by one ulp)
    dup = np.nonzero(times[1:] <= times[:-1])[0] if unique else []
    while len(dup):
        for i in dup + 1:
            if times[i] <= times[i - 1]:
                times[i] = np.nextafter(times[i - 1], np.float32(np.inf))
        dup = np.nonzero(times[1:] <= times[:-1])[0]
    return times, cell.astype(np.int64)
