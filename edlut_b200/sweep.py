"""Batched parameter sweep: many independent LIF networks in one persistent kernel.

``Sweep`` wraps the ``eb_sweep_*`` entry points of include/edlut_b200.h.  Each
network is one LIF population (80/20 excitatory/inhibitory sources) plus input
neurons driven by given spike times, Bernoulli(p) connectivity generated on the
device, one delay, static weights.  Every network's spike train equals a run of
the same network alone on the plain path (:class:`~edlut_b200.simulation.Simulation`);
:meth:`Sweep.solo_description` builds that network.

>>> specs = sweep_networks(n_networks=4096)
>>> sw = Sweep.from_specs(specs, n_steps_max=10_000)
>>> sw.autotune(500)
>>> sw.run(10_000)
>>> steps, cells = sw.spikes(17)
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from ._lib import INTEGRATORS, c_f32p, c_i32p, c_i64p, check, load
from .network import MODEL_DEFAULTS, MODEL_PARAM_ORDER, Layer, NetworkDescription

_LIF = "LIFTimeDrivenModel"


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(ct)


class Sweep:
    def __init__(self, n_networks: int, integrator: str = "RK2", dt: float = 1e-4,
                 delay: float = 1e-3, seed: int = 1, device: int = 0):
        L = load()
        h = ctypes.c_void_p()
        check(L.eb_sweep_create(device, int(n_networks), INTEGRATORS[integrator], ctypes.c_float(dt),
                                ctypes.c_float(delay), ctypes.c_uint64(seed), ctypes.byref(h)))
        self._h, self._L = h, L
        self.n_networks = n_networks
        self.integrator, self.dt, self.delay, self.seed, self.device = integrator, dt, delay, seed, device
        self.sizes = np.zeros(n_networks, np.int64)
        self.n_inputs = np.zeros(n_networks, np.int64)
        self.n_exc = np.zeros(n_networks, np.int64)
        self.params: list = [None] * n_networks
        self.inputs: list = [None] * n_networks

    @classmethod
    def from_specs(cls, specs, n_steps_max: int, integrator: str = "RK2", dt: float = 1e-4,
                   delay: float = 1e-3, seed: int = 1, device: int = 0,
                   max_rate_hz: float = 200.0) -> "Sweep":
        """Build a sweep from :func:`edlut_b200.configs.sweep_networks` specifications."""
        sw = cls(len(specs), integrator, dt, delay, seed, device)
        for i, s in enumerate(specs):
            sw.set_network(i, s["n"], s["n_in"], s["n_exc"], s["params"], s["p"], s["w_exc_max"],
                           s["w_inh_max"], s["w_in_max"])
            sw.set_inputs(i, s["times"], s["cells"])
        sw.build(n_steps_max, max_rate_hz)
        return sw

    # ------------------------------------------------------------ building --
    def set_network(self, i: int, n: int, n_in: int, n_exc: int, params: dict, p: float,
                    w_exc_max: float, w_inh_max: float, w_in_max: float) -> None:
        full = dict(MODEL_DEFAULTS[_LIF])
        full.update(params)
        pv = np.array([full[k] for k in MODEL_PARAM_ORDER[_LIF]], np.float32)
        check(self._L.eb_sweep_set_network(self._h, int(i), int(n), int(n_in), int(n_exc), _ptr(pv, c_f32p),
                                           ctypes.c_float(p), ctypes.c_float(w_exc_max),
                                           ctypes.c_float(w_inh_max), ctypes.c_float(w_in_max)))
        self.sizes[i], self.n_inputs[i], self.n_exc[i] = n, n_in, n_exc
        self.params[i] = full

    def set_inputs(self, i: int, times, cells) -> None:
        t = np.ascontiguousarray(times, np.float32)
        c = np.ascontiguousarray(cells, np.int32)
        check(self._L.eb_sweep_set_inputs(self._h, int(i), len(t), _ptr(t, c_f32p), _ptr(c, c_i32p)))
        self.inputs[i] = (t, c)

    def build(self, n_steps_max: int, max_rate_hz: float = 200.0) -> None:
        check(self._L.eb_sweep_build(self._h, int(n_steps_max), ctypes.c_float(max_rate_hz)))

    def configure(self, block: int = 0, steps_per_launch: int = 0) -> None:
        check(self._L.eb_sweep_configure(self._h, int(block), int(steps_per_launch)))

    def autotune(self, trial_steps: int = 500) -> dict:
        b, s, ms = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_float(0)
        check(self._L.eb_sweep_autotune(self._h, int(trial_steps), ctypes.byref(b), ctypes.byref(s),
                                        ctypes.byref(ms)))
        return dict(block=b.value, steps_per_launch=s.value, trial_ms=ms.value)

    # ------------------------------------------------------------- running --
    def reset(self) -> None:
        check(self._L.eb_sweep_reset(self._h))

    def run(self, n_steps: int) -> None:
        check(self._L.eb_sweep_run(self._h, int(n_steps)))

    def run_async(self, n_steps: int) -> None:
        check(self._L.eb_sweep_run_async(self._h, int(n_steps)))

    def sync(self) -> None:
        check(self._L.eb_sweep_sync(self._h))

    def stream(self) -> int:
        s = ctypes.c_void_p()
        check(self._L.eb_sweep_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    # ------------------------------------------------------------- outputs --
    def spikes(self, i: int):
        """Spikes of network i: (step [1-based], neuron), sorted by (step, neuron)."""
        n = ctypes.c_int64(0)
        rc = self._L.eb_sweep_get_spikes(self._h, int(i), 0, ctypes.byref(n), None, None)
        if rc not in (0, -4) or (rc == -4 and n.value == 0):
            check(rc)
        st = np.zeros(max(n.value, 1), np.int32)
        ce = np.zeros(max(n.value, 1), np.int32)
        check(self._L.eb_sweep_get_spikes(self._h, int(i), n.value, ctypes.byref(n), _ptr(st, c_i32p),
                                          _ptr(ce, c_i32p)))
        return st[:n.value].astype(np.int64), ce[:n.value].astype(np.int64)

    def spike_counts(self) -> np.ndarray:
        c = np.zeros(self.n_networks, np.int64)
        check(self._L.eb_sweep_spike_counts(self._h, _ptr(c, c_i64p)))
        return c

    def synapses(self, i: int):
        """Synapses of network i in delivery order: (source, target, weight)."""
        m = ctypes.c_int64(0)
        rc = self._L.eb_sweep_get_synapses(self._h, int(i), 0, ctypes.byref(m), None, None, None)
        if rc not in (0, -4):
            check(rc)
        src = np.zeros(max(m.value, 1), np.int32)
        tgt = np.zeros(max(m.value, 1), np.int32)
        w = np.zeros(max(m.value, 1), np.float32)
        check(self._L.eb_sweep_get_synapses(self._h, int(i), m.value, ctypes.byref(m), _ptr(src, c_i32p),
                                            _ptr(tgt, c_i32p), _ptr(w, c_f32p)))
        return src[:m.value], tgt[:m.value], w[:m.value]

    def state(self, i: int, var: int = 0) -> np.ndarray:
        out = np.zeros(int(self.sizes[i]), np.float32)
        check(self._L.eb_sweep_get_state(self._h, int(i), int(var), _ptr(out, c_f32p)))
        return out

    def info(self) -> dict:
        syn, nb, ev = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
        b, s, g = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        check(self._L.eb_sweep_info(self._h, ctypes.byref(syn), ctypes.byref(nb), ctypes.byref(ev),
                                    ctypes.byref(b), ctypes.byref(s), ctypes.byref(g)))
        return dict(synapses=syn.value, device_bytes=nb.value, events=ev.value, block=b.value,
                    steps_per_launch=s.value, grid=g.value)

    def solo_description(self, i: int):
        """Network i alone, for the plain path: (NetworkDescription, input times, input
        cells).  The LIF layer comes first (neurons 0..n-1, as in the sweep), the input
        neurons after it."""
        n, n_in, n_exc = int(self.sizes[i]), int(self.n_inputs[i]), int(self.n_exc[i])
        net = NetworkDescription()
        net.add_layer(Layer(n, _LIF, dict(self.params[i]), integrator=self.integrator, dt=self.dt,
                            name="sweep_lif_%d" % i))
        inp = net.add_layer(Layer(n_in, "InputSpikeNeuronModel", output=0))
        src, tgt, w = self.synapses(i)
        stype = ((src >= n_exc) & (src < n)).astype(np.int32)
        net.add_synapses(src.astype(np.int64), tgt.astype(np.int64), self.delay, stype, w, w, -1)
        t, c = self.inputs[i]
        return net, t, c.astype(np.int64) + inp.start

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.eb_sweep_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
