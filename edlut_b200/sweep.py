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
        self.explicit: list = [None] * n_networks
        self.n_obs = 0

    @classmethod
    def from_specs(cls, specs, n_steps_max: int, integrator: str = "RK2", dt: float = 1e-4,
                   delay: float = 1e-3, seed: int = 1, device: int = 0,
                   max_rate_hz: float = 200.0) -> "Sweep":
        """Build a sweep from :func:`edlut_b200.configs.sweep_networks` specifications."""
        sw = cls(len(specs), integrator, dt, delay, seed, device)
        for i, s in enumerate(specs):
            sw.set_network(i, s["n"], s["n_in"], s["n_exc"], s["params"], s.get("p", 0.0),
                           s.get("w_exc_max", 0.0), s.get("w_inh_max", 0.0), s.get("w_in_max", 0.0))
            if "src" in s:
                sw.set_synapses(i, s["src"], s["tgt"], s["w"])
                sw.explicit[i] = True
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

    def set_synapses(self, i: int, src, tgt, w) -> None:
        """Explicit connectivity of network i (sources: LIF neurons 0..n-1, then the
        inputs n..n+n_in-1), weights in this order."""
        s_ = np.ascontiguousarray(src, np.int32)
        t_ = np.ascontiguousarray(tgt, np.int32)
        w_ = np.ascontiguousarray(w, np.float32)
        check(self._L.eb_sweep_set_synapses(self._h, int(i), len(s_), _ptr(s_, c_i32p), _ptr(t_, c_i32p),
                                            _ptr(w_, c_f32p)))

    def set_params(self, i: int, params: dict) -> None:
        """New LIF parameters of network i (after build: from the next launch / reset)."""
        full = dict(self.params[i])
        full.update(params)
        pv = np.array([full[k] for k in MODEL_PARAM_ORDER[_LIF]], np.float32)
        check(self._L.eb_sweep_set_params(self._h, int(i), _ptr(pv, c_f32p)))
        self.params[i] = full

    def set_weights(self, w) -> None:
        """All weights (networks in order, each in its set_synapses order): a numpy
        array or a CUDA float32 tensor."""
        if hasattr(w, "data_ptr"):
            check(self._L.eb_sweep_set_weights(self._h, ctypes.c_void_p(w.data_ptr()), 1))
        else:
            a = np.ascontiguousarray(w, np.float32)
            check(self._L.eb_sweep_set_weights(self._h, a.ctypes.data_as(ctypes.c_void_p), 0))

    def get_weights(self) -> np.ndarray:
        w = np.zeros(max(self.info()["synapses"], 1), np.float32)
        check(self._L.eb_sweep_get_weights(self._h, w.ctypes.data_as(ctypes.c_void_p), 0))
        return w[:self.info()["synapses"]]

    def set_observed(self, idx) -> None:
        """Record V after every step of neurons idx[network][m]."""
        a = np.ascontiguousarray(idx, np.int32)
        self.n_obs = a.shape[1] if a.ndim == 2 else 0
        check(self._L.eb_sweep_set_observed(self._h, int(self.n_obs), _ptr(a.reshape(-1), c_i32p)))

    def trace(self, n_steps: int, out=None):
        """Observed traces [networks, n_steps, m] (into ``out``, a CUDA tensor, if given)."""
        if out is not None:
            check(self._L.eb_sweep_get_trace(self._h, ctypes.c_void_p(out.data_ptr()), 1))
            return out
        a = np.zeros((self.n_networks, n_steps, self.n_obs), np.float32)
        check(self._L.eb_sweep_get_trace(self._h, a.ctypes.data_as(ctypes.c_void_p), 0))
        return a

    def set_checkpoints(self, every: int) -> None:
        check(self._L.eb_sweep_set_checkpoints(self._h, int(every)))

    def adjoint(self, grad_trace, grad_w=None):
        """dL/d(params) [networks, 4] (g_leak, e_leak, tau_exc, tau_inh) and dL/dw for
        the checkpointed run just made.  grad_trace: numpy [networks, steps, m] or a
        CUDA tensor; grad_w: a CUDA tensor to fill (else a numpy array is returned)."""
        gp = np.zeros((self.n_networks, 4), np.float64)
        if hasattr(grad_trace, "data_ptr"):
            gt, gt_dev = ctypes.c_void_p(grad_trace.data_ptr()), 1
        else:
            g = np.ascontiguousarray(grad_trace, np.float32)
            gt, gt_dev = g.ctypes.data_as(ctypes.c_void_p), 0
        if grad_w is not None:
            check(self._L.eb_sweep_adjoint(self._h, gt, gt_dev, ctypes.c_void_p(grad_w.data_ptr()), 1,
                                           gp.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
            return gp, grad_w
        gw = np.zeros(max(self.info()["synapses"], 1), np.float32)
        check(self._L.eb_sweep_adjoint(self._h, gt, gt_dev, gw.ctypes.data_as(ctypes.c_void_p), 0,
                                       gp.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return gp, gw[:self.info()["synapses"]]

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
