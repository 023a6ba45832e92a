"""Python front end of the device-resident network (the C ABI of include/edlut_b200.h).

``Simulation`` plays the role of the reference's ``Simulation`` /
``PySimulation_API`` for the time-driven path: build a network (from a
:class:`~edlut_b200.network.NetworkDescription` or from the reference's network
and weights files), inject input spikes, advance it step by step on the GPU and
read spikes, states and weights back.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import INTEGRATORS, KINDS, c_f32p, c_f64p, c_i32p, c_i64p, check, load
from .network import MODEL_PARAM_ORDER, NetworkDescription


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(ct)


class Simulation:
    """A network on one GPU.

    >>> sim = Simulation.from_description(net, device=0)
    >>> sim.inject_spikes(times, cells)
    >>> sim.run(10_000)
    >>> steps, cells = sim.spikes()
    """

    def __init__(self, device: int = 0, record_capacity: Optional[int] = None,
                 graph_steps: int = 0, bucket_limit: int = 0, input_multiplicity: int = 0,
                 persistent: bool = False, random_seed: Optional[int] = None,
                 wide_indegree: Optional[int] = None):
        L = load()
        h = ctypes.c_void_p()
        check(L.eb_ctx_create(device, None, ctypes.byref(h)))
        self._h = h
        self._L = L
        self.device = device
        self.n_synapses = 0
        self.sorted_perm = None
        if record_capacity is not None:
            check(L.eb_set_record_capacity(h, int(record_capacity)))
        if graph_steps:
            check(L.eb_set_graph_steps(h, int(graph_steps)))
        check(L.eb_set_persistent(h, 1 if persistent else 0))
        if random_seed is not None:
            check(L.eb_set_random_seed(h, int(random_seed)))
        if bucket_limit or input_multiplicity:
            check(L.eb_set_bucket_limit(h, int(bucket_limit), int(input_multiplicity)))
        if wide_indegree is not None:
            check(L.eb_set_wide_indegree(h, int(wide_indegree)))

    # ------------------------------------------------------------ building --
    @classmethod
    def from_description(cls, net: NetworkDescription, device: int = 0, **kw) -> "Simulation":
        sim = cls(device=device, **kw)
        for q, layer in enumerate(net.layers):
            sim.add_population(layer.model, layer.n, layer.integrator, layer.bdf_order, layer.dt,
                               layer.full_params() if layer.model in MODEL_PARAM_ORDER else None)
            if layer.log:
                sim.set_monitor(q, True)
        for name, params in net.rules:
            if name != "STDP":
                raise NotImplementedError("learning rule %s is outside this path (only STDP)" % name)
            sim.add_stdp_rule(*params)
        sim.set_connectivity(net.src, net.tgt, net.delay, net.stype, net.weight, net.max_weight,
                             net.wchange)
        sim.finalize()
        return sim

    @classmethod
    def from_files(cls, network_file: str, weights_file: str, device: int = 0, **kw) -> "Simulation":
        """Load a reference network file and weights file (EDLUT text formats)."""
        sim = cls(device=device, **kw)
        check(sim._L.eb_load_network_files(sim._h, network_file.encode(), weights_file.encode()))
        return sim

    def add_population(self, model: str, n: int, integrator: str = "Euler", bdf_order: int = 2,
                       dt: float = 1e-4, params: Optional[dict] = None) -> int:
        base = model[:-4] if model.endswith("_GPU") else model
        kind = KINDS[base]
        first = ctypes.c_int64(0)
        if kind == 0:
            check(self._L.eb_add_population(self._h, 0, int(n), 0, 0, ctypes.c_float(0.0), None, 0,
                                            ctypes.byref(first)))
        else:
            order = MODEL_PARAM_ORDER[base]
            pv = np.array([params[k] for k in order], np.float32)
            check(self._L.eb_add_population(self._h, kind, int(n), INTEGRATORS[integrator], int(bdf_order),
                                            ctypes.c_float(dt), _ptr(pv, c_f32p), len(pv),
                                            ctypes.byref(first)))
        return first.value

    def add_stdp_rule(self, max_ltp, tau_ltp, max_ltd, tau_ltd) -> int:
        r = ctypes.c_int(0)
        check(self._L.eb_add_stdp_rule(self._h, ctypes.c_float(max_ltp), ctypes.c_float(tau_ltp),
                                       ctypes.c_float(max_ltd), ctypes.c_float(tau_ltd), ctypes.byref(r)))
        return r.value

    def set_connectivity(self, src, tgt, delay, stype, weight, max_weight, rule=None) -> None:
        m = len(src)
        self._syn = dict(
            src=np.ascontiguousarray(src, np.int64), tgt=np.ascontiguousarray(tgt, np.int64),
            delay=np.ascontiguousarray(delay, np.float32), stype=np.ascontiguousarray(stype, np.int32),
            weight=np.ascontiguousarray(weight, np.float32),
            maxw=np.ascontiguousarray(max_weight, np.float32),
            rule=np.ascontiguousarray(rule if rule is not None else np.full(m, -1), np.int32))
        s = self._syn
        check(self._L.eb_set_connectivity(self._h, m, _ptr(s["src"], c_i64p), _ptr(s["tgt"], c_i64p),
                                          _ptr(s["delay"], c_f32p), _ptr(s["stype"], c_i32p),
                                          _ptr(s["weight"], c_f32p), _ptr(s["maxw"], c_f32p),
                                          _ptr(s["rule"], c_i32p)))
        self.n_synapses = m

    def finalize(self) -> np.ndarray:
        perm = np.zeros(max(self.n_synapses, 1), np.int64)
        check(self._L.eb_finalize(self._h, _ptr(perm, c_i64p)))
        self._syn = None
        self.sorted_perm = perm[:self.n_synapses]
        return self.sorted_perm

    # ------------------------------------------------------------- running --
    def set_poisson_rates(self, first: int, rates_hz) -> None:
        """Per-neuron frequencies of Poisson generator neurons first, first+1, ..."""
        r = np.ascontiguousarray(rates_hz, np.float32)
        check(self._L.eb_set_poisson_rates(self._h, int(first), len(r), _ptr(r, c_f32p)))

    def inject_spikes(self, times: Sequence[float], cells: Sequence[int]) -> None:
        t = np.ascontiguousarray(times, np.float32)
        c = np.ascontiguousarray(cells, np.int64)
        check(self._L.eb_inject_spikes(self._h, len(t), _ptr(t, c_f32p), _ptr(c, c_i64p)))

    def load_input_file(self, path: str) -> None:
        check(self._L.eb_load_input_file(self._h, path.encode()))

    def run(self, n_steps: int) -> None:
        check(self._L.eb_run(self._h, int(n_steps)))

    def run_async(self, n_steps: int) -> None:
        check(self._L.eb_run_async(self._h, int(n_steps)))

    def sync(self) -> None:
        check(self._L.eb_sync(self._h))

    # ------------------------------------------------------------- outputs --
    def spikes(self):
        """Drain recorded spikes: (step [1-based], cell), sorted by (step, cell)."""
        n = ctypes.c_int64(0)
        rc = self._L.eb_get_spikes(self._h, 0, ctypes.byref(n), None, None)
        if rc not in (0, -4):
            check(rc)
        steps = np.zeros(max(n.value, 1), np.int64)
        cells = np.zeros(max(n.value, 1), np.int64)
        check(self._L.eb_get_spikes(self._h, n.value, ctypes.byref(n), _ptr(steps, c_i64p),
                                    _ptr(cells, c_i64p)))
        return steps[:n.value], cells[:n.value]

    def step_time(self, k: int) -> float:
        t = ctypes.c_double(0)
        check(self._L.eb_step_time(self._h, int(k), ctypes.byref(t)))
        return t.value

    def get_state(self, first: int, n: int, var: int = 0) -> np.ndarray:
        out = np.zeros(n, np.float32)
        check(self._L.eb_get_state(self._h, int(first), int(n), int(var), _ptr(out, c_f32p)))
        return out

    def set_state(self, first: int, values, var: int = 0) -> None:
        v = np.ascontiguousarray(values, np.float32)
        check(self._L.eb_set_state(self._h, int(first), len(v), int(var), _ptr(v, c_f32p)))

    def set_trace(self, first: int, n: int, steps: int) -> None:
        check(self._L.eb_set_trace(self._h, int(first), int(n), int(steps)))
        self._trace_shape = (steps, n, 8)

    def get_trace(self) -> np.ndarray:
        out = np.zeros(self._trace_shape, np.float32)
        check(self._L.eb_get_trace(self._h, _ptr(out, c_f32p)))
        return out

    def weights(self) -> np.ndarray:
        w = np.zeros(max(self.n_synapses, 1), np.float32)
        check(self._L.eb_get_weights(self._h, _ptr(w, c_f32p)))
        return w[:self.n_synapses]

    def write_spikes(self, path: str, append: bool = False) -> None:
        """Drain recorded spikes into `path` in the reference's -of file format."""
        check(self._L.eb_write_spikes(self._h, os.fsencode(path), int(bool(append))))

    def set_output(self, pop: int, on: bool = True) -> None:
        check(self._L.eb_set_output(self._h, int(pop), int(bool(on))))

    def set_monitor(self, pop: int, on: bool = True) -> None:
        """Monitor the states of population `pop` (the layer line's log column)."""
        check(self._L.eb_set_monitor(self._h, int(pop), int(bool(on))))

    def open_monitor(self, path: str, chunk_steps: int = 0, delivery_capacity: int = 0) -> None:
        """Write the monitored populations' states to `path` in the reference's -logp
        format as the following runs advance (``run`` only, not ``run_async``)."""
        check(self._L.eb_open_monitor(self._h, os.fsencode(path), int(chunk_steps), int(delivery_capacity)))

    def close_monitor(self) -> None:
        check(self._L.eb_close_monitor(self._h))

    def save_weights(self, path: str) -> None:
        """Write the weights in the reference's weights-file format (-sf)."""
        check(self._L.eb_save_weights(self._h, os.fsencode(path)))

    def set_weights(self, w) -> None:
        w = np.ascontiguousarray(w, np.float32)
        check(self._L.eb_set_weights(self._h, _ptr(w, c_f32p)))

    def counters(self):
        s, sp, ev = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
        check(self._L.eb_get_counters(self._h, ctypes.byref(s), ctypes.byref(sp), ctypes.byref(ev)))
        return dict(steps=s.value, spikes=sp.value, events=ev.value)

    def population_events(self, pop: int) -> int:
        """Synaptic events delivered into population ``pop`` (layer index)."""
        e = ctypes.c_int64(0)
        check(self._L.eb_get_population_events(self._h, int(pop), ctypes.byref(e)))
        return e.value

    def launch_count(self) -> int:
        """Kernels launched so far (graph nodes counted per replay)."""
        n = ctypes.c_int64(0)
        check(self._L.eb_launch_count(self._h, ctypes.byref(n)))
        return n.value

    def device_bytes(self) -> int:
        b = ctypes.c_int64(0)
        check(self._L.eb_device_bytes(self._h, ctypes.byref(b)))
        return b.value

    def snapshot(self, slot: int = 0) -> None:
        check(self._L.eb_snapshot(self._h, int(slot)))

    def restore(self, slot: int = 0) -> None:
        check(self._L.eb_restore(self._h, int(slot)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.eb_ctx_destroy(self._h)
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
