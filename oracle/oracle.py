"""TEST INFRASTRUCTURE ONLY: ctypes front end of the CPU oracle (edlut_oracle.c).

Used by tests/, ``__graft_entry__.smoke()`` and bench.py's ``cpu_baseline`` leg as
the checker; the shipped library never imports it.  ``run()`` takes an
:class:`edlut_b200.network.NetworkDescription` plus input spikes and returns spikes,
state traces and final weights, in the float32 mirror of the reference CPU code
(``fp64=False``) or in FP64 with exact exponentials (``fp64=True``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

KIND = {"InputSpikeNeuronModel": 0, "LIFTimeDrivenModel": 1, "AdExTimeDrivenModel": 2,
        "HHTimeDrivenModel": 3, "PoissonGeneratorDeviceVector": 4}
INTEG = {"Euler": 0, "RK2": 1, "RK4": 2, "BDF": 3}
MAXV = 8


class EoPop(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("integ", ctypes.c_int32), ("bdf_order", ctypes.c_int32),
                ("first", ctypes.c_int32), ("n", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("dt", ctypes.c_float), ("params", ctypes.c_float * 16)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
        _lib.eo_run.restype = ctypes.c_int
        _lib.eo_round_delay.restype = ctypes.c_double
        _lib.eo_round_delay.argtypes = [ctypes.c_float]
        _lib.eo_set_seed.argtypes = [ctypes.c_uint32]
    return _lib


def set_seed(seed: int) -> None:
    """RandomGenerator::srand value for the Poisson generators (default 1)."""
    lib().eo_set_seed(int(seed))


def _p(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def pops_of(net):
    from edlut_b200.network import MODEL_PARAM_ORDER
    pops = (EoPop * len(net.layers))()
    first = 0
    for i, l in enumerate(net.layers):
        base = l.model[:-4] if l.model.endswith("_GPU") else l.model
        pops[i].kind = KIND[base]
        pops[i].integ = INTEG.get(l.integrator, 0)
        pops[i].bdf_order = l.bdf_order
        pops[i].first = first
        pops[i].n = l.n
        pops[i].dt = l.dt
        if base in MODEL_PARAM_ORDER:
            fp = l.full_params()
            for j, k in enumerate(MODEL_PARAM_ORDER[base]):
                pops[i].params[j] = fp[k]
        first += l.n
    return pops


def run(net, in_times, in_cells, nsteps: int, fp64: bool = False, trace=(0, 0, 0),
        spike_cap: int | None = None, tail: bool = False):
    """Run the oracle.  ``trace`` = (steps, first_cell, n_cells).

    Returns dict(spike_step, spike_cell, trace[steps, n, 8], w_final, sorted_perm, n_events).
    """
    L = lib()
    pops = pops_of(net)
    m = net.n_synapses
    src = np.ascontiguousarray(net.src, np.int64)
    tgt = np.ascontiguousarray(net.tgt, np.int64)
    delay = np.ascontiguousarray(net.delay, np.float32)
    stype = np.ascontiguousarray(net.stype, np.int32)
    w = np.ascontiguousarray(net.weight, np.float32)
    mw = np.ascontiguousarray(net.max_weight, np.float32)
    rule = np.ascontiguousarray(net.wchange, np.int32)
    stdp = np.ascontiguousarray(np.array([r[1] for r in net.rules], np.float32).reshape(-1), np.float32)
    if stdp.size == 0:
        stdp = np.zeros(4, np.float32)
    it = np.ascontiguousarray(in_times, np.float32)
    ic = np.ascontiguousarray(in_cells, np.int64)
    ts, tf, tn = trace
    tr = np.zeros((max(ts, 1), max(tn, 1), MAXV), np.float64)
    cap = spike_cap or (net.n_neurons * nsteps // 2 + 1024)
    ss = np.zeros(cap, np.int64)
    sc = np.zeros(cap, np.int64)
    wf = np.zeros(max(m, 1), np.float64)
    perm = np.zeros(max(m, 1), np.int64)
    nsp = ctypes.c_int64(0)
    nev = ctypes.c_int64(0)
    rc = L.eo_run(ctypes.c_int32(len(net.layers)), pops, ctypes.c_int64(net.n_neurons),
                  ctypes.c_int64(m), _p(src, ctypes.c_int64), _p(tgt, ctypes.c_int64),
                  _p(delay, ctypes.c_float), _p(stype, ctypes.c_int32), _p(w, ctypes.c_float),
                  _p(mw, ctypes.c_float), _p(rule, ctypes.c_int32),
                  ctypes.c_int32(len(net.rules)), _p(stdp, ctypes.c_float),
                  ctypes.c_int64(len(it)), _p(it, ctypes.c_float), _p(ic, ctypes.c_int64),
                  ctypes.c_int64(nsteps), ctypes.c_int32(1 if fp64 else 0), ctypes.c_int32(1 if tail else 0),
                  ctypes.c_int64(ts), ctypes.c_int64(tf), ctypes.c_int64(tn),
                  _p(tr, ctypes.c_double), ctypes.c_int64(cap), ctypes.byref(nsp),
                  _p(ss, ctypes.c_int64), _p(sc, ctypes.c_int64), _p(wf, ctypes.c_double),
                  _p(perm, ctypes.c_int64), ctypes.byref(nev))
    if rc != 0:
        raise RuntimeError("oracle eo_run failed with code %d" % rc)
    n = nsp.value
    return dict(spike_step=ss[:n].copy(), spike_cell=sc[:n].copy(), trace=tr[:ts, :tn],
                w_final=wf[:m], sorted_perm=perm[:m], n_events=nev.value)


def round_delay(d: float) -> float:
    return lib().eo_round_delay(ctypes.c_float(d))


# ---------------------------------------------------------------- reference ----
def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "ref_harness"))


def run_reference(net, in_times, in_cells, nsteps: int, workdir: str, trace=(0, 0, 0), exe: str | None = None):
    """Run the reference EDLUT CPU kernel (oracle/_ref/ref_harness, or the harness
    binary ``exe`` built against another build of the reference) on the same network.

    Returns dict(spike_time, spike_cell, trace[steps, n, nvars], syn (sorted records),
    w_final (original order), counts, of_text / sf_text / logp_text (bytes of the
    reference's output-spike, saved-weights and state-monitor files))."""
    from edlut_b200.network import write_input_spikes
    netf, wf = net.write_files(workdir)
    inp = os.path.join(workdir, "inputs.cfg")
    write_input_spikes(inp, in_times, in_cells)
    dt = next(l.dt for l in net.layers if l.model not in ("InputSpikeNeuronModel",))
    cmd = [exe or os.path.join(REF_DIR, "ref_harness"), os.path.basename(netf), os.path.basename(wf),
           "inputs.cfg", str(nsteps), repr(float(np.float32(dt))), "out"] + [str(x) for x in trace]
    r = subprocess.run(cmd, cwd=workdir, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference harness failed: %s %s" % (r.stdout[-1000:], r.stderr[-1000:]))
    raw = np.fromfile(os.path.join(workdir, "out.spikes"), np.uint8)
    rec = np.frombuffer(raw[8:].tobytes(), dtype=[("t", "<f8"), ("c", "<i8")])
    out = dict(spike_time=rec["t"].copy(), spike_cell=rec["c"].copy())
    if trace[2] > 0:
        raw = np.fromfile(os.path.join(workdir, "out.trace"), np.uint8)
        h = np.frombuffer(raw[:12].tobytes(), np.int32)
        out["trace"] = np.frombuffer(raw[12:].tobytes(), np.float32).reshape(h[0], h[1], h[2])
    raw = np.fromfile(os.path.join(workdir, "out.syn"), np.uint8)
    out["syn"] = np.frombuffer(raw[8:].tobytes(), dtype=[("orig", "<i8"), ("src", "<i8"), ("tgt", "<i8"),
                                                           ("delay", "<f8"), ("type", "<i4"), ("w", "<f4")])
    raw = np.fromfile(os.path.join(workdir, "out.wfinal"), np.uint8)
    out["w_final"] = np.frombuffer(raw[8:].tobytes(), np.float32).copy()
    with open(os.path.join(workdir, "out.counts")) as f:
        out["counts"] = [int(x) for x in f.read().split()]
    # the reference's own output files: spikes (-of) and weights (-sf)
    for key, ext in (("of_text", ".of"), ("sf_text", ".sf"), ("logp_text", ".logp")):
        path = os.path.join(workdir, "out" + ext)
        if os.path.exists(path):
            with open(path, "rb") as f:
                out[key] = f.read()
    return out


def step_times(dt: float, nsteps: int) -> np.ndarray:
    """Update times t_k, k=0..nsteps (t_0 = 0), accumulated as the reference does."""
    t = np.zeros(nsteps + 1, np.float64)
    d = float(np.float32(dt))
    acc = 0.0
    for k in range(1, nsteps + 1):
        acc += d
        t[k] = acc
    return t
