"""Generate the golden fixtures under tests/golden/ by running the reference EDLUT
CPU kernel (built from the reference sources by
``make -C oracle ref REF=<reference tree>/Kernel``, so this runs only where the
reference is mounted).

    python tests/golden/make_golden.py            # all small cases
    python tests/golden/make_golden.py c1_lif     # cases whose name contains 'c1_lif'
    python tests/golden/make_golden.py full       # the full-size benchmark cases (minutes)

Each case is a seeded network from edlut_b200.configs (so tests rebuild the same
network anywhere); the fixture ``<case>.npz`` holds what the reference produced:
spike steps and cells, the first state-variable traces of a few neurons, final
weights (plastic cases), a SHA-256 of the reference synapse order, and counts.
For FILE_CASES the reference's own output-spike (-of) and saved-weights (-sf)
files are kept as ``<case>.of.gz`` and ``<case>.sf.gz``.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from edlut_b200 import configs as C  # noqa: E402
from oracle import oracle as O       # noqa: E402

# name -> (builder, kwargs, nsteps, (trace_steps, trace_first, trace_n))
CASES = {
    "c1_lif_euler": ("lif_recurrent", {}, 10000, (1000, 100, 16)),
}
for _m in ("LIFTimeDrivenModel", "AdExTimeDrivenModel", "HHTimeDrivenModel"):
    for _i, _o in (("Euler", 1), ("RK2", 1), ("RK4", 1), ("BDF", 1), ("BDF", 2), ("BDF", 3), ("BDF", 4),
                   ("BDF", 5), ("BDF", 6)):
        _dt = 5e-5 if _m.startswith("HH") else 1e-4
        CASES["%s_%s%s_stdp" % (_m[:-15].lower(), _i.lower(), _o if _i == "BDF" else "")] = (
            "parity_network", dict(model=_m, integrator=_i, bdf_order=_o, stdp=True,
                                   delays=(1e-3, 2e-3, 1.5e-3), dt=_dt), 2000, (500, 40, 8))
# edge cases
CASES["lif_subdt_delays"] = ("parity_network", dict(model="LIFTimeDrivenModel", integrator="Euler",
                                                    delays=(1.5e-4, 1.49e-3, 2.3e-4), dt=1e-4, seed=3),
                             2000, (300, 40, 8))
# a 1 ms step with weights small enough that RK2 stays stable: finite dynamics
CASES["lif_coarse_dt"] = ("parity_network", dict(model="LIFTimeDrivenModel", integrator="RK2",
                                                 delays=(1e-4, 2e-4, 5e-4), dt=1e-3, seed=4, t_end=1.0,
                                                 weights=dict(w_in=0.15, w_exc=0.05, w_inh=0.2)),
                          1000, (300, 40, 8))
# the same step with the default weights: conductances past the explicit methods'
# stability bound, so V overflows to inf and NaN, which both sides must propagate
# (and reset) identically
CASES["lif_coarse_dt_overflow"] = ("parity_network", dict(model="LIFTimeDrivenModel", integrator="RK2",
                                                          delays=(1e-4, 2e-4, 5e-4), dt=1e-3, seed=4,
                                                          t_end=1.0),
                                   1000, (300, 40, 8))
CASES["adex_dense_fanin"] = ("parity_network", dict(model="AdExTimeDrivenModel", integrator="RK4", n=120,
                                                    p=0.6, stdp=True, seed=5, delays=(1e-3,)),
                             2000, (300, 40, 8))
CASES["cereb_small_rk4"] = ("cerebellar_layer", dict(n_granule=2000, n_mossy=100, n_purkinje=8,
                                                     pf_per_purkinje=1000, t_end=0.3),
                            3000, (300, 100, 8))
CASES["hh_small_bdf2"] = ("hh_network", dict(n=400, indeg=40, t_end=0.1), 2000, (400, 400, 8))
# device Poisson generators (PoissonGeneratorDeviceVector): two generator types, one
# of them split around the LIF layer (its seeds follow the first part's), STDP on
# the generator synapses
CASES["poisson_lif_rk2_stdp"] = ("poisson_network", dict(seed=6, w_in=0.05, w_exc=0.05, w_inh=0.5), 2000,
                                 (300, 70, 8))

# Fixtures that may hold non-finite state on purpose (every other fixture's traces
# are finite).
OVERFLOW_CASES = ("lif_coarse_dt_overflow",)

# The benchmark workloads at full size, over the first steps of their runs.  Their
# fixtures keep the spikes, the V traces of a few cells, counts and SHA-256 digests
# of the synapse order and of the final weights (with every 997th weight), instead
# of whole weight arrays.
#   c2_full_rk4: cerebellar layer, 250k AdEx granule + 200 LIF Purkinje x 50k
#                plastic synapses, RK4 at 0.1 ms; traces of 8 Purkinje cells
#   c3_full_bdf2: 100k HH neurons, in-degree 100, delays 1-5 ms, 200 Hz drive,
#                BDF2 at 0.05 ms, unique input times; traces of 8 HH cells
BIG_CASES = {
    "c2_full_rk4": ("cerebellar_layer", dict(t_end=0.052), 500, (500, 255000, 8)),
    "c3_full_bdf2": ("hh_network", dict(t_end=0.0102), 200, (200, 100000, 8)),
}


# cases whose reference output files (-of spikes, -sf weights) are kept as
# <case>.of.gz / <case>.sf.gz: one model population, so the reference writes a
# step's spikes in neuron order
FILE_CASES = ("adex_rk4_stdp",)

# cases whose model layer has its log column set; the reference's -logp state
# monitor file (every state variable of every neuron of the layer, each step) is
# kept as <case>.logp.gz.  Small networks: the file grows with neurons x steps.
for _m, _i in (("LIFTimeDrivenModel", "RK2"), ("AdExTimeDrivenModel", "RK4"), ("HHTimeDrivenModel", "BDF")):
    CASES["%s_logp" % _m[:-15].lower()] = (
        "parity_network", dict(model=_m, integrator=_i, bdf_order=2, n=24, n_inputs=12, stdp=True, seed=8, rate_hz=300.0,
                               delays=(1e-3, 2e-3), dt=5e-5 if _m.startswith("HH") else 1e-4), 200, (200, 12, 6))
LOG_CASES = ("lif_logp", "adex_logp", "hh_logp")


def build_case(name: str):
    builder, kw, nsteps, trace = CASES[name] if name in CASES else BIG_CASES[name]
    net, t, c = getattr(C, builder)(**kw)
    if name in LOG_CASES:
        for layer in net.layers:
            if layer.model != "InputSpikeNeuronModel":
                layer.log = 1
    return net, t, c, nsteps, trace


def perm_digest(perm: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(perm, np.int64).tobytes()).hexdigest()


def step_of_times(times: np.ndarray, dt: float, nsteps: int) -> np.ndarray:
    ts = O.step_times(dt, nsteps + 1)
    mid = (ts[1:] + ts[:-1]) / 2
    return np.searchsorted(mid, times)


def weights_digest(w: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(w, np.float32).tobytes()).hexdigest()


def make_big(name: str) -> dict:
    net, t, c, nsteps, trace = build_case(name)
    dt = next(l.dt for l in net.layers if l.model != "InputSpikeNeuronModel")
    with tempfile.TemporaryDirectory() as wd:
        R = O.run_reference(net, t, c, nsteps, wd, trace=trace)
    steps = step_of_times(R["spike_time"], dt, nsteps)
    order = np.lexsort((R["spike_cell"], steps))
    w = R["w_final"].astype(np.float32)
    out = dict(spike_step=steps[order].astype(np.int32), spike_cell=R["spike_cell"][order].astype(np.int32),
               trace=R["trace"][:, :, :1].astype(np.float32), counts=np.array(R["counts"], np.int64),
               perm_sha256=np.array(perm_digest(R["syn"]["orig"])), w_sha256=np.array(weights_digest(w)),
               w_sample=w[::997].copy())
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return dict(spikes=int(len(steps)), counts=[int(x) for x in R["counts"]])


def make(name: str) -> dict:
    if name in BIG_CASES:
        return make_big(name)
    net, t, c, nsteps, trace = build_case(name)
    dt = next(l.dt for l in net.layers if l.model != "InputSpikeNeuronModel")
    with tempfile.TemporaryDirectory() as wd:
        R = O.run_reference(net, t, c, nsteps, wd, trace=trace)
    steps = step_of_times(R["spike_time"], dt, nsteps)
    order = np.lexsort((R["spike_cell"], steps))
    nd = {"LIF": 1, "AdE": 2, "HHT": 4}
    model = next(l.model for l in net.layers
                 if l.model not in ("InputSpikeNeuronModel", "PoissonGeneratorDeviceVector"))
    out = dict(spike_step=steps[order].astype(np.int32), spike_cell=R["spike_cell"][order].astype(np.int32),
               trace=R["trace"][:, :, :nd[model[:3]]].astype(np.float32),
               counts=np.array(R["counts"], np.int64))
    if any(r >= 0 for r in net.wchange.tolist()):
        out["w_final"] = R["w_final"].astype(np.float32)
    out["perm_sha256"] = np.array(perm_digest(R["syn"]["orig"]))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    import gzip
    keep = ((("of_text", ".of.gz"), ("sf_text", ".sf.gz")) if name in FILE_CASES else ()) + \
        ((("logp_text", ".logp.gz"),) if name in LOG_CASES else ())
    for key, ext in keep:
        with gzip.GzipFile(os.path.join(HERE, name + ext), "wb", mtime=0) as f:
            f.write(R[key])
    return dict(spikes=int(len(steps)), counts=[int(x) for x in R["counts"]])


if __name__ == "__main__":
    if not O.ref_available():
        sys.exit("reference build missing: run `make -C oracle ref REF=<reference tree>/Kernel`")
    sel = sys.argv[1:]
    summary = {}
    for name in list(CASES) + list(BIG_CASES):
        if (sel and not any(s in name for s in sel)) or (not sel and name in BIG_CASES):
            continue
        summary[name] = make(name)
        print(name, summary[name], flush=True)
    manifest = os.path.join(HERE, "manifest.json")
    old = json.load(open(manifest)) if os.path.exists(manifest) else {}
    old.update(summary)
    with open(manifest, "w") as f:
        json.dump(old, f, indent=1, sort_keys=True)
