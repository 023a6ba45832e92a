#!/usr/bin/env python3
"""Benchmark of the time-driven simulation path on B200.

Workload (single-GPU): the cerebellar-layer network -- 250,000 granule-like AdEx
neurons, each with in-degree 4 from 5,000 Poisson mossy fibres (5-50 Hz uniform),
plus 200 Purkinje-like LIF neurons each receiving 50,000 granule synapses with
additive exponential STDP (A+ 1e-3, A- 1.05e-3, tau 20 ms); RK4, dt = 0.1 ms,
float32; synthetic seeded inputs (no dataset).  One benchmark step = 1,000
integration steps (100 ms of simulated time) of that network, continuing the
same simulation.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  ``value`` is neuron-updates/s with the inputs
already in HBM (device time, CUDA events on the library's stream, L2 flushed
between benchmark steps); ``e2e`` is the same metric through the public API with
the step's input spikes copied in from host memory and its spikes read back.
``--impl reference`` times the reference EDLUT CPU kernel (built from the
reference sources into oracle/_ref) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "neuron-updates/s"
UNIT = "neuron-updates/s"
STEPS_PER_BENCH_STEP = 1000
DT = 1e-4
WORKLOAD = "cerebellar-layer: 250k AdEx granule (in-degree 4 from 5k Poisson mossy 5-50 Hz) + 200 LIF Purkinje x 50k plastic granule synapses, STDP A+1e-3 A-1.05e-3 tau 20 ms, RK4 dt 0.1 ms, fp32"
BYTES_PER_UNIT = {"AdEx": 32, "LIF": 32, "HH": 48}  # algorithmic bytes per neuron-update
EVENT_BYTES = 8


def max_over_ranks(x: float, world: int) -> float:
    """The slowest rank's value (the job's time): all-reduce MAX over the process
    group, on the GPU with NCCL, on the CPU with gloo."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_seed(base: int, rank: int) -> int:
    """Workload seed of a replica: every rank simulates its own networks."""
    return base + rank


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML queries every 5 ms from a thread (read-only), or nvidia-smi at
    its 200 ms period where NVML cannot be opened."""

    # nvmlClocksEventReason* bits
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, gpu_index: int):
        self.proc = None
        self.thread = None
        self.samples = []
        try:
            self._start_nvml(gpu_index)
            return
        except Exception:
            self.thread = None
        self.path = tempfile.mktemp(prefix="clocks_", suffix=".csv")
        if shutil.which("nvidia-smi"):
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)

    def _start_nvml(self, gpu_index: int):
        import threading
        import pynvml as nv
        import torch
        nv.nvmlInit()
        try:
            pr = torch.cuda.get_device_properties(gpu_index)
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            h = nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            h = nv.nvmlDeviceGetHandleByIndex(gpu_index)
        self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        self.stop_flag = threading.Event()

        def loop():
            while not self.stop_flag.is_set():
                try:
                    self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), int(reasons(h))))
                except Exception:
                    pass
                self.stop_flag.wait(0.005)

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            if not self.samples:
                return None
            found = set()
            for _, bits in self.samples:
                found |= {n for n, b in self.REASONS.items() if bits & b}
            return {"sm_mhz": statistics.median(m for m, _ in self.samples), "sm_max_mhz": self.max_mhz,
                    "reasons": sorted(found), "samples": len(self.samples), "source": "NVML every 5 ms"}
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi every 200 ms"}


def build_workload(seed: int, t_end: float, scale: float = 1.0):
    from edlut_b200 import configs
    n_g = int(250_000 * scale)
    n_mf = max(1, int(5_000 * scale))
    n_pc = max(1, int(200 * scale))
    k = int(50_000 * scale)
    return configs.cerebellar_layer(seed=seed, n_granule=n_g, n_mossy=n_mf, n_purkinje=n_pc,
                                    pf_per_purkinje=k, t_end=t_end)


def layer_starts(net):
    """First neuron of each layer, plus the total."""
    return [int(x) for x in np.cumsum([0] + [l.n for l in net.layers])]


def roofline_bytes(net, pop_events, pop_spikes, n_int, window=1):
    """Algorithmic bytes per launch of each profiled kernel, keyed like the profile
    ("update[granule]", ...), from the events delivered into each population and the
    spikes of each population over `n_int` integration steps, for launches that run
    `window` steps.  Every unit counts for every step of the window: BYTES_PER_UNIT
    per neuron-update (the state read and written once per step, although a launch
    keeps it in registers between its steps), 8 B per delivered event (+8 B when the
    synapse is plastic) and 8 B per fanned-out event.  "post_stdp[...]" is the
    post-synaptic STDP of a population per integration step (8 B per plastic input
    synapse per spike); it runs deferred, inside the update and the flush kernels,
    so it counts only in the whole step's figure."""
    src = np.asarray(net.src)
    tgt = np.asarray(net.tgt)
    plastic = np.asarray(net.wchange) >= 0
    starts = layer_starts(net)
    out = {}
    for q, l in enumerate(net.layers):
        in_pop = (tgt >= starts[q]) & (tgt < starts[q + 1])
        frac_plastic = float(plastic[in_pop].mean()) if in_pop.any() else 0.0
        if l.model != "InputSpikeNeuronModel":
            mdl = "AdEx" if "AdEx" in l.model else "HH" if "HH" in l.model else "LIF"
            unit = BYTES_PER_UNIT[mdl] + (96 if mdl == "HH" and l.integrator == "BDF" else 0)
            ev = pop_events[q] / n_int
            out["update[%s]" % l.name] = window * (unit * l.n + EVENT_BYTES * ev * (1.0 + frac_plastic))
            if frac_plastic > 0:
                per_neuron = int((in_pop & plastic).sum()) / max(1, l.n)
                out["post_stdp[%s]" % l.name] = EVENT_BYTES * per_neuron * pop_spikes[q] / n_int
        # fan-out launched from this population's spikes: 8 B per event it writes
        from_pop = (src >= starts[q]) & (src < starts[q + 1])
        if from_pop.any():
            tq = np.searchsorted(starts, tgt[from_pop], side="right") - 1
            ev_out = sum(pop_events[t] for t in set(tq.tolist()))
            # input spikes fan out in their own kernel; model neurons' spikes inside the
            # population's update kernel
            key = "input_push[-]" if l.model == "InputSpikeNeuronModel" else "update[%s]" % l.name
            out[key] = out.get(key, 0.0) + window * EVENT_BYTES * ev_out / n_int
    return out


# ------------------------------------------------------------- our arm ----
def run_ours(args):
    import torch
    rank, world, local = env_rank()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    from edlut_b200.simulation import Simulation
    from edlut_b200 import _lib

    W, K = args.warmup, args.steps
    prof_steps = 1
    total_bench = W + K + prof_steps + K  # warmup, timed, profiled, e2e
    t_total = (total_bench * STEPS_PER_BENCH_STEP + 10) * DT
    net, tin, cin = build_workload(seed=rank_seed(1, rank), t_end=t_total, scale=args.scale)
    n_model = sum(l.n for l in net.layers if l.model != "InputSpikeNeuronModel")
    sim = Simulation.from_description(net, device=dev, record_capacity=8 << 20)
    L = _lib.load()
    import ctypes
    sp = ctypes.c_void_p()
    _lib.check(L.eb_stream(sim._h, ctypes.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value, device=torch.device("cuda", dev))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    # inputs of warmup + timed + profiled steps resident in HBM before timing
    n_dev_steps = (W + K + prof_steps) * STEPS_PER_BENCH_STEP
    t_dev_end = sim.step_time(n_dev_steps)
    sel = tin < t_dev_end
    sim.inject_spikes(tin[sel], cin[sel])
    _lib.check(L.eb_prestage(sim._h, n_dev_steps))

    for _ in range(W):
        sim.run(STEPS_PER_BENCH_STEP)
    sim.spikes()
    c0 = sim.counters()
    pe0 = [sim.population_events(q) for q in range(len(net.layers))]
    l0 = ctypes.c_int64(0)
    _lib.check(L.eb_launch_count(sim._h, ctypes.byref(l0)))
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    for i in range(K):
        with torch.cuda.stream(stream):
            flush.fill_(i & 0xff)  # evict L2 between benchmark steps (outside the timed events)
            ev[i][0].record(stream)
        sim.run_async(STEPS_PER_BENCH_STEP)
        ev[i][1].record(stream)
    sim.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    c1 = sim.counters()
    l1 = ctypes.c_int64(0)
    _lib.check(L.eb_launch_count(sim._h, ctypes.byref(l1)))
    sec = ms / 1e3
    sec = max_over_ranks(sec, world)
    updates_rank = n_model * STEPS_PER_BENCH_STEP * K
    events_rank = c1["events"] - c0["events"]
    spikes_rank = c1["spikes"] - c0["spikes"]
    pop_events = [sim.population_events(q) - pe0[q] for q in range(len(net.layers))]
    _, sp_cells = sim.spikes()
    starts = layer_starts(net)
    pop_spikes = [int(((sp_cells >= starts[q]) & (sp_cells < starts[q + 1])).sum()) for q in range(len(net.layers))]

    # per-kernel durations: the same steps replayed as a graph with event-record
    # nodes around every kernel on the stream it runs on
    _lib.check(L.eb_set_profile(sim._h, 1))
    for _ in range(prof_steps):
        sim.run(STEPS_PER_BENCH_STEP)  # a multiple of 8: the run path's 8-step windows
    n = ctypes.c_int(0)
    cap = 64
    kinds = (ctypes.c_int * cap)()
    popi = (ctypes.c_int * cap)()
    lau = (ctypes.c_int64 * cap)()
    tms = (ctypes.c_double * cap)()
    _lib.check(L.eb_get_profile(sim._h, cap, ctypes.byref(n), kinds, popi, lau, tms))
    _lib.check(L.eb_set_profile(sim._h, 0))
    kind_names = {0: "input_push", 1: "update", 2: "post_stdp", 3: "push", 4: "flush_post"}
    prof = []
    for i in range(n.value):
        pname = net.layers[popi[i]].name if popi[i] >= 0 else "-"
        prof.append(dict(kernel="%s[%s]" % (kind_names[kinds[i]], pname), launches=int(lau[i]),
                         total_ms=float(tms[i]), avg_us=1e3 * float(tms[i]) / max(1, int(lau[i]))))
    tot = sum(p["total_ms"] for p in prof) or 1.0
    for p in prof:
        p["share"] = p["total_ms"] / tot
    prof.sort(key=lambda p: -p["total_ms"])
    sim.spikes()

    # end to end through the public API: host input arrays in, spikes out
    e2e_s = 0.0
    h2d = d2h = 0
    for i in range(K):
        k_lo = sim.counters()["steps"]
        t_lo, t_hi = sim.step_time(k_lo), sim.step_time(k_lo + STEPS_PER_BENCH_STEP)
        m = (tin >= t_lo) & (tin < t_hi)
        ht = np.ascontiguousarray(tin[m])
        hc = np.ascontiguousarray(cin[m])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.inject_spikes(ht, hc)
        sim.run(STEPS_PER_BENCH_STEP)
        st, ce = sim.spikes()
        e2e_s += time.perf_counter() - t0
        h2d += int(m.sum()) * (8 + 4) + (STEPS_PER_BENCH_STEP + 1) * 8
        d2h += len(st) * 8 + 8
    e2e_s = max_over_ranks(e2e_s, world)

    # roofline: algorithmic bytes of each kernel per launch -- a launch runs
    # `window` steps of its population (neuron state read and written once per
    # launch, BYTES_PER_UNIT per neuron; per delivered event 8 B, +8 B when the
    # synapse is plastic, and 8 B per fanned-out event, every step) -- divided by
    # its measured average launch time
    peak, peak_kind = measured_peaks()
    n_int = STEPS_PER_BENCH_STEP * K
    n_prof_steps = prof_steps * STEPS_PER_BENCH_STEP
    for p in prof:
        window = max(1, round(n_prof_steps / max(1, p["launches"]))) if p["kernel"].startswith(("update", "input")) else 1
        p["steps_per_launch"] = window
        alg = roofline_bytes(net, pop_events, pop_spikes, n_int, window)
        p["alg_bytes_per_launch"] = alg.get(p["kernel"])
        p["achieved_gbs"] = (p["alg_bytes_per_launch"] / (p["avg_us"] * 1e-6) / 1e9
                             if p["alg_bytes_per_launch"] is not None else None)
    top = next(p for p in prof if p["alg_bytes_per_launch"] is not None)
    achieved = top["achieved_gbs"]
    step_bytes = sum(p["alg_bytes_per_launch"] * p["launches"] for p in prof
                     if p["alg_bytes_per_launch"] is not None) / n_prof_steps
    step_bytes += sum(v for k, v in roofline_bytes(net, pop_events, pop_spikes, n_int).items()
                      if k.startswith("post_stdp"))
    step_gbs = step_bytes / (sec / n_int) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        traffic = json.load(open(tf)).get(top["kernel"])

    # cpu baseline (rank 0 only, N=1): reference CPU kernel on a bounded sample
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_sample(args)

    result = {
        "metric": METRIC, "value": world * updates_rank / sec, "unit": UNIT, "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": 1e3 * sec / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (state), f64 (event times)",
        "data": "synthetic (seeded Poisson mossy-fibre inputs, random connectivity)",
        "config": {"workload": WORKLOAD, "integration_steps_per_step": STEPS_PER_BENCH_STEP,
                   "neurons": n_model, "synapses": int(net.n_synapses), "parallelism": "replicas" if world > 1 else "single",
                   "l2": "flushed (256 MB write) between timed steps", "scale": args.scale},
        "syn_events_per_s": world * events_rank / sec,
        "spikes_per_s": world * spikes_rank / sec,
        "e2e": {"value": world * updates_rank / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d // K,
                "d2h_bytes_per_step": d2h // K},
        "roofline": {"bound": "hbm", "kernel": top["kernel"], "achieved": achieved, "peak": peak,
                     "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "alg_bytes_per_launch": top["alg_bytes_per_launch"],
                     "avg_launch_us": top["avg_us"], "steps_per_launch": top["steps_per_launch"]},
        "step_roofline": {"alg_bytes_per_integration_step": step_bytes, "achieved": step_gbs,
                          "unit": "GB/s", "frac": step_gbs / peak},
        "kernels": prof[:8],
        "gpu_launches": int(l1.value - l0.value),
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    sim.close()
    if args.sweep_networks > 0:
        result["sweep"] = run_sweep(args, rank, world)
    if args.adjoint_networks > 0:
        result["adjoint"] = run_adjoint(args, rank, world)
    if args.hh_neurons > 0:
        result["hh"] = run_hh(args, rank, world)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))


SWEEP_WORKLOAD = ("batched sweep: independent LIF networks, sizes log-uniform 500-5000, 80/20 E/I, p=0.1, "
                  "100 Poisson inputs at 10 Hz each (per-network seeds), g_leak x U[0.7,1.3], E_leak 15 mV "
                  "below threshold x U[0.7,1.3], weight scale x U[0.7,1.3] (recurrent ranges x 1000/N), "
                  "1 ms delay, RK2 dt 0.1 ms, 1 s")


def run_sweep(args, rank, world):
    """Batched-sweep leg: all networks for 1 s of simulated time in one persistent
    kernel (graph-replayed chunks, autotuned launch shape), against looping the plain
    path over a sample of the same networks one at a time; the sampled networks'
    spikes must be identical in both."""
    import torch
    from edlut_b200.configs import sweep_networks
    from edlut_b200.simulation import Simulation
    from edlut_b200.sweep import Sweep
    from edlut_b200.shard import network_cost, partition
    nsteps = args.sweep_steps
    all_specs = sweep_networks(seed=1, n_networks=args.sweep_networks, t_end=nsteps * DT)
    # the networks are independent: each rank runs its cost-balanced slice
    lo, hi = partition([network_cost(sp) for sp in all_specs], world)[rank]
    specs = all_specs[lo:hi]
    sw = Sweep.from_specs(specs, n_steps_max=nsteps)
    tune = sw.autotune(min(500, nsteps))
    stream = torch.cuda.ExternalStream(sw.stream())
    times = []
    for rep in range(2):
        sw.reset()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sw.run_async(nsteps)
        b.record(stream)
        sw.sync()
        times.append(a.elapsed_time(b) / 1e3)
    sec = statistics.mean(times)
    sec = max_over_ranks(sec, world)
    info = sw.info()
    sizes = np.array([sp["n"] for sp in specs])
    tot = torch.tensor([float(sizes.sum()), float(info["synapses"]), float(info["events"])], dtype=torch.float64,
                       device="cuda")
    if world > 1:
        torch.distributed.all_reduce(tot)
    tot_neurons, tot_syn, tot_events = (float(v) for v in tot.tolist())
    # plain path, one network at a time, on networks spread over the size range
    sample = np.argsort(sizes)[np.linspace(0, len(sizes) - 1, args.sweep_sample).astype(int)]
    plain_s, identical = 0.0, True
    for i in sample:
        net, t_in, c_in = sw.solo_description(int(i))
        sim = Simulation.from_description(net, record_capacity=8 << 20)
        sim.inject_spikes(t_in, c_in)
        sp = ctypes_stream(sim)
        st = torch.cuda.ExternalStream(sp)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        sim.run_async(nsteps)
        b.record(st)
        sim.sync()
        plain_s += a.elapsed_time(b) / 1e3
        s1, c1 = sim.spikes()
        s2, c2 = sw.spikes(int(i))
        identical &= bool(len(s1) == len(s2) and np.array_equal(s1, s2) and np.array_equal(c1, c2))
        sim.close()
    plain_nps = len(sample) / plain_s
    nps = len(all_specs) / sec
    out = {"workload": SWEEP_WORKLOAD, "networks": len(all_specs), "steps": nsteps,
           "neurons": int(tot_neurons), "synapses": int(tot_syn),
           "ms": 1e3 * sec, "networks_per_s": nps,
           "neuron_updates_per_s": tot_neurons * nsteps / sec,
           "syn_events_per_s": tot_events / sec,
           "scaling": "strong (the networks split across ranks)" if world > 1 else "single",
           "plain_loop_networks_per_s": plain_nps, "speedup_vs_plain_loop": nps / world / plain_nps,
           "plain_loop_sample": int(len(sample)), "identical_spikes_in_sample": identical,
           "autotune": tune, "device_gb": info["device_bytes"] / 1e9, "timing": "CUDA events, mean of 2 runs"}
    sw.close()
    return out


HH_WORKLOAD = ("stiff Hodgkin-Huxley network: HH neurons (Na/K/leak, reference default parameters), fixed in-degree "
               "100 from uniformly random sources (80/20 E/I), integer delays uniform 1-5 ms, one 200 Hz Poisson "
               "drive per neuron, BDF order 2 at dt 0.05 ms, fp32 state, 500 ms")


HH_BUCKET_LIMIT = 64


def run_hh(args, rank, world):
    """Stiff HH leg: the whole 500 ms (10,000 BDF2 steps) of the HH network after a
    short untimed warm-up, device-timed with CUDA events on the simulation stream.
    Algorithmic bytes per neuron-update: 48 B of HH state (V, m, h, n, gE, gI) plus
    96 B of BDF2 history, 8 B per delivered event and per fanned-out event."""
    import torch
    from edlut_b200.configs import hh_network
    from edlut_b200.simulation import Simulation
    dt, warm, nsteps = 5e-5, 200, args.hh_steps
    net, tin, cin = hh_network(seed=rank_seed(1, rank), n=args.hh_neurons, t_end=(warm + nsteps + 10) * dt,
                               unique_times=False)
    n = net.layers[1].n
    # about 0.5 arrivals per neuron and step: 64 bucket slots per neuron instead of
    # in-degree x 2 (an overflow would end the run with EB_ERR_OVERFLOW)
    sim = Simulation.from_description(net, record_capacity=16 << 20, bucket_limit=HH_BUCKET_LIMIT)
    sim.inject_spikes(tin, cin)
    from edlut_b200 import _lib
    L = _lib.load()
    _lib.check(L.eb_prestage(sim._h, warm + nsteps))
    sim.run(warm)
    sim.spikes()
    c0 = sim.counters()
    st = torch.cuda.ExternalStream(ctypes_stream(sim))
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    sim.run_async(nsteps)
    b.record(st)
    sim.sync()
    sec = max_over_ranks(a.elapsed_time(b) / 1e3, world)
    c1 = sim.counters()
    events = c1["events"] - c0["events"]
    spikes = c1["spikes"] - c0["spikes"]
    alg = (BYTES_PER_UNIT["HH"] + 96) * n * nsteps + EVENT_BYTES * events * 2
    peak, peak_kind = measured_peaks()
    sim.close()
    return {"workload": HH_WORKLOAD, "neurons": n * world, "synapses": int(net.n_synapses) * world,
            "steps": nsteps, "ms": 1e3 * sec, "us_per_step": 1e6 * sec / nsteps,
            "neuron_updates_per_s": world * n * nsteps / sec, "syn_events_per_s": world * events / sec,
            "spikes_per_s": world * spikes / sec, "mean_rate_hz": spikes / n / (nsteps * dt),
            "alg_bytes_per_step": alg / nsteps, "achieved_gbs": alg / sec / 1e9,
            "frac": alg / sec / 1e9 / peak, "peak": peak, "peak_source": peak_kind,
            "timing": "CUDA events around the run on the simulation stream, inputs resident"}


ADJOINT_WORKLOAD = ("adjoint fitting: LIF networks of 10k neurons (80/20 E/I, in-degree exactly 100 recurrent + 10 "
                    "from 100 Poisson inputs at 10 Hz), RK2 dt 0.1 ms, 5,000 steps, checkpoints every 100 steps; "
                    "loss = MSE of the V traces of 256 observed neurons per network against traces from hidden "
                    "ground-truth g_leak/E_leak/tau_AMPA/tau_GABA (x U[0.7,1.3]); gradients for those four "
                    "parameters per network and every weight")


def run_adjoint(args, rank, world):
    """Adjoint leg: forward (the method's own time stepping, trace of the observed
    neurons) and forward + backward (adjoint kernel, one recomputation per
    checkpoint segment) on the fitting workload, timed with CUDA events."""
    import torch
    from edlut_b200.adjoint import TraceModel
    from edlut_b200.configs import adjoint_networks, perturbed_params
    from edlut_b200.shard import network_cost, partition
    B_all, n, steps, every = args.adjoint_networks, args.adjoint_neurons, args.adjoint_steps, 100
    all_specs = adjoint_networks(seed=7, n_networks=B_all, n=n, t_end=steps * DT)
    # independent networks: each rank fits its slice of the batch
    lo, hi = partition([network_cost(sp) for sp in all_specs], world)[rank]
    specs = all_specs[lo:hi]
    B = len(specs)
    obs = np.stack([np.random.default_rng([7, i]).choice(n, 256, replace=False) for i in range(lo, hi)])
    model = TraceModel(specs, steps, obs, integrator="RK2", checkpoint_every=every)
    rng = np.random.default_rng(99)
    truth = np.array([[perturbed_params(s["params"], rng)[k] for k in ("g_leak", "e_leak", "tau_exc", "tau_inh")]
                      for s in all_specs])[lo:hi]
    w0 = model.initial_weights()
    with torch.no_grad():
        target = model(torch.tensor(truth), w0).clone()
    params = model.initial_params().requires_grad_()
    weights = w0.clone().requires_grad_()

    def fwd_only():
        with torch.no_grad():
            return model(params, weights)

    def fwd_bwd():
        params.grad = None
        weights.grad = None
        loss = ((model(params, weights) - target) ** 2).mean()
        loss.backward()
        return loss

    def timed(fn, reps=2):
        out = []
        for _ in range(reps):
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            out.append(a.elapsed_time(b) / 1e3)
        return min(out)
    fwd_only()
    fwd_bwd()
    t_f = max_over_ranks(timed(fwd_only), world)
    t_fb = max_over_ranks(timed(fwd_bwd), world)
    loss = float(fwd_bwd().detach())
    gp = params.grad.numpy()
    gw = weights.grad
    info = model.sweep.info()
    out = {"workload": ADJOINT_WORKLOAD, "networks": B_all, "networks_per_rank": B, "neurons_per_network": n,
           "steps": steps, "scaling": "strong (the batch split across ranks)" if world > 1 else "single",
           "checkpoint_every": every, "observed_per_network": 256, "weights": int(model.n_weights),
           "forward_ms": 1e3 * t_f, "forward_backward_ms": 1e3 * t_fb, "cost_ratio": t_fb / t_f,
           "backward_over_forward": (t_fb - t_f) / t_f, "loss": loss,
           "grad_params_norm": float(np.linalg.norm(gp)), "grad_w_norm": float(torch.linalg.norm(gw)),
           "neuron_updates_per_s_forward": B_all * n * steps / t_f, "device_gb": info["device_bytes"] / 1e9,
           "timing": "CUDA events around the whole call (host parameter upload, forward kernels, trace copy; "
                     "backward adds recompute + adjoint kernels), best of 2"}
    model.sweep.close()
    return out


def ctypes_stream(sim):
    import ctypes
    from edlut_b200 import _lib
    sp = ctypes.c_void_p()
    _lib.check(sim._L.eb_stream(sim._h, ctypes.byref(sp)))
    return sp.value


# ------------------------------------------------------- reference arm ----
REF_WARM_STEPS = 500       # reference run-in before its timed samples (past the start-up transient)
REF_SINGLE_SAMPLES = 2     # samples of the 1-thread reference run


def ref_binary(name="ref_bench"):
    p = os.path.join(ROOT, "oracle", "_ref", name)
    return p if os.path.exists(p) else None


class ReferenceWorkload:
    """The benchmark network written once in the reference's file formats (network,
    weights, model .cfg and input-spike files) for the reference's own CPU kernel:
    the same builder, seed and size as the GPU arm's rank 0."""

    def __init__(self, steps_needed: int, seed: int = 1, scale: float = 1.0):
        from edlut_b200.network import write_input_spikes
        net, tin, cin = build_workload(seed=seed, t_end=(steps_needed + 20) * DT, scale=scale)
        self.n_model = sum(l.n for l in net.layers if l.model != "InputSpikeNeuronModel")
        self.dir = tempfile.mkdtemp(prefix="edlut_ref_")
        self.netf, self.wf = (os.path.basename(p) for p in net.write_files(self.dir))
        write_input_spikes(os.path.join(self.dir, "inputs.cfg"), tin, cin)
        self.scale = scale

    def time(self, threads: int, warm: int, sample_steps: int, samples: int) -> dict:
        """Run oracle/_ref/ref_bench (the reference's Simulation with `threads` OpenMP
        queues): set-up and `warm` steps untimed, then `samples` timed samples of
        `sample_steps` integration steps each, wall clock per sample."""
        cmd = [ref_binary(), self.netf, self.wf, "inputs.cfg", str(threads), repr(float(np.float32(DT))),
               str(warm), str(sample_steps), str(samples)]
        r = subprocess.run(cmd, cwd=self.dir, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("ref_bench failed: " + r.stdout[-500:] + r.stderr[-500:])
        out = json.loads(r.stdout.strip().splitlines()[-1])
        out["value"] = [self.n_model * sample_steps / s for s in out["sample_s"]]
        out["events_per_s"] = [e / s for e, s in zip(out["events"], out["sample_s"])]
        return out

    def close(self):
        shutil.rmtree(self.dir, ignore_errors=True)


def ref_sample_text(threads: int, n_model: int, warm: int, per: int, n: int, scale: float) -> str:
    size = "full size" if scale == 1.0 else "scale %g" % scale
    return ("reference EDLUT CPU kernel (its Simulation class, %d OpenMP queue%s), the benchmark's cerebellar "
            "network at %s (%d model neurons, same seed and inputs), %d samples of %d integration steps after "
            "%d untimed steps; set-up excluded" % (threads, "s" if threads > 1 else "", size, n_model, n, per,
                                                     warm, ))


def cpu_reference_sample(args, samples: int = 3):
    """CPU baseline of the GPU arm: the reference's own CPU kernel on the same
    workload, all host cores and one thread, a few samples each.  Falls back to the
    C oracle port (single thread, 1/10 scale) when the reference build is absent."""
    per = args.cpu_sample_steps
    cores = os.cpu_count() or 1
    if ref_binary() is None:
        from oracle import oracle as O
        net, tin, cin = build_workload(seed=1, t_end=(per + 20) * DT, scale=0.1)
        n_model = sum(l.n for l in net.layers if l.model != "InputSpikeNeuronModel")
        t0 = time.perf_counter()
        r = O.run(net, tin, cin, per)
        el = time.perf_counter() - t0
        return {"value": n_model * per / el, "unit": UNIT, "cores": 1, "kind": "port",
                "sample": "C oracle port, cerebellar layer at 1/10 scale, %d steps" % per,
                "syn_events_per_s": r["n_events"] / el, "same_config": False}
    wl = ReferenceWorkload(REF_WARM_STEPS + per * samples, scale=args.scale)
    try:
        allc = wl.time(cores, REF_WARM_STEPS, per, samples)
        one = wl.time(1, REF_WARM_STEPS, per, REF_SINGLE_SAMPLES)
    finally:
        wl.close()
    return {"value": statistics.mean(allc["value"]), "unit": UNIT, "cores": allc["queues"], "kind": "reference",
            "sample": ref_sample_text(allc["queues"], wl.n_model, REF_WARM_STEPS, per, samples, args.scale),
            "syn_events_per_s": statistics.mean(allc["events_per_s"]), "same_config": args.scale == 1.0,
            "setup_s": allc["setup_s"],
            "single_thread": {"value": statistics.mean(one["value"]), "cores": 1,
                              "syn_events_per_s": statistics.mean(one["events_per_s"]),
                              "sample": ref_sample_text(1, wl.n_model, REF_WARM_STEPS, per, REF_SINGLE_SAMPLES,
                                                        args.scale)}}


def run_reference(args):
    """Reference arm: the reference's own CPU kernel (oracle/_ref/ref_bench, built
    from the reference sources) on the GPU arm's workload, every host core; each
    benchmark step is one sample of --cpu-sample-steps integration steps of the one
    loaded network (set-up once, untimed).  A 1-thread run is reported beside it."""
    rank, world, _ = env_rank()
    if rank != 0:
        return
    W, K = args.warmup, args.steps
    per = args.cpu_sample_steps
    cores = os.cpu_count() or 1
    if ref_binary() is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU kernel not built (oracle/_ref/ref_bench)"}))
        return
    wl = ReferenceWorkload(REF_WARM_STEPS + per * (W + K), scale=args.scale)
    try:
        allc = wl.time(cores, REF_WARM_STEPS + per * W, per, K)
        one = wl.time(1, REF_WARM_STEPS, per, REF_SINGLE_SAMPLES)
    finally:
        wl.close()
    v = statistics.mean(allc["value"])
    ev = statistics.mean(allc["events_per_s"])
    sample = ref_sample_text(allc["queues"], wl.n_model, REF_WARM_STEPS + per * W, per, K, args.scale)
    result = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": K,
              "warmup": W, "ms_per_step": 1e3 * statistics.mean(allc["sample_s"]), "higher_is_better": True,
              "scaling": "weak", "vs_baseline": None, "dtype": "f32 (state), f64 (event times)",
              "data": "synthetic (seeded Poisson mossy-fibre inputs, random connectivity)",
              "config": {"workload": WORKLOAD, "integration_steps_per_step": per, "neurons": wl.n_model,
                         "scale": args.scale, "sample": sample},
              "syn_events_per_s": ev,
              "cpu_baseline": {"value": v, "unit": UNIT, "cores": allc["queues"], "kind": "reference",
                               "sample": sample},
              "single_thread": {"value": statistics.mean(one["value"]), "cores": 1,
                                "syn_events_per_s": statistics.mean(one["events_per_s"]),
                                "sample": ref_sample_text(1, wl.n_model, REF_WARM_STEPS, per, REF_SINGLE_SAMPLES,
                                                          args.scale)},
              "setup_s": allc["setup_s"], "host_cores": cores,
              "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(result))


def run_for_profiler(args):
    """Build the workload and run it with no timing, for an external profiler:
    `args.prof_warm` warm-up steps then `args.prof_run` steps, graph replay of
    `args.graph_steps` steps (1: one launch per kernel, so each is listed)."""
    from edlut_b200.simulation import Simulation
    n = args.prof_warm + args.prof_run
    net, tin, cin = build_workload(1, (n + 20) * DT, args.scale)
    sim = Simulation.from_description(net, graph_steps=args.graph_steps)
    sim.inject_spikes(tin, cin)
    sim.run(args.prof_warm)
    t0 = time.perf_counter()
    sim.run(args.prof_run)
    el = time.perf_counter() - t0
    print(json.dumps({"profile_run_steps": args.prof_run, "wall_ms_per_step": 1e3 * el / max(1, args.prof_run),
                      "counters": sim.counters()}))
    sim.close()


def run_for_profiler_hh(args):
    """The stiff HH network (``--hh-neurons``) run untimed for an external profiler:
    `args.prof_warm` warm-up steps then `args.prof_run` steps on the default path."""
    from edlut_b200.configs import hh_network
    from edlut_b200.simulation import Simulation
    n = args.prof_warm + args.prof_run
    net, tin, cin = hh_network(seed=1, n=args.hh_neurons, t_end=(n + 10) * 5e-5, unique_times=False)
    sim = Simulation.from_description(net, bucket_limit=HH_BUCKET_LIMIT)
    sim.inject_spikes(tin, cin)
    sim.run(args.prof_warm)
    sim.run(args.prof_run)
    print(json.dumps({"profile_run_steps": args.prof_run, "counters": sim.counters()}))
    sim.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--cpu-sample-steps", type=int, default=50,
                    help="integration steps per reference CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-run", action="store_true", help="untimed run for an external profiler")
    ap.add_argument("--prof-warm", type=int, default=300)
    ap.add_argument("--prof-run", type=int, default=50)
    ap.add_argument("--graph-steps", type=int, default=1)
    ap.add_argument("--sweep-networks", type=int, default=4096, help="batched-sweep leg (0: skip)")
    ap.add_argument("--sweep-steps", type=int, default=10000)
    ap.add_argument("--sweep-sample", type=int, default=6, help="networks also run alone on the plain path")
    ap.add_argument("--profile-sweep", action="store_true", help="untimed sweep run for an external profiler")
    ap.add_argument("--adjoint-networks", type=int, default=64, help="adjoint leg (0: skip)")
    ap.add_argument("--hh-neurons", type=int, default=100000, help="stiff HH leg (0: skip)")
    ap.add_argument("--hh-steps", type=int, default=10000)
    ap.add_argument("--profile-hh", action="store_true", help="untimed stiff-HH run for an external profiler")
    ap.add_argument("--adjoint-neurons", type=int, default=10000)
    ap.add_argument("--adjoint-steps", type=int, default=5000)
    args = ap.parse_args()
    if args.profile_run:
        run_for_profiler(args)
        return
    if args.profile_hh:
        run_for_profiler_hh(args)
        return
    if args.profile_sweep:
        from edlut_b200.configs import sweep_networks
        from edlut_b200.sweep import Sweep
        specs = sweep_networks(seed=1, n_networks=args.sweep_networks, t_end=args.sweep_steps * DT)
        sw = Sweep.from_specs(specs, n_steps_max=args.sweep_steps)
        sw.configure(block=512, steps_per_launch=args.sweep_steps)
        sw.run(args.sweep_steps)
        print(json.dumps({"profile_sweep_networks": len(specs), "steps": args.sweep_steps, **sw.info()}))
        sw.close()
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
