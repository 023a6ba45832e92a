"""GPU tests of the C-ABI behaviour around the hot path: graph replay vs plain
launches, chunked runs, snapshot/restore, the reference-format file readers,
error paths that leave the context usable, determinism, and size-independent
properties of a benchmark-size run."""
import os
import subprocess

import numpy as np
import pytest

from tests._cases import build_case, spike_pairs

pytestmark = pytest.mark.gpu


def make_sim(net, **kw):
    from edlut_b200.simulation import Simulation
    return Simulation.from_description(net, **kw)


def run_case(name, chunks=None, **kw):
    net, t, c, nsteps, trace = build_case(name)
    sim = make_sim(net, **kw)
    sim.inject_spikes(t, c)
    for n in (chunks or [nsteps]):
        sim.run(n)
    st, ce = sim.spikes()
    w = sim.weights()
    sim.close()
    return spike_pairs(st, ce), w


def test_graph_and_plain_launches_agree():
    a, wa = run_case("adex_rk4_stdp", graph_steps=64, persistent=False)
    b, wb = run_case("adex_rk4_stdp", graph_steps=1, persistent=False)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(wa, wb)


@pytest.mark.parametrize("name", ["cereb_small_rk4", "hh_small_bdf2", "lif_coarse_dt", "adex_dense_fanin"])
def test_persistent_kernel_and_graphs_agree(name):
    a, wa = run_case(name, persistent=True)
    b, wb = run_case(name, persistent=False)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(wa, wb)


def test_chunked_runs_agree():
    a, wa = run_case("lif_bdf2_stdp")
    b, wb = run_case("lif_bdf2_stdp", chunks=[1, 63, 64, 500, 372, 1000])
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(wa, wb)


def test_runs_are_deterministic():
    a, wa = run_case("cereb_small_rk4")
    b, wb = run_case("cereb_small_rk4")
    np.testing.assert_array_equal(a, b)
    assert wa.tobytes() == wb.tobytes()


def test_snapshot_restore_replays_identically():
    net, t, c, nsteps, _ = build_case("hh_bdf2_stdp")
    sim = make_sim(net)
    sim.inject_spikes(t, c)
    sim.run(700)
    sim.spikes()
    sim.snapshot(0)
    sim.run(600)
    s1 = spike_pairs(*sim.spikes())
    w1 = sim.weights()
    sim.restore(0)
    sim.run(600)
    s2 = spike_pairs(*sim.spikes())
    w2 = sim.weights()
    sim.close()
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(w1, w2)


def test_inputs_injected_after_restore_join_in_time_order():
    """After a restore, inputs injected for the new timeline may precede inputs that
    were staged for the abandoned one: they are merged in time order, so the run
    equals one that had every input from the start."""
    net, t, c, nsteps, _ = build_case("lif_rk2_stdp")
    K, M = 600, 1400
    sim = make_sim(net)
    t_k = sim.step_time(K)
    late = (np.arange(len(t)) % 2 == 1) & (t >= t_k)
    sim.inject_spikes(t, c)
    sim.run(M)
    ref = spike_pairs(*sim.spikes())
    w_ref = sim.weights()
    sim.close()
    sim = make_sim(net)
    sim.inject_spikes(t[~late], c[~late])
    sim.run(K)
    sim.snapshot(0)
    sim.run(M - K)  # stages the early inputs beyond step K
    sim.restore(0)
    sim.inject_spikes(t[late], c[late])
    sim.run(M - K)
    got = spike_pairs(*sim.spikes())
    counters = sim.counters()
    w = sim.weights()
    sim.close()
    np.testing.assert_array_equal(got[got[:, 0] > K], ref[ref[:, 0] > K])
    np.testing.assert_array_equal(w, w_ref)
    assert counters["steps"] == M


@pytest.mark.parametrize("case", ["lif_rk2_stdp", "poisson_lif_rk2_stdp"])
def test_reference_files_load_identically(tmp_path, case):
    """eb_load_network_files / eb_load_input_file read the reference's own text
    formats (network, weights, model .cfg -- Poisson generator .cfg included --,
    input spikes) into the same network."""
    from edlut_b200.network import write_input_spikes
    from edlut_b200.simulation import Simulation
    net, t, c, nsteps, _ = build_case(case)
    netf, wf = net.write_files(str(tmp_path))
    inp = os.path.join(str(tmp_path), "inputs.cfg")
    write_input_spikes(inp, t, c)
    cwd = os.getcwd()
    os.chdir(str(tmp_path))
    try:
        sim = Simulation.from_files(os.path.basename(netf), os.path.basename(wf))
        sim.n_synapses = net.n_synapses
        sim.load_input_file("inputs.cfg")
        sim.run(nsteps)
        a = spike_pairs(*sim.spikes())
        wa = sim.weights()
        sim.close()
    finally:
        os.chdir(cwd)
    b, wb = run_case(case)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(wa, wb)


def test_random_weights_follow_reference_lcg(tmp_path, oracle):
    """A negative weight in the weights file draws uniform [0, max_weight] weights
    from the reference's LCG (seed 1), in file order."""
    from edlut_b200.simulation import Simulation
    net, t, c, nsteps, _ = build_case("lif_euler_stdp")
    netf, wf = net.write_files(str(tmp_path))
    with open(wf, "w") as f:
        f.write("0 -1\n")  # all synapses random
    cwd = os.getcwd()
    os.chdir(str(tmp_path))
    try:
        sim = Simulation.from_files(os.path.basename(netf), os.path.basename(wf))
        sim.n_synapses = net.n_synapses
        w = sim.weights()
        sim.close()
    finally:
        os.chdir(cwd)
    # restate the LCG here: next = (next*1103515245 + 12345) & 0x7fffffff, first state 1
    nxt = 1
    exp = np.zeros(net.n_synapses, np.float32)
    for i in range(net.n_synapses):
        nxt = (nxt * 1103515245 + 12345) & 0x7FFFFFFF
        exp[i] = np.float32(np.float32(nxt) / np.float32(2147483647)) * net.max_weight[i]
    np.testing.assert_array_equal(w, exp)


def test_bucket_overflow_is_reported_and_context_survives():
    from edlut_b200._lib import EdlutError
    net, t, c, nsteps, _ = build_case("adex_dense_fanin")
    sim = make_sim(net, bucket_limit=1)
    sim.inject_spikes(t, c)
    with pytest.raises(EdlutError) as e:
        sim.run(500)
    assert e.value.code == -4
    # the context stays usable: state, counters and snapshots still work
    v = sim.get_state(net.layers[0].n, 10)
    assert np.all(np.isfinite(v))
    assert sim.counters()["steps"] == 500
    sim.snapshot(0)
    sim.restore(0)
    sim.close()


def test_persistent_barrier_timeout_is_reported_and_context_recovers():
    """The persistent kernel's grid-barrier waits are bounded: with block 0 made to
    withhold its arrivals and a short wait limit, every wait runs out, the run
    returns an error (no hang, no fault), and after a restore the context runs on
    to the same result as an undisturbed run."""
    from edlut_b200._lib import EdlutError
    net, t, c, nsteps, _ = build_case("cereb_small_rk4")
    ref, w_ref = run_case("cereb_small_rk4", persistent=True)
    sim = make_sim(net, persistent=True)
    sim.inject_spikes(t, c)
    sim.snapshot(0)
    L = sim._L
    assert L.eb_set_barrier_wait(sim._h, 1 << 12, 1) == 0
    with pytest.raises(EdlutError) as e:
        sim.run(64)
    assert e.value.code == -2 and "timed out" in str(e.value)
    assert L.eb_set_barrier_wait(sim._h, 1 << 24, 0) == 0
    sim.restore(0)
    sim.run(nsteps)
    got = spike_pairs(*sim.spikes())
    w = sim.weights()
    sim.close()
    np.testing.assert_array_equal(got, ref)
    np.testing.assert_array_equal(w, w_ref)


def test_bad_calls_return_errors():
    from edlut_b200._lib import EdlutError
    from edlut_b200.simulation import Simulation
    sim = Simulation()
    with pytest.raises(EdlutError):
        sim.run(10)  # not finalized
    from edlut_b200.network import MODEL_DEFAULTS
    sim.add_population("LIFTimeDrivenModel", 10, "Euler", 1, 1e-4, MODEL_DEFAULTS["LIFTimeDrivenModel"])
    sim.finalize()
    with pytest.raises(EdlutError):  # populations cannot be added after finalize
        sim.add_population("LIFTimeDrivenModel", 10, "Euler", 1, 1e-4, MODEL_DEFAULTS["LIFTimeDrivenModel"])
    from edlut_b200.simulation import Simulation as S2
    s2 = S2()
    assert s2._L.eb_add_population(s2._h, 1, 10, 9, 1, 1e-4, None, 0, None) == -6  # unknown integrator
    assert s2._L.eb_add_population(s2._h, 1, 0, 0, 1, 1e-4, None, 0, None) == -1   # empty population
    s2.close()
    sim.close()


def test_input_before_current_time_rejected():
    from edlut_b200._lib import EdlutError
    net, t, c, nsteps, _ = build_case("lif_euler_stdp")
    sim = make_sim(net)
    sim.run(100)
    with pytest.raises(EdlutError):
        sim.inject_spikes([0.001], [0])
    sim.close()


def test_empty_connectivity_matches_oracle(oracle):
    from edlut_b200.network import Layer, NetworkDescription
    from edlut_b200.configs import LIF_C1
    net = NetworkDescription()
    net.add_layer(Layer(100, "LIFTimeDrivenModel", dict(LIF_C1, e_leak=-40.0), integrator="RK4"))
    sim = make_sim(net)
    sim.set_trace(0, 4, 50)
    sim.run(200)
    tr = sim.get_trace()
    st, ce = sim.spikes()
    o = oracle.run(net, np.zeros(0, np.float32), np.zeros(0, np.int64), 200, trace=(50, 0, 4),
                   spike_cap=100 * 200 + 16)
    np.testing.assert_array_equal(spike_pairs(st, ce), spike_pairs(o["spike_step"], o["spike_cell"]))
    np.testing.assert_array_equal(tr, o["trace"].astype(np.float32))
    sim.close()


@pytest.mark.slow
def test_benchmark_size_properties():
    """Full cerebellar-layer network (11M synapses): size-independent checks --
    spikes recorded for both layers, plastic weights within [0, max], no overflow,
    and two runs from the same seed give byte-identical weights."""
    import bench
    net, t, c = bench.build_workload(seed=1, t_end=0.06)
    outs = []
    for _ in range(2):
        sim = make_sim(net)
        sim.inject_spikes(t, c)
        sim.run(500)
        st, ce = sim.spikes()
        w = sim.weights()
        outs.append((st, ce, w))
        sim.close()
    st, ce, w = outs[0]
    n_mf, n_g = net.layers[0].n, net.layers[1].n
    assert ((ce >= n_mf) & (ce < n_mf + n_g)).sum() > 0
    plastic = net.wchange >= 0
    assert np.all(w[plastic] >= 0) and np.all(w[plastic] <= net.max_weight[plastic])
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    assert outs[0][2].tobytes() == outs[1][2].tobytes()


@pytest.mark.slow
def test_hh_benchmark_size_properties():
    """Full stiff Hodgkin-Huxley network (100k HH neurons, BDF2 at 0.05 ms, 10.1M
    synapses with 1-5 ms delays, a 200 Hz drive per neuron): captured graphs of
    8-step windows give the same spikes and membrane potentials as one launch per
    step, the network spikes, and a second run is identical."""
    from edlut_b200.configs import hh_network
    nsteps = 600
    net, t, c = hh_network(seed=1, t_end=(nsteps + 10) * 5e-5, unique_times=False)
    first, n = net.layers[0].n, net.layers[1].n
    outs = []
    for graph_steps in (0, 1, 0):
        sim = make_sim(net, graph_steps=graph_steps)
        sim.inject_spikes(t, c)
        sim.run(nsteps)
        st, ce = sim.spikes()
        outs.append((spike_pairs(st, ce), sim.get_state(first, n, 0)))
        sim.close()
    assert len(outs[0][0]) > 1000
    for o in outs[1:]:
        np.testing.assert_array_equal(o[0], outs[0][0])
        assert o[1].tobytes() == outs[0][1].tobytes()


def test_spike_drains_are_sorted_on_the_device():
    """eb_get_spikes sorts the recording buffer on the device (a radix sort over
    the varying bits of step and neuron).  With E_leak above threshold every
    neuron fires in every step, so each drain is the full (step, neuron) grid of
    the steps since the previous drain: millions of records over many tiles and
    digit passes, uneven step ranges, and a one-step drain."""
    from edlut_b200.network import Layer, NetworkDescription
    from edlut_b200.configs import LIF_C1
    n = 70_000
    net = NetworkDescription()
    net.add_layer(Layer(n, "LIFTimeDrivenModel", dict(LIF_C1, e_leak=-40.0), integrator="Euler"))
    sim = make_sim(net, record_capacity=16 << 20)
    done = 0
    for run in (37, 200, 1, 8):
        sim.run(run)
        st, ce = sim.spikes()
        steps = np.arange(done + 1, done + run + 1, dtype=np.int64)
        np.testing.assert_array_equal(st, np.repeat(steps, n))
        np.testing.assert_array_equal(ce, np.tile(np.arange(n, dtype=np.int64), run))
        done += run
    st, ce = sim.spikes()
    assert len(st) == 0
    sim.close()


def test_output_files_match_the_reference_files(tmp_path):
    """eb_write_spikes and eb_save_weights write the reference's -of spike file and
    -sf weights file byte for byte (the reference's own files, kept with the
    golden fixtures); a population whose output flag is off writes nothing."""
    from tests._cases import load_golden_text
    from tests.golden.make_golden import FILE_CASES
    for name in FILE_CASES:
        net, t, c, nsteps, trace = build_case(name)
        sim = make_sim(net)
        sim.inject_spikes(t, c)
        sim.run(nsteps // 2)
        of = str(tmp_path / (name + ".of"))
        sim.write_spikes(of)
        sim.run(nsteps - nsteps // 2)
        sim.write_spikes(of, append=True)
        sf = str(tmp_path / (name + ".sf"))
        sim.save_weights(sf)
        assert open(of, "rb").read() == load_golden_text(name, ".of")
        assert open(sf, "rb").read() == load_golden_text(name, ".sf")
        model = next(q for q, l in enumerate(net.layers) if l.model != "InputSpikeNeuronModel")
        sim.set_output(model, False)
        sim.run(200)
        sim.write_spikes(of)
        assert open(of, "rb").read() == b""
        sim.close()
