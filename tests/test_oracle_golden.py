"""The CPU oracle reproduces the reference's own outputs (golden fixtures made by
running the reference EDLUT CPU kernel, tests/golden/make_golden.py) bit for bit:
spike steps and cells, state traces, final STDP weights, synapse order, counts."""
import numpy as np
import pytest

from tests._cases import CASES, build_case, load_golden, perm_digest, spike_pairs


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_fixture(oracle, name):
    net, t, c, nsteps, trace = build_case(name)
    g = load_golden(name)
    r = oracle.run(net, t, c, nsteps, trace=trace)
    np.testing.assert_array_equal(spike_pairs(r["spike_step"], r["spike_cell"]),
                                  spike_pairs(g["spike_step"], g["spike_cell"]))
    nd = g["trace"].shape[2]
    np.testing.assert_array_equal(r["trace"][:, :, :nd].astype(np.float32), g["trace"])
    if "w_final" in g:
        np.testing.assert_array_equal(r["w_final"].astype(np.float32), g["w_final"])
    assert perm_digest(r["sorted_perm"]) == str(g["perm_sha256"])
    assert r["n_events"] == int(g["counts"][1])
    assert len(r["spike_step"]) == int(g["counts"][0])


def test_fp64_oracle_is_close_to_float_mirror(oracle):
    """The FP64 restatement (exact exp) stays close to the float32 mirror over the
    first 100 ms of the recurrent LIF workload; this is the error yardstick."""
    net, t, c, nsteps, trace = build_case("c1_lif_euler")
    a = oracle.run(net, t, c, 1000, trace=(1000, 100, 16))
    b = oracle.run(net, t, c, 1000, fp64=True, trace=(1000, 100, 16))
    rms = float(np.sqrt(np.mean((a["trace"][:, :, 0] - b["trace"][:, :, 0]) ** 2)))
    assert rms < 1e-2, rms


def test_delay_rounding_matches_reference_rule(oracle):
    # RoundPropagationDelay: floor(d*1e4 + 5e-5)*1e-4, minimum 1e-4 (Network.cpp:1311-1317)
    assert oracle.round_delay(0.001) == 10 * 0.0001
    assert oracle.round_delay(0.00149) == 14 * 0.0001
    assert oracle.round_delay(0.00005) == 0.0001
    assert oracle.round_delay(0.0) == 0.0001
    assert oracle.round_delay(0.005) == 50 * 0.0001


def test_reference_output_files_agree_with_fixture():
    """The reference's own -of spike file and -sf weights file kept for a case hold
    the same spikes and weights as its binary fixture: the spike lines are the
    update times of the fixture's steps (printed with %f) and its neurons in
    (step, neuron) order; the weights file is the fixture's final weights in the
    SaveWeights run-length format."""
    from oracle.oracle import step_times
    from tests._cases import load_golden_text, weights_file_text
    from tests.golden.make_golden import FILE_CASES
    for name in FILE_CASES:
        g = load_golden(name)
        net, t, c, nsteps, trace = build_case(name)
        dt = next(l.dt for l in net.layers if l.model != "InputSpikeNeuronModel")
        ts = step_times(dt, nsteps)
        pairs = spike_pairs(g["spike_step"], g["spike_cell"])
        expect = "".join("%f\t%d\n" % (ts[s], cell) for s, cell in pairs.tolist()).encode()
        assert load_golden_text(name, ".of") == expect
        assert load_golden_text(name, ".sf") == weights_file_text(g["w_final"])


def test_fixture_dynamics_are_finite():
    """Every fixture's traces stay finite except the cases kept to pin overflow
    (their inf / NaN propagation and reset must match too)."""
    from tests.golden.make_golden import OVERFLOW_CASES
    for name in CASES:
        tr = load_golden(name)["trace"]
        if name in OVERFLOW_CASES:
            assert not np.isfinite(tr).all(), name
        else:
            assert np.isfinite(tr).all(), name


def test_reference_monitor_files_agree_with_fixture():
    """The reference's own -logp state-monitor file kept for a case agrees with its
    binary fixture: after each step, a line per neuron that spiked then a line per
    monitored neuron, at the step's update time, whose membrane potentials are the
    fixture's trace; between the steps one line per delivered synaptic event."""
    from oracle.oracle import step_times
    from tests._cases import load_golden_text
    from tests.golden.make_golden import LOG_CASES
    for name in LOG_CASES:
        g = load_golden(name)
        net, t, c, nsteps, (tsteps, tfirst, tn) = build_case(name)
        dt = next(l.dt for l in net.layers if l.model != "InputSpikeNeuronModel")
        ts = step_times(dt, nsteps)
        mon, first = [], 0
        for l in net.layers:
            if l.model != "InputSpikeNeuronModel":
                mon.extend(range(first, first + l.n))
            first += l.n
        rows = [ln.split("\t") for ln in load_golden_text(name, ".logp").decode().splitlines()]
        spikes = {}
        for s, cell in spike_pairs(g["spike_step"], g["spike_cell"]).tolist():
            spikes.setdefault(s, []).append(cell)
        i, deliveries = 0, 0
        for k in range(1, nsteps + 1):
            tk = "%f" % float(np.float32(ts[k]))
            want = spikes.get(k, []) + mon
            while [int(r[1]) for r in rows[i:i + len(want)]] != want or any(r[0] != tk for r in rows[i:i + len(want)]):
                assert int(rows[i][1]) in mon
                assert float(ts[k - 1]) - 1e-6 <= float(rows[i][0]) <= float(ts[k]) + 1e-6
                deliveries += 1
                i += 1
            block = {int(r[1]): r for r in rows[i + len(want) - len(mon):i + len(want)]}
            for r in rows[i:i + len(want) - len(mon)]:
                assert r == block[int(r[1])]
            if k <= tsteps:
                v = ["%1.12f" % float(x) for x in g["trace"][k - 1, :, 0]]
                assert [block[cell][2] for cell in range(tfirst, tfirst + tn)] == v
            i += len(want)
        deliveries += len(rows) - i
        assert deliveries == int(g["counts"][1])
