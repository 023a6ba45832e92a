"""The reference's Python interface (PySimulation_API) on the GPU: a network
built with the reference's calls and run in RunSimulation slots gives the
oracle's spikes, at the reference's spike times, and the -of file driver writes
them in the reference's format."""
import numpy as np
import pytest

from tests._cases import spike_pairs

pytestmark = pytest.mark.gpu


def test_python_interface_run_matches_the_oracle(oracle, tmp_path):
    from edlut_b200.network import poisson_input_times
    from tests.test_api_host import build_api
    sim, inp, out, rule, syn = build_api()
    of = str(tmp_path / "out.dat")
    sim.AddFileOutputSpikeActivityDriver(of)
    t, c = poisson_input_times(np.random.default_rng(3), 3, 80.0, 0.3)
    sim.AddExternalSpikeActivity(t.astype(np.float64).tolist(), (c + inp[0]).tolist())
    sim.Initialize()
    times, cells = [], []
    for k in range(1, 31):  # slots of 10 ms, as the reference's python examples run
        sim.RunSimulation(0.01 * k)
        tt, cc = sim.GetSpikeActivity()
        times += tt
        cells += cc
    nsteps = sim._sim.counters()["steps"]
    assert nsteps == 3000
    r = oracle.run(sim._net, t, c + inp[0], nsteps)
    keep = np.isin(r["spike_cell"], out)
    ref = spike_pairs(r["spike_step"][keep], r["spike_cell"][keep])
    assert len(ref) > 20
    steps = [int(np.argmin(np.abs(oracle.step_times(1e-4, nsteps) - x))) for x in times]
    np.testing.assert_array_equal(spike_pairs(steps, cells), ref)
    ts = oracle.step_times(1e-4, nsteps)
    np.testing.assert_array_equal(np.asarray(times), ts[ref[:, 0]])
    assert open(of).read() == "".join("%f\t%d\n" % (ts[s], cl) for s, cl in ref.tolist())
    np.testing.assert_array_equal(np.float32(sim.GetWeights()), r["w_final"].astype(np.float32))
    n_eq, vals = sim.GetCompressedWeights()
    assert sum(n_eq) == len(syn)


def test_python_interface_monitor_drivers(oracle, tmp_path):
    """AddFileOutputMonitorDriver through RunSimulation slots: the spike monitor
    holds the monitored layer's spikes in the -of format, and the state monitor is
    the file one device run of the same network writes (the format the reference
    files pin)."""
    from edlut_b200.network import poisson_input_times
    from edlut_b200.simulation import Simulation
    from tests.test_api_host import build_api
    sim, inp, out, rule, syn = build_api(log=True)
    sf, pf = str(tmp_path / "states.txt"), str(tmp_path / "spikes.txt")
    sim.AddFileOutputMonitorDriver(sf, True)
    sim.AddFileOutputMonitorDriver(pf, False)
    t, c = poisson_input_times(np.random.default_rng(4), 3, 80.0, 0.1)
    sim.AddExternalSpikeActivity(t.astype(np.float64).tolist(), (c + inp[0]).tolist())
    sim.Initialize()
    for k in range(1, 11):
        sim.RunSimulation(0.01 * k)
    nsteps = sim._sim.counters()["steps"]
    r = oracle.run(sim._net, t, c + inp[0], nsteps)
    keep = np.isin(r["spike_cell"], out)
    ref = spike_pairs(r["spike_step"][keep], r["spike_cell"][keep])
    assert len(ref) > 5
    ts = oracle.step_times(1e-4, nsteps)
    assert open(pf).read() == "".join("%f\t%d\n" % (ts[s], cl) for s, cl in ref.tolist())
    one = Simulation.from_description(sim._net)
    one.inject_spikes(t, c + inp[0])
    f1 = str(tmp_path / "one.txt")
    one.open_monitor(f1)
    one.run(nsteps)
    one.close_monitor()
    one.close()
    sim._sim.close_monitor()
    got = open(sf).read()
    assert got == open(f1).read()
    assert got.count("\n") >= 2 * nsteps
