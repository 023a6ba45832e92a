"""GPU tests of the batched parameter sweep (eb_sweep_*): every network's spike
train and final state equal a run of the same network alone on the plain path
(and, for a small sweep, the CPU oracle); results do not depend on the launch
configuration the autotuner picks, on chunking, or on resets."""
import numpy as np
import pytest

from edlut_b200.configs import sweep_networks
from tests._cases import spike_pairs

pytestmark = pytest.mark.gpu


def make_sweep(specs, nsteps, **kw):
    from edlut_b200.sweep import Sweep
    kw.setdefault("max_rate_hz", 1500.0)  # small networks here fire far above the sweep's rates
    return Sweep.from_specs(specs, n_steps_max=nsteps, **kw)


def solo(sw, i, nsteps):
    from edlut_b200.simulation import Simulation
    net, t, c = sw.solo_description(i)
    sim = Simulation.from_description(net, record_capacity=4_000_000)
    sim.inject_spikes(t, c)
    sim.run(nsteps)
    st, ce = sim.spikes()
    v = sim.get_state(0, int(sw.sizes[i]), 0)
    sim.close()
    return st, ce, v


def assert_network_matches(sw, i, nsteps):
    st, ce, v = solo(sw, i, nsteps)
    s2, c2 = sw.spikes(i)
    assert len(st) == len(s2), (i, len(st), len(s2))
    np.testing.assert_array_equal(st, s2)
    np.testing.assert_array_equal(ce, c2)
    np.testing.assert_array_equal(v, sw.state(i, 0))
    return len(st)


@pytest.mark.parametrize("integrator", ["RK2", "Euler", "RK4"])
def test_every_network_matches_its_solo_run(integrator):
    nsteps = 2500
    specs = sweep_networks(seed=5, n_networks=8, n_min=150, n_max=1200, t_end=nsteps * 1e-4)
    sw = make_sweep(specs, nsteps, integrator=integrator)
    sw.configure(block=128, steps_per_launch=700)  # several chunks, one graph
    sw.run(nsteps)
    total = sum(assert_network_matches(sw, i, nsteps) for i in range(len(specs)))
    assert total > 0
    assert sw.spike_counts().sum() == total
    sw.close()


@pytest.mark.parametrize("dt,delay", [(1e-4, 0.35e-3), (1e-4, 2.0e-3), (5e-5, 1e-3), (2e-4, 1e-4)])
def test_delay_grids(dt, delay):
    nsteps = int(round(0.2 / dt))
    specs = sweep_networks(seed=7, n_networks=4, n_min=200, n_max=800, t_end=nsteps * dt, dt=dt)
    sw = make_sweep(specs, nsteps, dt=dt, delay=delay)
    sw.run(nsteps)
    for i in range(len(specs)):
        assert_network_matches(sw, i, nsteps)
    sw.close()


def test_synchronous_bursts_take_several_delivery_passes():
    # E_leak above threshold: the spike test does not look at refractoriness, so every
    # neuron fires in every step (more sources in one step than one delivery pass lists)
    nsteps = 600
    specs = sweep_networks(seed=9, n_networks=3, n_min=1400, n_max=2000, t_end=nsteps * 1e-4)
    for s in specs:
        s["params"]["e_leak"] = -45.0
    sw = make_sweep(specs, nsteps, max_rate_hz=10000.0)
    sw.run(nsteps)
    for i in range(len(specs)):
        st, _ = sw.spikes(i)
        assert np.bincount(st).max() > 512
        assert_network_matches(sw, i, nsteps)
    sw.close()


def test_small_sweep_matches_the_oracle(oracle):
    nsteps = 1500
    specs = sweep_networks(seed=11, n_networks=3, n_min=100, n_max=160, t_end=nsteps * 1e-4)
    sw = make_sweep(specs, nsteps)
    sw.run(nsteps)
    for i in range(len(specs)):
        net, t, c = sw.solo_description(i)
        r = oracle.run(net, t, c, nsteps)
        np.testing.assert_array_equal(spike_pairs(r["spike_step"], r["spike_cell"]),
                                      spike_pairs(*sw.spikes(i)))
    sw.close()


def test_launch_configurations_chunking_and_reset_agree():
    nsteps = 1200
    specs = sweep_networks(seed=13, n_networks=24, n_min=300, n_max=3000, t_end=nsteps * 1e-4)
    sw = make_sweep(specs, nsteps)
    sw.configure(block=512, steps_per_launch=nsteps)
    sw.run(nsteps)
    ref = [sw.spikes(i) for i in range(len(specs))]
    v_ref = [sw.state(i) for i in range(len(specs))]
    for block, spl, chunks in [(128, 100, [1200]), (256, 333, [1, 399, 800]), (1024, 50, [600, 600])]:
        sw.reset()
        sw.configure(block=block, steps_per_launch=spl)
        for n in chunks:
            sw.run(n)
        for i in range(len(specs)):
            s, c = sw.spikes(i)
            np.testing.assert_array_equal(s, ref[i][0])
            np.testing.assert_array_equal(c, ref[i][1])
            np.testing.assert_array_equal(sw.state(i), v_ref[i])
    cfg = sw.autotune(200)
    assert cfg["block"] in (128, 256, 512, 1024) and cfg["steps_per_launch"] > 0 and cfg["trial_ms"] > 0
    sw.run(nsteps)
    for i in range(len(specs)):
        np.testing.assert_array_equal(sw.spikes(i)[1], ref[i][1])
    sw.close()


def test_errors_leave_the_sweep_usable():
    from edlut_b200._lib import EdlutError
    nsteps = 300
    specs = sweep_networks(seed=15, n_networks=2, n_min=100, n_max=200, t_end=nsteps * 1e-4)
    sw = make_sweep(specs, nsteps)
    with pytest.raises(EdlutError):
        sw.run(nsteps + 1)
    with pytest.raises(EdlutError):
        sw.configure(block=96)
    sw.run(nsteps)
    assert_network_matches(sw, 0, nsteps)
    sw.close()
