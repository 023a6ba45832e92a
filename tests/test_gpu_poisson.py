"""GPU tests of the device Poisson generators (PoissonGeneratorDeviceVector): the
golden fixture from the reference is covered by test_gpu_parity; here per-neuron
rates, the random seed and snapshot/restore of the generator state, each against
the CPU oracle."""
import numpy as np
import pytest

from edlut_b200.configs import poisson_network
from edlut_b200.network import Layer, NetworkDescription
from tests._cases import spike_pairs

pytestmark = pytest.mark.gpu


def run_gpu(net, nsteps, rates=None, seed=None):
    from edlut_b200.simulation import Simulation
    sim = Simulation.from_description(net, random_seed=seed)
    if rates is not None:
        first, r = rates
        sim.set_poisson_rates(first, r)
    sim.run(nsteps)
    out = spike_pairs(*sim.spikes()), sim.weights()
    sim.close()
    return out


def test_generator_seed_matches_the_oracle(oracle):
    net, _, _ = poisson_network(seed=8, t_end=0.15)
    try:
        oracle.set_seed(12345)
        o = oracle.run(net, [], [], 1500)
    finally:
        oracle.set_seed(1)
    s, w = run_gpu(net, 1500, seed=12345)
    np.testing.assert_array_equal(s, spike_pairs(o["spike_step"], o["spike_cell"]))
    np.testing.assert_array_equal(w, o["w_final"].astype(np.float32))
    s1, _ = run_gpu(net, 1500)
    assert not np.array_equal(s, s1)  # the seed matters


def test_per_neuron_rates_match_layers_of_those_rates(oracle):
    """One generator population with rates set per neuron equals, spike for spike,
    consecutive generator layers with those rates (same seed order)."""
    def net_of(layers):
        net = NetworkDescription()
        starts = [net.add_layer(Layer(g, "PoissonGeneratorDeviceVector", dict(frequency=f), name="gen%d" % i)).start
                  for i, (g, f) in enumerate(layers)]
        lif = net.add_layer(Layer(50, "LIFTimeDrivenModel", {}, integrator="Euler", name="lif"))
        rng = np.random.default_rng(3)
        g_total = sum(g for g, _ in layers)
        m = rng.random((g_total, 50)) < 0.3
        s, t = np.nonzero(m)
        net.add_synapses(s, t + lif.start, 1e-3, 0, (rng.random(len(s)) * 3).astype(np.float32), 3.0, -1)
        return net
    one = net_of([(60, 25.0)])
    rates = np.r_[np.full(30, 25.0), np.full(30, 90.0)].astype(np.float32)
    s_gpu, _ = run_gpu(one, 2000, rates=(0, rates))
    two = net_of([(30, 25.0), (30, 90.0)])
    o = oracle.run(two, [], [], 2000)
    np.testing.assert_array_equal(s_gpu, spike_pairs(o["spike_step"], o["spike_cell"]))


def test_generator_state_survives_snapshot_restore():
    from edlut_b200.simulation import Simulation
    net, _, _ = poisson_network(seed=9, t_end=0.1)
    sim = Simulation.from_description(net)
    sim.run(300)
    sim.spikes()
    sim.snapshot(0)
    sim.run(400)
    a = spike_pairs(*sim.spikes())
    sim.restore(0)
    sim.run(400)
    b = spike_pairs(*sim.spikes())
    sim.close()
    np.testing.assert_array_equal(a, b)
    assert len(a) > 0
