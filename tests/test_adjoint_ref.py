"""CPU checks of the FP64 reference adjoint (the yardstick of the GPU adjoint): on
small LIF networks its gradients with respect to g_leak, E_leak, tau_exc, tau_inh
and synaptic weights match FP64 central finite differences of the C oracle."""
import numpy as np
import pytest

from edlut_b200.configs import adjoint_networks, perturbed_params
from edlut_b200.network import Layer, NetworkDescription


def small_network(seed, integrator, n=60, n_in=20, nsteps=200):
    # weights in the range where the explicit integrators stay stable at C_m = 2
    spec = adjoint_networks(seed=seed, n_networks=1, n=n, indeg=10, n_inputs=n_in, in_indeg=4,
                            rate_hz=50.0, t_end=nsteps * 1e-4, w_exc_max=0.5, w_inh_max=2.0, w_in_max=2.0)[0]
    net = NetworkDescription()
    net.add_layer(Layer(n, "LIFTimeDrivenModel", dict(spec["params"]), integrator=integrator, dt=1e-4, name="lif"))
    net.add_layer(Layer(n_in, "InputSpikeNeuronModel", output=0))
    stype = ((spec["src"] >= spec["n_exc"]) & (spec["src"] < n)).astype(np.int32)
    net.add_synapses(spec["src"].astype(np.int64), spec["tgt"].astype(np.int64), 1e-3, stype, spec["w"], spec["w"], -1)
    return net, spec["times"], spec["cells"].astype(np.int64) + n


@pytest.mark.parametrize("integrator", ["Euler", "RK2", "RK4"])
def test_fp64_adjoint_matches_finite_differences(integrator):
    from oracle import adjoint_ref as A
    nsteps = 200
    net, t, c = small_network(3, integrator, nsteps=nsteps)
    obs = np.arange(0, 60, 4)
    rng = np.random.default_rng(0)
    target = -65.0 + 5.0 * rng.standard_normal((nsteps, len(obs)))

    def loss(tr):
        return float(np.mean((tr[:, obs] - target) ** 2))

    traj = A.trajectory_fp64(net, t, c, nsteps)
    assert traj["spiked"].sum() > 5
    assert np.abs(traj["V_post"]).max() < 200.0
    V = traj["V_post"][:, obs]
    g_trace = 2.0 * (V - target) / V.size
    grad, muE, muI = A.adjoint_fp64(traj, obs, g_trace)
    gw = A.weight_grad(net, traj, muE, muI)
    for j, name in enumerate(["g_leak", "e_leak", "tau_exc", "tau_inh"]):
        fd, same = A.finite_difference(net, t, c, nsteps, loss, ("param", name))
        assert same, name
        assert abs(grad[j] - fd) <= 1e-5 * abs(fd) + 1e-12, (name, grad[j], fd)
    # weights with arrivals and the largest gradients, plus some at random
    cand = np.argsort(-np.abs(gw))[:6].tolist() + rng.choice(len(gw), 6, replace=False).tolist()
    for q in cand:
        fd, same = A.finite_difference(net, t, c, nsteps, loss, ("weight", int(q)))
        if not same:
            continue
        assert abs(gw[q] - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(gw).max()), (q, gw[q], fd)
