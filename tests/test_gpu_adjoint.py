"""GPU tests of the adjoint (eb_sweep_adjoint and the torch.autograd.Function over
it): on small LIF networks the gradients with respect to g_leak, E_leak, tau_exc,
tau_inh and the weights match FP64 central finite differences of the C oracle and
the FP64 reference adjoint within 1e-3 relative; they are deterministic, do not
depend on the checkpoint interval beyond rounding, and flow through autograd."""
import numpy as np
import pytest

from edlut_b200.configs import ADJOINT_PARAMS, adjoint_networks
from edlut_b200.network import Layer, NetworkDescription

pytestmark = pytest.mark.gpu

N, N_IN, STEPS = 60, 20, 200


def specs_for(seed, n_networks=3, rate_hz=50.0, w_in_max=2.0):
    return adjoint_networks(seed=seed, n_networks=n_networks, n=N, indeg=10, n_inputs=N_IN, in_indeg=4,
                            rate_hz=rate_hz, t_end=STEPS * 1e-4, w_exc_max=0.5, w_inh_max=2.0, w_in_max=w_in_max)


def description(spec, integrator):
    """The network of one spec for the oracle, synapses in spec (caller) order."""
    net = NetworkDescription()
    net.add_layer(Layer(N, "LIFTimeDrivenModel", dict(spec["params"]), integrator=integrator, dt=1e-4, name="lif"))
    net.add_layer(Layer(N_IN, "InputSpikeNeuronModel", output=0))
    stype = ((spec["src"] >= spec["n_exc"]) & (spec["src"] < N)).astype(np.int32)
    net.add_synapses(spec["src"].astype(np.int64), spec["tgt"].astype(np.int64), 1e-3, stype, spec["w"], spec["w"], -1)
    return net, spec["times"], spec["cells"].astype(np.int64) + N


def run_gpu(specs, integrator, obs, targets, every=50):
    from edlut_b200.sweep import Sweep
    sw = Sweep.from_specs(specs, n_steps_max=STEPS, integrator=integrator, max_rate_hz=2000.0)
    sw.set_observed(np.broadcast_to(obs, (len(specs), len(obs))))
    sw.set_checkpoints(every)
    sw.reset()
    sw.run(STEPS)
    tr = sw.trace(STEPS)
    g = (2.0 * (tr - targets) / tr[0].size).astype(np.float32)
    gp, gw = sw.adjoint(g)
    return sw, tr, gp, gw


def split_w(specs, gw):
    out, o = [], 0
    for s in specs:
        out.append(gw[o:o + len(s["w"])])
        o += len(s["w"])
    return out


# "bursting": strong fast drive, so the observed neurons spike many times inside the
# loss window and E_leak's gradient is carried mostly by the resets V <- E_leak
@pytest.mark.parametrize("integrator,drive", [("RK2", "moderate"), ("Euler", "moderate"), ("RK4", "moderate"),
                                              ("RK2", "bursting")])
def test_gpu_adjoint_matches_fp64_adjoint_and_finite_differences(oracle, integrator, drive):
    from oracle import adjoint_ref as A
    specs = specs_for(21) if drive == "moderate" else specs_for(25, rate_hz=300.0, w_in_max=4.0)
    obs = np.arange(0, N, 4)
    rng = np.random.default_rng(1)
    targets = (-65.0 + 5.0 * rng.standard_normal((len(specs), STEPS, len(obs)))).astype(np.float32)
    sw, tr, gp, gw = run_gpu(specs, integrator, obs, targets)
    gws = split_w(specs, gw)
    for b, spec in enumerate(specs):
        net, t, c = description(spec, integrator)
        traj = A.trajectory_fp64(net, t, c, STEPS)
        # same spike train in the float32 forward and the FP64 oracle
        st, ce = sw.spikes(b)
        o_st, o_ce = traj["spikes"]
        keep = o_ce < N
        assert sorted(zip(st.tolist(), ce.tolist())) == sorted(zip(o_st[keep].tolist(), o_ce[keep].tolist()))
        V = traj["V_post"][:, obs]
        ref_p, muE, muI = A.adjoint_fp64(traj, obs, 2.0 * (V - targets[b]) / V.size)
        ref_w = A.weight_grad(net, traj, muE, muI)
        np.testing.assert_allclose(gp[b], ref_p, rtol=1e-3, atol=1e-6 * np.abs(ref_p).max())
        err = np.linalg.norm(gws[b] - ref_w) / np.linalg.norm(ref_w)
        assert err < 1e-3, err
        tg = targets[b]

        def loss(trace):
            return float(np.mean((trace[:, obs] - tg) ** 2))
        for j, name in enumerate(ADJOINT_PARAMS):
            fd, same = A.finite_difference(net, t, c, STEPS, loss, ("param", name))
            assert same
            assert abs(gp[b, j] - fd) <= 1e-3 * abs(fd) + 1e-9, (b, name, gp[b, j], fd)
        if drive == "bursting":
            assert len(st) >= 5 * len(obs), len(st)  # many resets inside the window
        # the largest weight gradients whose perturbation keeps the spike train
        # (a changed train makes the finite difference a jump, not a derivative):
        # at least two of them must be checked per network
        checked = 0
        for q in np.argsort(-np.abs(ref_w))[:24]:
            fd, same = A.finite_difference(net, t, c, STEPS, loss, ("weight", int(q)))
            if not same:
                continue
            assert abs(gws[b][q] - fd) <= 1e-3 * abs(fd) + 1e-6, (b, q, gws[b][q], fd)
            checked += 1
            if checked == 4:
                break
        assert checked >= 2, (b, checked)
    sw.close()


def test_gpu_adjoint_is_deterministic_and_checkpoint_independent():
    specs = specs_for(22)
    obs = np.arange(0, N, 3)
    rng = np.random.default_rng(2)
    targets = (-60.0 + 3.0 * rng.standard_normal((len(specs), STEPS, len(obs)))).astype(np.float32)
    _, tr1, gp1, gw1 = run_gpu(specs, "RK2", obs, targets, every=50)
    _, tr2, gp2, gw2 = run_gpu(specs, "RK2", obs, targets, every=50)
    assert gp1.tobytes() == gp2.tobytes() and gw1.tobytes() == gw2.tobytes()
    _, tr3, gp3, gw3 = run_gpu(specs, "RK2", obs, targets, every=200)
    _, tr4, gp4, gw4 = run_gpu(specs, "RK2", obs, targets, every=7)
    np.testing.assert_array_equal(tr1, tr3)
    for gp, gw in ((gp3, gw3), (gp4, gw4)):
        np.testing.assert_allclose(gp, gp1, rtol=1e-5, atol=1e-9)
        np.testing.assert_allclose(gw, gw1, rtol=1e-4, atol=1e-6 * np.abs(gw1).max())


def test_traces_equal_the_plain_path():
    """The forward under the adjoint is the unchanged method: observed traces equal
    the plain path's recorded states of the same network."""
    from edlut_b200.simulation import Simulation
    specs = specs_for(23, n_networks=2)
    obs = np.arange(0, N, 5)
    targets = np.zeros((2, STEPS, len(obs)), np.float32)
    sw, tr, _, _ = run_gpu(specs, "RK2", obs, targets)
    for b, spec in enumerate(specs):
        net, t, c = description(spec, "RK2")
        sim = Simulation.from_description(net)
        sim.set_trace(0, N, STEPS)
        sim.inject_spikes(t, c)
        sim.run(STEPS)
        ref = sim.get_trace()[:, obs, 0]
        sim.close()
        np.testing.assert_array_equal(tr[b], ref)
    sw.close()


def test_autograd_function_gives_the_adjoint_gradients():
    import torch
    from edlut_b200.adjoint import TraceModel
    specs = specs_for(24, n_networks=2)
    obs = np.arange(0, N, 4)
    model = TraceModel(specs, STEPS, obs, integrator="RK2", checkpoint_every=40)
    params = model.initial_params().requires_grad_()
    weights = model.initial_weights().requires_grad_()
    target = torch.full((2, STEPS, len(obs)), -62.0, device="cuda")
    tr = model(params, weights)
    loss = ((tr - target) ** 2).mean()
    loss.backward()
    # the same gradients from the library call directly
    g = (2.0 * (tr.detach() - target) / tr.numel()).contiguous()
    model.sweep.reset()
    model.sweep.run(STEPS)
    gp, gw = model.sweep.adjoint(g.cpu().numpy())
    np.testing.assert_allclose(params.grad.numpy(), gp, rtol=1e-6)
    np.testing.assert_allclose(weights.grad.cpu().numpy(), gw, rtol=1e-6, atol=1e-12)
