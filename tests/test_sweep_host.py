"""CPU tests of the sweep workload generator (no GPU)."""
import numpy as np

from edlut_b200.configs import LIF_C1, sweep_networks


def test_sweep_specs_are_seeded_and_in_range():
    a = sweep_networks(seed=3, n_networks=64, t_end=0.1)
    b = sweep_networks(seed=3, n_networks=64, t_end=0.1)
    sizes = np.array([s["n"] for s in a])
    assert sizes.min() >= 500 and sizes.max() <= 5000
    for x, y in zip(a, b):
        assert x["n"] == y["n"] and x["params"] == y["params"]
        np.testing.assert_array_equal(x["times"], y["times"])
        np.testing.assert_array_equal(x["cells"], y["cells"])
    gl = np.array([s["params"]["g_leak"] for s in a]) / LIF_C1["g_leak"]
    assert gl.min() >= 0.7 - 1e-6 and gl.max() <= 1.3 + 1e-6
    el = np.array([s["params"]["e_leak"] for s in a])
    assert (el < LIF_C1["v_thr"]).all()  # every network stays below threshold at rest
    # per-network Poisson seeds: input trains differ between networks
    assert not np.array_equal(a[0]["times"], a[1]["times"])
    for s in a:
        assert (np.diff(s["times"]) >= 0).all()
        assert s["cells"].min() >= 0 and s["cells"].max() < s["n_in"]


def test_sweep_weight_scaling_keeps_mean_drive():
    a = sweep_networks(seed=4, n_networks=32, t_end=0.05)
    for s in a:
        # recurrent range x size / 1000 is the weight-scale factor, the same as the input range's
        k = s["w_exc_max"] * s["n"] / 1000.0 / 0.5
        assert abs(k - s["w_in_max"] / 0.5) < 1e-4 * max(1.0, k)
