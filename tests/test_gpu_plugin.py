"""The reference engine with this library's neuron-model plugins: the reference's
own Simulation (events, spike delivery, STDP, outputs), built from its sources by
edlut_b200/plugin/Makefile, loads unchanged network files naming
LIFTimeDrivenModel_GPU / AdExTimeDrivenModel_GPU / HHTimeDrivenModel_GPU, and the
factory variant binds those names to the plugins, which hold the neurons on the
GPU through the C ABI (eb_fold_arrivals of the delivered weights, one eb_run step
per UpdateState).  The result must be the reference CPU models' result, the
golden fixture, bit for bit: spikes, monitored state traces, final STDP weights,
synapse order and event counts."""
import os
import tempfile

import numpy as np
import pytest

from tests._cases import build_case, load_golden, perm_digest, spike_pairs

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "edlut_b200", "plugin", "_build", "ref_harness_b200")


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="plugin engine not built (make -C edlut_b200/plugin REF=...)")
@pytest.mark.parametrize("name", ["lif_rk2_stdp", "adex_rk4_stdp", "hh_bdf2_stdp", "lif_bdf3_stdp", "cereb_small_rk4"])
def test_reference_engine_with_plugins_matches_fixture(name):
    from oracle import oracle as O
    from tests.golden.make_golden import step_of_times
    net, t, c, nsteps, trace = build_case(name)
    for layer in net.layers:
        if layer.model not in ("InputSpikeNeuronModel", "PoissonGeneratorDeviceVector"):
            layer.model = layer.model + "_GPU"   # the reference's GPU model names
            layer.log = 1                        # monitored: the plugin mirrors its state to the engine
    g = load_golden(name)
    with tempfile.TemporaryDirectory() as wd:
        R = O.run_reference(net, t, c, nsteps, wd, trace=trace, exe=HARNESS)
    dt = next(l.dt for l in net.layers if l.model != "InputSpikeNeuronModel")
    steps = step_of_times(R["spike_time"], dt, nsteps)
    np.testing.assert_array_equal(spike_pairs(steps, R["spike_cell"]), spike_pairs(g["spike_step"], g["spike_cell"]))
    nd = g["trace"].shape[2]
    np.testing.assert_array_equal(R["trace"][:, :, :nd], g["trace"])
    if "w_final" in g:
        np.testing.assert_array_equal(R["w_final"], g["w_final"])
    assert perm_digest(R["syn"]["orig"]) == str(g["perm_sha256"])
    assert R["counts"] == [int(x) for x in g["counts"]]
