"""The reference's Python interface (PySimulation_API, Kernel/python/
simulation_wrapper.pyx) over this library: network construction from the
reference's calls and dictionary keys, and the errors for what the path does not
cover (host logic, no GPU)."""
import numpy as np
import pytest


def build_api(log=False):
    import edlut_b200.api as pyedlut
    sim = pyedlut.PySimulation_API()
    inp = sim.AddNeuronLayer(num_neurons=3, model_name="InputSpikeNeuronModel", param_dict={},
                             log_activity=False, output_activity=False)
    im = pyedlut.PyModelDescription(model_name="RK2", params_dict={"step": 0.0001})
    out = sim.AddNeuronLayer(num_neurons=2, model_name="LIFTimeDrivenModel",
                             param_dict={"v_thr": -50.0, "e_leak": -65.0, "g_leak": 0.2, "c_m": 2.0,
                                         "tau_ref": 1.0, "int_meth": im},
                             log_activity=log, output_activity=True)
    rule = sim.AddLearningRule("STDP", {"max_LTP": 0.016, "tau_LTP": 0.010, "max_LTD": 0.033, "tau_LTD": 0.005})
    syn = sim.AddSynapticLayer([inp[0], inp[1], inp[2], out[0]], [out[0], out[1], out[1], out[1]],
                               {"weight": [6.0, 5.0, 5.0, 4.0], "max_weight": 10.0, "type": [0, 0, 1, 0],
                                "delay": 0.001, "wchange": [rule, -1, -1, rule], "trigger_wchange": -1})
    return sim, inp, out, rule, syn


def test_layers_rules_and_synapses_follow_the_reference_calls():
    sim, inp, out, rule, syn = build_api()
    assert inp == [0, 1, 2] and out == [3, 4] and rule == 0 and syn == [0, 1, 2, 3]
    net = sim._net
    assert [l.model for l in net.layers] == ["InputSpikeNeuronModel", "LIFTimeDrivenModel"]
    lif = net.layers[1]
    assert lif.integrator == "RK2" and lif.dt == pytest.approx(1e-4) and lif.output == 1
    from edlut_b200.network import MODEL_DEFAULTS
    assert lif.full_params()["v_thr"] == -50.0
    assert lif.full_params()["tau_exc"] == MODEL_DEFAULTS["LIFTimeDrivenModel"]["tau_exc"]  # a default
    assert net.rules == [("STDP", [0.016, 0.010, 0.033, 0.005])]
    np.testing.assert_array_equal(net.src, [0, 1, 2, 3])
    np.testing.assert_array_equal(net.tgt, [3, 4, 4, 4])
    np.testing.assert_array_equal(net.stype, [0, 0, 1, 0])
    np.testing.assert_array_equal(net.wchange, [0, -1, -1, 0])
    np.testing.assert_array_equal(net.weight, np.float32([6, 5, 5, 4]))
    np.testing.assert_array_equal(net.max_weight, np.float32([10] * 4))
    np.testing.assert_array_equal(net.delay, np.float32([0.001] * 4))


def test_catalogue_and_defaults():
    import edlut_b200.api as pyedlut
    sim = pyedlut.PySimulation_API()
    assert "AdExTimeDrivenModel_GPU" in sim.GetAvailableNeuronModels()
    assert sim.GetAvailableIntegrationMethods() == ["Euler", "RK2", "RK4", "BDF"]
    assert sim.GetIntegrationMethodDefParams("BDF")["bdf_order"] == 2
    assert sim.GetLearningRuleDefParams("STDP") == {"max_LTP": 0.010, "tau_LTP": 0.100, "max_LTD": 0.020,
                                                    "tau_LTD": 0.100}
    d = sim.GetNeuronModelDefParams("HHTimeDrivenModel")
    assert d["g_na"] == 20000.0 and d["int_meth"].model_name == "Euler"


def test_what_the_path_does_not_cover_raises():
    import edlut_b200.api as pyedlut
    sim = pyedlut.PySimulation_API()
    with pytest.raises(NotImplementedError):
        sim.AddNeuronLayer(1, "IzhikevichTimeDrivenModel", {})
    with pytest.raises(NotImplementedError):
        sim.AddLearningRule("AdditiveKernel", {})
    with pytest.raises(NotImplementedError):
        sim.AddNeuronLayer(1, "LIFTimeDrivenModel",
                           {"int_meth": pyedlut.PyModelDescription("Bifixed_Euler", {"step": 1e-4})})
    with pytest.raises(ValueError):
        sim.AddNeuronLayer(1, "LIFTimeDrivenModel", {"not_a_parameter": 1.0})
    sim.AddNeuronLayer(2, "InputSpikeNeuronModel", {})
    with pytest.raises(NotImplementedError):
        sim.AddSynapticLayer([0], [1], {"trigger_wchange": 0})
    with pytest.raises(ValueError):
        sim.AddSynapticLayer([0, 1], [1], {})
    with pytest.raises(NotImplementedError):
        sim.AddExternalCurrentActivity([0.1], [0], [1.0])
    with pytest.raises(RuntimeError):
        sim.RunSimulation(0.01)


def test_monitor_drivers_register_before_initialize(tmp_path):
    """AddFileOutputMonitorDriver creates its file; one state file per simulation;
    only layers added with log_activity (and not input layers) are monitored."""
    sim, inp, out, rule, syn = build_api(log=True)
    f1, f2, f3 = (str(tmp_path / n) for n in ("s.txt", "p.txt", "q.txt"))
    sim.AddFileOutputMonitorDriver(f1, True)
    sim.AddFileOutputMonitorDriver(f2, False)
    assert open(f1).read() == "" and open(f2).read() == ""
    with pytest.raises(NotImplementedError):
        sim.AddFileOutputMonitorDriver(f3, True)
    assert sim._log_pop == [False, True]
    assert [l.log for l in sim._net.layers] == [0, 1]
