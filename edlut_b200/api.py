"""The reference's Python interface, ``pyedlut.PySimulation_API``
(Kernel/python/simulation_wrapper.pyx:14-710, over Simulation_API.cpp), for the
models on this path, running on the B200 kernels through the C ABI.

A script written against pyedlut for time-driven LIF / AdEx / HH layers, input
spike neurons, device Poisson generators and STDP runs unchanged after
``import edlut_b200.api as pyedlut``: the same method names, argument meanings,
dictionary keys ('int_meth', 'weight', 'max_weight', 'type', 'delay', 'wchange',
'trigger_wchange'), returned index lists and spike-activity tuples.  What the
path does not cover (other neuron models, current inputs, trigger learning rules,
weight-file drivers) raises ``NotImplementedError`` naming the call, where the
reference would run it on the CPU.

As in the reference, layers, learning rules and synaptic layers are only
registered until ``Initialize``; spikes injected before ``Initialize`` are kept
and delivered after it.  ``RunSimulation(t)`` advances every update step whose
time is at most t: at equal times the reference's update event outranks its stop
event (include/simulation/Event.h:37).
"""
from __future__ import annotations

from typing import Dict, List, Sequence

import numpy as np

from .network import INPUT_MODELS, INTEGRATORS, MODEL_DEFAULTS, MODEL_PARAM_ORDER, Layer, NetworkDescription

__all__ = ["PyModelDescription", "PySimulation_API"]

_TIME_DRIVEN = ("LIFTimeDrivenModel", "AdExTimeDrivenModel", "HHTimeDrivenModel")
_MODELS = INPUT_MODELS + ("PoissonGeneratorDeviceVector",) + _TIME_DRIVEN + tuple(m + "_GPU" for m in _TIME_DRIVEN)
# STDPWeightChange::GetDefaultParameters (src/learning_rules/STDPWeightChange.cpp:182-189)
_STDP_DEFAULTS = {"max_LTP": 0.010, "tau_LTP": 0.100, "max_LTD": 0.020, "tau_LTD": 0.100}


class PyModelDescription:
    """A model name with its parameters (simulation_wrapper.pyx:14-19); used for
    the 'int_meth' entry of a neuron layer: model_name 'Euler', 'RK2', 'RK4' or
    'BDF', params_dict {'step': seconds[, 'bdf_order': 1..6]}."""

    def __init__(self, model_name, params_dict):
        self.model_name = model_name
        self.params_dict = params_dict


def _per_synapse(value, n: int, name: str, dtype):
    a = np.asarray(value, dtype)
    if a.ndim == 0:
        return np.full(n, a, dtype)
    if len(a) != n:
        raise ValueError("AddSynapticLayer: '%s' has %d values for %d synapses" % (name, len(a), n))
    return a


class PySimulation_API:
    def __init__(self):
        self._net = NetworkDescription()
        self._sim = None
        self._seed = None
        self._pending_in: List[tuple] = []
        self._spikes_t: List[float] = []
        self._spikes_c: List[int] = []
        self._out_files: List[str] = []
        self._output_pop: List[bool] = []
        self._log_pop: List[bool] = []
        self._mon_spike_files: List[str] = []
        self._mon_state_file = None

    # ------------------------------------------------------------ catalogue --
    def GetAvailableNeuronModels(self) -> List[str]:
        return list(_MODELS)

    def GetAvailableIntegrationMethods(self) -> List[str]:
        return list(INTEGRATORS)

    def GetAvailableLearningRules(self) -> List[str]:
        return ["STDP"]

    def GetNeuronModelDefParams(self, model_name: str) -> Dict[str, object]:
        if model_name not in _MODELS:
            raise NotImplementedError("GetNeuronModelDefParams: %s is outside this path" % model_name)
        d = dict(MODEL_DEFAULTS.get(model_name, {}))
        if model_name.replace("_GPU", "") in _TIME_DRIVEN:
            d["int_meth"] = PyModelDescription("Euler", {"step": 1e-4})
        return d

    def GetIntegrationMethodDefParams(self, model_name: str) -> Dict[str, object]:
        if model_name not in INTEGRATORS:
            raise NotImplementedError("GetIntegrationMethodDefParams: %s is outside this path" % model_name)
        d = {"name": model_name, "step": 1e-4}
        if model_name == "BDF":
            d["bdf_order"] = 2  # BDFn.h:852
        return d

    def GetLearningRuleDefParams(self, model_name: str) -> Dict[str, float]:
        if model_name != "STDP":
            raise NotImplementedError("GetLearningRuleDefParams: %s is outside this path" % model_name)
        return dict(_STDP_DEFAULTS)

    # ------------------------------------------------------------- building --
    def _check_open(self, call: str) -> None:
        if self._sim is not None:
            raise RuntimeError("%s after Initialize" % call)

    def AddNeuronLayer(self, num_neurons=1, model_name="InputSpikeNeuronModel", param_dict={},
                       log_activity=False, output_activity=False) -> List[int]:
        self._check_open("AddNeuronLayer")
        if model_name not in _MODELS:
            raise NotImplementedError("AddNeuronLayer: neuron model %s is outside this path" % model_name)
        params = dict(param_dict)
        kw = {}
        if model_name.replace("_GPU", "") in _TIME_DRIVEN:
            im = params.pop("int_meth", None)
            if im is not None:
                if im.model_name not in INTEGRATORS:
                    raise NotImplementedError("AddNeuronLayer: integration method %s is outside this path"
                                              % im.model_name)
                kw = dict(integrator=im.model_name, dt=float(im.params_dict.get("step", 1e-4)),
                          bdf_order=int(im.params_dict.get("bdf_order", 2)))
            known = set(MODEL_PARAM_ORDER[model_name])
            unknown = set(params) - known
            if unknown:
                raise ValueError("AddNeuronLayer: unknown parameters for %s: %s" % (model_name, sorted(unknown)))
        elif model_name == "PoissonGeneratorDeviceVector":
            unknown = set(params) - {"frequency"}
            if unknown:
                raise ValueError("AddNeuronLayer: unknown parameters for %s: %s" % (model_name, sorted(unknown)))
        elif params:
            raise ValueError("AddNeuronLayer: %s takes no parameters" % model_name)
        r = self._net.add_layer(Layer(int(num_neurons), model_name, params, output=int(bool(output_activity)),
                                      log=int(bool(log_activity)), **kw))
        self._output_pop.append(bool(output_activity))
        self._log_pop.append(bool(log_activity) and model_name not in INPUT_MODELS)
        return list(r)

    def AddLearningRule(self, model_name: str, param_dict: Dict[str, float]) -> int:
        self._check_open("AddLearningRule")
        if model_name != "STDP":
            raise NotImplementedError("AddLearningRule: learning rule %s is outside this path" % model_name)
        p = dict(_STDP_DEFAULTS)
        p.update(param_dict)
        self._net.rules.append(("STDP", [p["max_LTP"], p["tau_LTP"], p["max_LTD"], p["tau_LTD"]]))
        return len(self._net.rules) - 1

    def AddSynapticLayer(self, source_list: Sequence[int], target_list: Sequence[int],
                         param_dict: Dict[str, object]) -> List[int]:
        self._check_open("AddSynapticLayer")
        src = np.asarray(source_list, np.int64)
        tgt = np.asarray(target_list, np.int64)
        if len(src) != len(tgt):
            raise ValueError("AddSynapticLayer: %d sources for %d targets" % (len(src), len(tgt)))
        n = len(src)
        trig = _per_synapse(param_dict.get("trigger_wchange", -1), n, "trigger_wchange", np.int32)
        if np.any(trig >= 0):
            raise NotImplementedError("AddSynapticLayer: trigger learning rules are outside this path")
        first = self._net.n_synapses
        self._net.add_synapses(src, tgt,
                               _per_synapse(param_dict.get("delay", 0.001), n, "delay", np.float32),
                               _per_synapse(param_dict.get("type", 0), n, "type", np.int32),
                               _per_synapse(param_dict.get("weight", 1.0), n, "weight", np.float32),
                               _per_synapse(param_dict.get("max_weight", 1.0), n, "max_weight", np.float32),
                               _per_synapse(param_dict.get("wchange", -1), n, "wchange", np.int32))
        return list(range(first, first + n))

    def SetRandomGeneratorSeed(self, seed: int) -> None:
        self._check_open("SetRandomGeneratorSeed")
        self._seed = int(seed)

    def SetSimulationParameters(self, params_dict) -> None:
        # num_threads / num_simulation_queues / resolution shape the reference's
        # OpenMP queues; one device context replaces them
        pass

    def AddFileOutputSpikeActivityDriver(self, file_name: str) -> None:
        self._out_files.append(str(file_name))
        with open(file_name, "w"):
            pass

    def AddFileOutputMonitorDriver(self, file_name: str, monitor_state: bool) -> None:
        """A monitor file for the layers added with log_activity
        (Simulation_API::AddFileOutputMonitorDriver, src/simulation/Simulation_API.cpp:263):
        monitor_state true writes their states in the -logp format (a line at each
        delivery into a monitored neuron and after each step, see
        ``Simulation.open_monitor``); false writes their spikes in the -of format.
        One state file per simulation."""
        self._check_open("AddFileOutputMonitorDriver")
        if monitor_state:
            if self._mon_state_file is not None:
                raise NotImplementedError("AddFileOutputMonitorDriver: one state monitor file per simulation")
            self._mon_state_file = str(file_name)
        else:
            self._mon_spike_files.append(str(file_name))
        with open(file_name, "w"):
            pass

    def Initialize(self) -> None:
        self._check_open("Initialize")
        from .simulation import Simulation
        self._sim = Simulation.from_description(self._net, random_seed=self._seed)
        for q, on in enumerate(self._output_pop):
            self._sim.set_output(q, on)
        if self._mon_state_file is not None:
            self._sim.open_monitor(self._mon_state_file)
        for t, c in self._pending_in:
            self._sim.inject_spikes(t, c)
        self._pending_in.clear()

    # -------------------------------------------------------------- running --
    def AddExternalSpikeActivity(self, event_times_list, neuron_indices_list) -> None:
        t = np.asarray(event_times_list, np.float64).astype(np.float32)
        c = np.asarray(neuron_indices_list, np.int64)
        if self._sim is None:
            self._pending_in.append((t, c))
        else:
            self._sim.inject_spikes(t, c)

    def RunSimulation(self, end_simulation_time: float) -> None:
        if self._sim is None:
            raise RuntimeError("RunSimulation before Initialize")
        k = self._sim.counters()["steps"]
        n = 0
        while self._sim.step_time(k + n + 1) <= end_simulation_time:
            n += 1
        if n:
            self._sim.run(n)
        st, ce = self._sim.spikes()
        layer = self._net.layer_of()[ce] if len(ce) else np.zeros(0, np.int64)
        if self._mon_spike_files:
            mon = np.array([self._log_pop[q] for q in layer], bool)
            lines = ["%f\t%d\n" % (self._sim.step_time(int(s)), int(c)) for s, c in zip(st[mon], ce[mon])]
            for f in self._mon_spike_files:
                with open(f, "a") as fh:
                    fh.writelines(lines)
        out = np.array([self._output_pop[q] for q in layer], bool)
        st, ce = st[out], ce[out]
        times = [self._sim.step_time(int(s)) for s in st]
        self._spikes_t.extend(times)
        self._spikes_c.extend(int(x) for x in ce)
        for f in self._out_files:
            with open(f, "a") as fh:
                fh.writelines("%f\t%d\n" % (t, c) for t, c in zip(times, ce.tolist()))

    def GetSpikeActivity(self):
        """(event times, neuron indices) of the output layers' spikes since the last
        call, in (time, neuron) order; the buffer is emptied."""
        out = (self._spikes_t, self._spikes_c)
        self._spikes_t, self._spikes_c = [], []
        return out

    def GetWeights(self) -> List[float]:
        return self._sim.weights().astype(np.float64).tolist()

    def GetSelectedWeights(self, indexes) -> List[float]:
        w = self._sim.weights()
        return [float(w[i]) for i in indexes]

    def GetCompressedWeights(self):
        """Runs of equal consecutive weights, Network::GetCompressedWeights
        (src/spike/Network.cpp:1204-1231): (run lengths, run values)."""
        w = self._sim.weights()
        n_eq, vals = [], []
        i = 0
        while i < len(w):
            j = i + 1
            while j < len(w) and w[j] == w[i]:
                j += 1
            n_eq.append(j - i)
            vals.append(float(w[i]))
            i = j
        return n_eq, vals

    def __getattr__(self, name):
        if name[:1].isupper():
            raise NotImplementedError("PySimulation_API.%s is outside this path" % name)
        raise AttributeError(name)
