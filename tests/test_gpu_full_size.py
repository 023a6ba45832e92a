"""GPU parity at the benchmark sizes: the default graph path against the
reference's own outputs for the first steps of the full-size workloads.

* c2_full_rk4: the cerebellar layer (250k AdEx granule cells fed by 5k mossy
  fibres, 200 LIF Purkinje cells x 50k plastic granule synapses under STDP),
  RK4 at 0.1 ms, 500 steps;
* c3_full_bdf2: the stiff network (100k HH neurons, in-degree 100, delays
  1-5 ms, one 200 Hz drive each), BDF2 at 0.05 ms, 200 steps, unique input
  times.

Every spike (step, cell), the V traces of 8 cells, the synapse order, the event
count and the final weights (SHA-256 of all 11M, plus every 997th value) must
equal the reference's bit for bit."""
import hashlib

import numpy as np
import pytest

from tests._cases import build_case, load_golden, perm_digest, spike_match_fraction, spike_pairs

pytestmark = pytest.mark.gpu

# Arrival slots per neuron and step for the stiff network (about 0.5 expected; an
# overflow ends the run with EB_ERR_OVERFLOW rather than a wrong result).
BUCKET_LIMIT = {"c3_full_bdf2": 64}


@pytest.mark.parametrize("name", ["c2_full_rk4", "c3_full_bdf2"])
def test_full_size_matches_reference(name):
    from edlut_b200.simulation import Simulation
    net, t, c, nsteps, trace = build_case(name)
    g = load_golden(name)
    sim = Simulation.from_description(net, bucket_limit=BUCKET_LIMIT.get(name, 0))
    sim.inject_spikes(t, c)
    ts, tf, tn = trace
    sim.set_trace(tf, tn, ts)
    sim.run(nsteps)
    st, ce = sim.spikes()
    tr = sim.get_trace()
    w = sim.weights()
    counters = sim.counters()
    perm = sim.sorted_perm
    sim.close()
    got = spike_pairs(st, ce)
    ref = spike_pairs(g["spike_step"], g["spike_cell"])
    same, near = spike_match_fraction(ref, got)
    assert same >= 0.999 and near == 1.0, (same, near)
    np.testing.assert_array_equal(got, ref)
    np.testing.assert_array_equal(tr[:, :, :1], g["trace"])
    assert counters["events"] == int(g["counts"][1])
    assert counters["spikes"] == int(g["counts"][0])
    assert perm_digest(perm) == str(g["perm_sha256"])
    np.testing.assert_array_equal(w[::997], g["w_sample"])
    assert hashlib.sha256(np.ascontiguousarray(w, np.float32).tobytes()).hexdigest() == str(g["w_sha256"])
