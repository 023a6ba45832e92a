"""The arrival-count coverage network reaches every regime of the block-per-neuron
update (checked on the oracle's spike train, no GPU)."""
import numpy as np


def test_wide_fanin_network_reaches_every_arrival_regime(oracle):
    from edlut_b200.configs import wide_fanin_network
    net, t, c = wide_fanin_network()
    o = oracle.run(net, t, c, 400, trace=(0, 0, 0))
    starts = np.cumsum([0] + [l.n for l in net.layers])
    src, tgt, d = np.asarray(net.src), np.asarray(net.tgt), np.asarray(net.delay)
    relay = (src >= starts[1]) & (src < starts[2]) & (tgt == starts[2])
    step_of = {}
    for j, cell in zip(o["spike_step"], o["spike_cell"]):
        if starts[1] <= cell < starts[2]:
            step_of.setdefault(int(cell), []).append(int(j))
    counts = {}
    for s_, dd in zip(src[relay], d[relay]):
        for j in step_of.get(int(s_), []):
            k = j + int(round(float(dd) / 1e-4))
            counts[k] = counts.get(k, 0) + 1
    v = np.array(list(counts.values()))
    assert (v > 1024).any()
    assert ((v > 256) & (v <= 1024)).any()
    assert ((v > 128) & (v <= 256)).any()
    assert ((v > 16) & (v <= 128)).any()
    # the targets fire (deferred post-synaptic STDP has spikes to apply)
    assert ((o["spike_cell"] >= starts[2]) & (o["spike_cell"] < starts[3])).sum() > 10
