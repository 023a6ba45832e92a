"""GPU test of eb_fold_arrivals (the functional delivery op) against a host
restatement of the reference's per-arrival fold: per target, weights added one
by one in order of (arrival time, position), float32 sums bit for bit."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def host_fold(target, stype, weight, time, m, g0):
    g = [g0[0].copy(), g0[1].copy(), g0[2].copy()]
    order = np.lexsort((np.arange(len(target)), time))
    for i in order:
        g[stype[i]][target[i]] = np.float32(g[stype[i]][target[i]] + weight[i])
    return g


def make_batch(seed, n, m):
    rng = np.random.default_rng(seed)
    target = rng.integers(0, m, n).astype(np.int32)
    stype = rng.integers(0, 3, n).astype(np.int8)
    weight = (rng.random(n) * 2.0).astype(np.float32)
    time = np.round(rng.random(n) * 50) * 1e-5  # many exact ties
    g0 = [(rng.random(m) * 5).astype(np.float32) for _ in range(3)]
    return target, stype, weight, time, g0


def device_fold(fn, target, stype, weight, time, g0):
    import torch
    from edlut_b200 import _lib
    dev = torch.device("cuda", 0)
    t = torch.from_numpy(target).to(dev)
    s = torch.from_numpy(stype).to(dev)
    w = torch.from_numpy(weight).to(dev)
    tm = torch.from_numpy(time).to(dev)
    g = [torch.from_numpy(x.copy()).to(dev) for x in g0]
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = fn(ctypes.c_void_p(stream), len(target), t.data_ptr(), s.data_ptr(), w.data_ptr(), tm.data_ptr(),
            len(g0[0]), g[0].data_ptr(), g[1].data_ptr(), g[2].data_ptr())
    _lib.check(rc)
    torch.cuda.synchronize()
    return [x.cpu().numpy() for x in g]


# (100000, 1): every arrival on one target, the per-target sort's worst case
@pytest.mark.parametrize("n,m", [(0, 10), (1, 1), (5000, 37), (200000, 3000), (100000, 1)])
def test_fold_matches_host_order(n, m):
    from edlut_b200 import _lib
    L = _lib.load()
    target, stype, weight, time, g0 = make_batch(7, n, m)
    ref = host_fold(target, stype, weight, time, m, g0)
    got = device_fold(L.eb_fold_arrivals, target, stype, weight, time, g0)
    for a, b in zip(got, ref):
        np.testing.assert_array_equal(a, b)
