"""eb_fold_arrivals_noalloc: the fold of synaptic arrivals for callers that cannot
allocate device memory while they run (a real-time closed-loop controller, or an
engine that owns all device memory).  It must give exactly what the allocating
eb_fold_arrivals gives, on two calls in a row (the shared scratch keeps the first
call's contents and must be cleared), and refuse batches beyond its fixed size.
Kept in a file of its own that pytest collects last."""
import ctypes

import numpy as np
import pytest

from tests.test_gpu_fold import device_fold, make_batch

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_fold_twice():
    from edlut_b200 import _lib
    L = _lib.load()
    for seed, n, m in ((11, 120000, 4000), (12, 3000, 97)):  # second call smaller than the first
        target, stype, weight, time, g0 = make_batch(seed, n, m)
        want = device_fold(L.eb_fold_arrivals, target, stype, weight, time, g0)
        got = device_fold(L.eb_fold_arrivals_noalloc, target, stype, weight, time, g0)
        for a, b in zip(got, want):
            np.testing.assert_array_equal(a, b)


def test_noalloc_rejects_batches_beyond_its_scratch():
    import torch
    from edlut_b200 import _lib
    L = _lib.load()
    n = (1 << 18) + 1
    t = torch.zeros(n, dtype=torch.int32, device="cuda")
    s = torch.zeros(n, dtype=torch.int8, device="cuda")
    w = torch.zeros(n, dtype=torch.float32, device="cuda")
    g = torch.zeros(8, dtype=torch.float32, device="cuda")
    rc = L.eb_fold_arrivals_noalloc(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), n, t.data_ptr(),
                                    s.data_ptr(), w.data_ptr(), None, 8, g.data_ptr(), g.data_ptr(),
                                    g.data_ptr())
    assert rc == -1
    assert b"262144" in L.eb_last_error()
