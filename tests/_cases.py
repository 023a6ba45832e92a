"""Shared helpers of the parity tests: golden cases and comparisons."""
import os

import numpy as np

from tests.golden.make_golden import CASES, build_case, perm_digest  # noqa: F401

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def spike_pairs(steps, cells):
    steps = np.asarray(steps, np.int64)
    cells = np.asarray(cells, np.int64)
    o = np.lexsort((cells, steps))
    return np.stack([steps[o], cells[o]], 1)


def spike_match_fraction(a, b):
    """Fraction of spikes of `a` with an identical (step, cell) in `b`, and the
    fraction within one step, as the parity criterion counts them."""
    sa = set(map(tuple, a.tolist()))
    sb = set(map(tuple, b.tolist()))
    if not sa:
        return 1.0, 1.0
    same = len(sa & sb) / len(sa)
    near = sum(1 for (s, c) in sa if (s, c) in sb or (s - 1, c) in sb or (s + 1, c) in sb) / len(sa)
    return same, near


def load_golden_text(name, ext):
    """Bytes of the reference's own output file kept for a case (ext ".of": output
    spikes, ".sf": saved weights)."""
    import gzip
    with gzip.open(os.path.join(GOLDEN, name + ext + ".gz"), "rb") as f:
        return f.read()


def weights_file_text(w):
    """Network::SaveWeights' format (src/spike/Network.cpp:1165-1202): runs of equal
    consecutive weights, one "%i %g" line per run."""
    w = np.asarray(w, np.float32)
    lines = []
    i = 0
    while i < len(w):
        j = i + 1
        while j < len(w) and w[j] == w[i]:
            j += 1
        lines.append("%i %g\n" % (j - i, float(w[i])))
        i = j
    return "".join(lines).encode()
