"""Host logic of the batched encoder's bulk read-back: splitting the packed result per image."""
import numpy as np

from roger_b200 import _lib as L
from roger_b200.batch import split_packed


def _naive(first, descs, data):
    out = []
    for i in range(len(first) - 1):
        a, b = first[i], first[i + 1]
        d = descs[a:b].copy()
        base = int(d["offset"][0]) if b > a else 0
        end = int(d["offset"][-1] + max(int(d["length"][-1]), 0)) if b > a else 0
        d["offset"] -= base
        out.append((d, data[base:end]))
    return out


def test_split_matches_the_per_image_loop():
    rng = np.random.default_rng(5)
    counts = [3, 0, 7, 1, 0, 12, 5]
    n = sum(counts)
    d = np.zeros(n, L.CB_DESC)
    d["length"] = rng.integers(0, 50, n)
    d["length"][4] = 0
    d["offset"] = np.concatenate([[0], np.cumsum(d["length"])[:-1]])
    data = rng.integers(0, 256, int(d["length"].sum()) + 3).astype(np.uint8)
    first = np.concatenate([[0], np.cumsum(counts)])
    got, want = split_packed(first, d, data), _naive(first, d, data)
    assert len(got) == len(want) == len(counts)
    for (gd, gb), (wd, wb) in zip(got, want):
        assert np.array_equal(gd, wd) and np.array_equal(np.asarray(gb), np.asarray(wb))
