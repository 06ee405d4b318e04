"""Host logic of the pipelined batched encoder: the split of a batch into consecutive groups."""
import numpy as np
import pytest

from roger_b200.batch import PipelinedBatchEncoder


@pytest.mark.parametrize("n,parts", [(1, 1), (1, 4), (5, 2), (14, 3), (40, 4), (3, 8)])
def test_groups_cover_the_batch_in_order(n, parts):
    rng = np.random.default_rng(n * 10 + parts)
    descs = [dict(w=int(rng.integers(16, 2000)), h=int(rng.integers(16, 2000)), ncomp=int(rng.choice([1, 3])))
             for _ in range(n)]
    g = PipelinedBatchEncoder.split_groups(descs, parts)
    assert g[0][0] == 0 and g[-1][1] == n
    assert all(a < b for a, b in g)
    assert all(g[k][1] == g[k + 1][0] for k in range(len(g) - 1))
    assert 1 <= len(g) <= min(parts, n)


def test_equal_images_split_evenly():
    descs = [dict(w=512, h=512, ncomp=3)] * 8
    assert PipelinedBatchEncoder.split_groups(descs, 2) == [(0, 4), (4, 8)]
    assert PipelinedBatchEncoder.split_groups(descs, 4) == [(0, 2), (2, 4), (4, 6), (6, 8)]
