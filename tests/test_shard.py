"""Multi-GPU sharding, tested on the CPU: the LPT partition of an image set, the code-block count
it uses (against the library's own), a world-size-2 gloo run in which each rank takes its share
of the 256-image mixed set and the per-image byte counts are gathered on every rank, and a
world-size-2 gloo run of the set encoder (shard.encode_set) whose per-rank encodes are the
oracle's, so that the gathered counts are those of real codestreams."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from roger_b200 import shard, synth


def test_lpt_covers_every_item_once_and_balances():
    rng = np.random.default_rng(1)
    for n, m in [(1, 1), (7, 3), (256, 2), (256, 8), (5, 8)]:
        costs = list(rng.integers(1, 10_000, n))
        parts = shard.lpt_partition(costs, m)
        assert len(parts) == m
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(n))
        loads = [sum(costs[i] for i in p) for p in parts]
        bound = max(max(costs), sum(costs) / m)
        assert max(loads) <= 4.0 / 3.0 * bound + 1e-9
    assert shard.lpt_partition([5, 5, 5], 2) == shard.lpt_partition([5, 5, 5], 2)  # deterministic


def test_codeblock_count_matches_library():
    from roger_b200._lib import lib
    for w, h, L, cb in [(4096, 4096, 6, 64), (1000, 77, 3, 32), (65, 2048, 5, 64), (64, 64, 3, 32)]:
        assert shard.codeblocks_of(w, h, L, cb) == lib().j2k_codeblock_count(w, h, L, cb, cb)


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    descs = synth.mixed_set(256)
    mine = shard.shard(descs, rank, world)
    counts = [d["w"] * d["h"] * d["ncomp"] // 7 + d["index"] for d in (descs[i] for i in mine)]
    allc = shard.gather_counts(mine, counts, len(descs))
    if rank == 0:
        np.save(out_path, np.concatenate([allc, np.array(mine, dtype=np.int64)]))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_gloo_shard_and_gather(tmp_path):
    out = str(tmp_path / "counts.npy")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    res = np.load(out)
    descs = synth.mixed_set(256)
    allc, mine0 = res[:256], res[256:]
    expect = np.array([d["w"] * d["h"] * d["ncomp"] // 7 + d["index"] for d in descs])
    assert np.array_equal(allc, expect)
    mine1 = shard.shard(descs, 1, 2)
    assert sorted(list(mine0) + mine1) == list(range(256))
    c = [shard.image_cost(d) for d in descs]
    l0, l1 = sum(c[i] for i in mine0), sum(c[i] for i in mine1)
    assert max(l0, l1) / min(l0, l1) < 1.05


def _set_descs():
    return synth.mixed_set(48, seed=900, lo=40, hi=200)


def _oracle_share(descs, images):
    from oracle import oracle as O
    return [O.encode_image(im, d["levels"], d["cb"], d["cb"], d["kernel"] == 53) for d, im in zip(descs, images)]


def _encode_set_rank(rank, world, port, out_dir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    descs = _set_descs()
    loaded = []

    def load(i):
        loaded.append(i)
        return synth.mixed_image(descs[i])
    idx, streams, counts = shard.encode_set(descs, load, rank, world, encode_share=_oracle_share)
    assert sorted(loaded) == list(idx)  # only this rank's own images were loaded
    np.save(os.path.join(out_dir, f"r{rank}.npy"),
            np.array([np.array(idx, np.int64), counts, np.array([len(x) for x in streams], np.int64)],
                     dtype=object), allow_pickle=True)
    with open(os.path.join(out_dir, f"r{rank}.bin"), "wb") as f:
        for x in streams:
            f.write(x)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_set_encoder_gathers_real_codestream_sizes(tmp_path):
    from oracle import oracle as O
    mp.start_processes(_encode_set_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    descs = _set_descs()
    ref = [O.encode_image(synth.mixed_image(d), d["levels"], d["cb"], d["cb"], d["kernel"] == 53) for d in descs]
    seen = []
    for r in range(2):
        idx, counts, sizes = np.load(str(tmp_path / f"r{r}.npy"), allow_pickle=True)
        assert np.array_equal(counts, [len(x) for x in ref])  # every rank holds every image's size
        blob = open(str(tmp_path / f"r{r}.bin"), "rb").read()
        off = 0
        for i, n in zip(idx, sizes):
            assert blob[off:off + n] == ref[i]
            off += n
        assert list(idx) == shard.shard(descs, r, 2)
        seen += list(idx)
    assert sorted(seen) == list(range(len(descs)))
