"""Sharding a set of images across GPUs (one process per GPU), and the multi-GPU set encoder.

Images, their tiles and their code-blocks are independent, so a multi-GPU encode needs no
exchange on the data path: each rank encodes its own share and writes its own codestreams.
The share is a greedy longest-processing-time (LPT) partition by estimated cost:
  cost(image) = pixels * levels + code-blocks * blocks_weight
(the DWT work grows with pixels and levels; tier-1 with the number of code-blocks).  LPT
assigns images in decreasing cost to the least-loaded rank, which keeps the makespan within
4/3 of the optimum.  The only collective is an optional gather of per-image byte counts to
rank 0 (for writing an index), over whatever process group the caller set up (NCCL on GPUs,
gloo in the CPU tests).
"""
import heapq
import math

import numpy as np


def codeblocks_of(w, h, levels, cb):
    """Number of code-blocks of one component (cb x cb blocks over every subband)."""
    n = 0
    ws, hs = [w], [h]
    for _ in range(levels):
        ws.append((ws[-1] + 1) // 2)
        hs.append((hs[-1] + 1) // 2)
    n += math.ceil(ws[levels] / cb) * math.ceil(hs[levels] / cb)
    for k in range(1, levels + 1):
        lw, lh = ws[k], hs[k]
        pw, ph = ws[k - 1], hs[k - 1]
        for bw, bh in ((pw - lw, lh), (lw, ph - lh), (pw - lw, ph - lh)):
            if bw > 0 and bh > 0:
                n += math.ceil(bw / cb) * math.ceil(bh / cb)
    return n


def image_cost(desc, blocks_weight=4096):
    """Estimated cost of one image description (dict with w, h, ncomp, levels, cb)."""
    w, h, nc, levels, cb = desc["w"], desc["h"], desc.get("ncomp", 1), desc["levels"], desc["cb"]
    return nc * (w * h * levels + codeblocks_of(w, h, levels, cb) * blocks_weight)


def lpt_partition(costs, nranks):
    """Greedy LPT: returns one list of item indices per rank (each list in increasing index
    order).  Ties go to the lowest rank, so the result is deterministic."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0, r) for r in range(nranks)]
    heapq.heapify(heap)
    parts = [[] for _ in range(nranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def shard(descs, rank, world, blocks_weight=4096):
    """Indices of the images rank `rank` of `world` encodes."""
    costs = [image_cost(d, blocks_weight) for d in descs]
    return lpt_partition(costs, world)[rank]


def gather_counts(local_indices, local_counts, n_total, group=None):
    """Gather per-image byte counts to every rank (all_gather of a dense vector where each rank
    fills its own images).  Returns a numpy int64 array of n_total counts."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    v = torch.zeros(n_total, dtype=torch.int64, device=dev)
    if len(local_indices):
        v[torch.as_tensor(local_indices, device=dev)] = torch.as_tensor(local_counts, dtype=torch.int64, device=dev)
    dist.all_reduce(v, op=dist.ReduceOp.SUM, group=group)
    return v.cpu().numpy()


def _gpu_encode_share(descs, images):
    """Encodes one rank's images with one batched encoder on the current CUDA device (one
    launch sequence for the whole share) and returns each image's codestream."""
    import torch
    from .batch import BatchEncoder
    from .codec import Context
    if not descs:
        return []
    be = BatchEncoder([dict(w=d["w"], h=d["h"], ncomp=d["ncomp"], kernel=d["kernel"], levels=d["levels"],
                            cb=d["cb"], steps=d.get("steps")) for d in descs],
                      ctx=Context(torch.cuda.current_device()))
    be.encode(images)
    return [be.codestream(i) for i in range(len(descs))]


def encode_set(descs, load_image, rank=0, world=1, encode_share=None, group=None, blocks_weight=4096):
    """Multi-GPU encoder of an image set: this rank encodes its LPT share of `descs` and the
    codestream sizes of every image are gathered to every rank.

    descs: one dict per image (w, h, ncomp, kernel, levels, cb[, steps]).
    load_image(i): image i as (h, w[, 3]) uint8 (numpy or CUDA tensor); called only for this
        rank's own images, so no rank holds the whole set.
    encode_share(share_descs, share_images): list of codestreams (bytes), one per image; by
        default one batched encode on this rank's GPU.
    Returns (indices of this rank's images, their codestreams, int64 array of every image's
    codestream bytes).  With world > 1 the byte-count gather is the one collective (an
    all-reduce over `group`); the encode itself exchanges nothing.  The reference encodes one
    image at a time on one in-order queue (src/OCLUtil.cpp:505-516)."""
    idx = shard(descs, rank, world, blocks_weight)
    mine = [descs[i] for i in idx]
    images = [load_image(i) for i in idx]
    streams = (encode_share or _gpu_encode_share)(mine, images)
    if len(streams) != len(idx):
        raise RuntimeError("encode_share returned a codestream count unlike its share")
    sizes = [len(s) for s in streams]
    if world > 1:
        counts = gather_counts(idx, sizes, len(descs), group)
    else:
        counts = np.zeros(len(descs), np.int64)
        counts[idx] = sizes
    return idx, streams, counts
