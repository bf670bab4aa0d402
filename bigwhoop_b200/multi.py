"""Several GPUs: a batch of independent fields partitioned across ranks.

Every field is its own codec, so a batch shards with no exchange of coefficients: rank r
compresses the fields assigned to it on its own GPU (one bwc_b200_compress_batch call), and the
codestreams are then gathered so that every rank holds all of them in field order.  The only
collective is that gather of the finished codestreams (bytes, a few percent of the input).

One process per GPU, launched by torchrun; torch.distributed carries the gather (NCCL between
GPUs, gloo on the CPU for the tests).
"""
from __future__ import annotations

from typing import Callable, List, Sequence

import numpy as np


def partition(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Field indices per rank: largest fields first, each to the rank with the least input bytes
    so far (ties to the lower rank).  Every rank's list is in ascending field order."""
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(x) for x in out]


def _default_compress(fields, specs, precision):
    from bigwhoop_b200 import bwc
    # codestreams depend on the process-wide gain table, which grows with every codec set up
    # (as in the reference); each rank's share starts from the reset state
    bwc.reset_gain_state(precision)
    comps = [bwc.Compressor(f, precision=precision, **spec) for f, spec in zip(fields, specs)]
    try:
        return bwc.compress_batch(comps)
    finally:
        for c in comps:
            c.close()


def compress_distributed(fields: Sequence[np.ndarray], specs: Sequence[dict], *,
                         precision: str = "double",
                         compress: Callable | None = None, group=None) -> List[bytes]:
    """Compresses the fields assigned to this rank and returns every field's codestream, in field
    order, on every rank.  ``specs[i]`` holds the Compressor keywords of field i (rate, decomp,
    codeblocks, ...).  Every rank must pass the same fields and specs.  ``compress(fields, specs,
    precision)`` replaces the per-rank compression (default: the gain table reset, then one
    bwc_b200_compress_batch call on the rank's current GPU), so a field's codestream equals the
    one a single process makes when it compresses that rank's share as one batch."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    parts = partition([f.nbytes for f in fields], world)
    mine = parts[rank]
    fn = compress or _default_compress
    streams = fn([fields[i] for i in mine], [specs[i] for i in mine], precision) if mine else []
    gathered: List = [None] * world
    dist.all_gather_object(gathered, list(zip(mine, streams)), group=group)
    out: List[bytes] = [b""] * len(fields)
    for pairs in gathered:
        for i, cs in pairs:
            out[i] = cs
    return out
