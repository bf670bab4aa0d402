"""Several ranks: a batch of fields partitioned across two gloo ranks on the CPU.

The per-rank compression is replaced by the reference library (oracle/_ref, on the CPU): the
test covers the host logic of the split -- the partition, each rank's share, the gather of the
codestreams into field order on every rank -- and checks every codestream against a single
process compressing the same share.  (The GPU compression of a share is bwc_b200_compress_batch,
tested against the reference in tests/test_gpu_batch.py and tests/test_gpu_fullsize.py.)
"""
import os
import pickle
import socket
import sys

import numpy as np
import pytest

from conftest import ROOT, need_ref
from bigwhoop_b200 import multi


def _specs():
    from bigwhoop_b200 import fields
    desc = fields.uneven_batch(seed=5, n_fields=7, lo=9, hi=28)
    fs = [fields.spectral_field(d["shape"], d["seed"]).astype(d["dtype"]) for d in desc]
    specs = [dict(decomp=(2, 2, 2, 0), codeblocks=(3, 3, 3, 0), rate=str(d["rate"])) for d in desc]
    return fs, specs


def _ref_compress(fields, specs, precision):
    """stand-in for a rank's GPU batch: the reference library on the CPU, Compressor keywords"""
    from oracle import ref
    ref.reset_gain_lut(precision)
    return [ref.compress(f, precision=precision, decomp=s["decomp"], cb=s["codeblocks"],
                         rate=s["rate"]) for f, s in zip(fields, specs)]


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        fs, specs = _specs()
        cs = multi.compress_distributed(fs, specs, compress=_ref_compress)
        with open(out_path % rank, "wb") as f:
            pickle.dump(cs, f)
    finally:
        dist.destroy_process_group()


def test_partition_balances_input_bytes():
    sizes = [100, 90, 80, 10, 10, 5, 1]
    parts = multi.partition(sizes, 2)
    assert sorted(parts[0] + parts[1]) == list(range(len(sizes)))
    loads = [sum(sizes[i] for i in p) for p in parts]
    assert abs(loads[0] - loads[1]) <= max(sizes)
    assert parts == multi.partition(sizes, 2)   # deterministic
    assert multi.partition(sizes, 1) == [list(range(len(sizes)))]
    assert multi.partition([5], 3) == [[0], [], []]


def test_two_gloo_ranks_gather_every_codestream_in_order(tmp_path):
    need_ref("double")
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "rank%d.pkl")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = [pickle.load(open(out % r, "rb")) for r in range(2)]
    assert got[0] == got[1]
    fs, specs = _specs()
    parts = multi.partition([f.nbytes for f in fs], 2)
    for share in parts:
        expect = _ref_compress([fs[i] for i in share], [specs[i] for i in share], "double")
        for i, cs in zip(share, expect):
            assert got[0][i] == cs, i
