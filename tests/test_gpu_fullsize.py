"""Byte-identity with the reference at the benchmark workloads' full sizes.

Each test codes one benchmark workload at its stated size through this library's C API and
through the reference library compiled from its own sources (oracle/_ref, all host threads),
and requires identical codestreams and bit-identical decompressed fields:

* the single large field: 512^3 FP64 through the double build and 512^3 FP32 through the
  single build (spectral field + 8 tanh shocks + constant quarter, seed 1, 4 levels, 32x32x16
  codeblocks, layers 0.5/1/2/4 bpv);
* the uneven batch: 64 fields (seed 2, extents U[33, 300], FP32/FP64, per-field rate and
  depth) through bwc_b200_compress_batch, every codestream against the reference's;
* the combined 4D workload: 384^3 x 8 FP64 advected field (seed 3), 3 spatial + 2 temporal
  levels, 32x32x8x2 codeblocks, 6 layers 0.25 ... 8 bpv, through the batched path with the
  learned warm start, and its full decompression.
"""
import os

import numpy as np
import pytest

from conftest import need_ref
from parity import n_bit_diffs
from bigwhoop_b200 import bwc, fields

pytestmark = pytest.mark.gpu

RATES = "0.5,1,2,4"


def _threads():
    return os.cpu_count() or 1


@pytest.mark.parametrize("precision", ["double", "single"])
def test_single_large_field_512cube(gpu, precision):
    import torch
    ref = need_ref(precision)
    dt = np.float64 if precision == "double" else np.float32
    f = fields.shock_field((512, 512, 512), 1, dtype=dt, device="cuda")
    host = f.cpu().numpy()
    del f
    torch.cuda.empty_cache()
    kw = dict(decomp=(4, 4, 4, 0), rate=RATES)
    ref.set_threads(_threads(), precision)
    ref.reset_gain_lut(precision)
    cs_ref = ref.compress(host, precision=precision, cb=(5, 5, 4, 0), **kw)
    bwc.reset_gain_state(precision)
    cs = bwc.compress_array(host, precision=precision, codeblocks=(5, 5, 4, 0), **kw)
    assert len(cs) == len(cs_ref)
    assert cs == cs_ref
    out = bwc.decompress_array(cs, precision)
    out_ref = ref.decompress(cs_ref, host.shape, host.dtype, precision)
    assert n_bit_diffs(out, out_ref) == 0


def test_uneven_batch_64_fields(gpu):
    """Every codestream of the batched call equals the reference's for that field, with the
    codecs set up in the same order on both sides (the process-wide gain table grows with every
    set-up, in both libraries)."""
    import torch
    ref = need_ref("double")
    desc = fields.uneven_batch(seed=2, n_fields=64)
    fs = []
    for d in desc:
        g = fields.shock_field(d["shape"], d["seed"], dtype=d["dtype"], slope=d["slope"],
                               device="cuda")
        fs.append(g.cpu().numpy())
    torch.cuda.empty_cache()
    ref.set_threads(_threads(), "double")
    ref.reset_gain_lut("double")
    cs_ref = []
    for f, d in zip(fs, desc):
        lv = d["levels"]
        cs_ref.append(ref.compress(f, decomp=(lv, lv, lv, 0), cb=(5, 5, 4, 0), rate=str(d["rate"])))
    bwc.reset_gain_state("double")
    comps = [bwc.Compressor(f, decomp=(d["levels"],) * 3 + (0,), codeblocks=(5, 5, 4, 0),
                            rate=str(d["rate"])) for f, d in zip(fs, desc)]
    try:
        out = bwc.compress_batch(comps)
    finally:
        for c in comps:
            c.close()
    bad = [i for i, (a, b) in enumerate(zip(out, cs_ref)) if a != b]
    assert not bad, bad
    # decompression of a few of them, bit for bit
    for i in (0, 17, 63):
        assert n_bit_diffs(bwc.decompress_array(out[i]),
                           ref.decompress(cs_ref[i], fs[i].shape, fs[i].dtype)) == 0, i


def test_combined_4d_384cube_8steps(gpu):
    import torch
    from bigwhoop_b200 import ratemodel
    ref = need_ref("double")
    rates = "0.25,0.5,1,2,4,8"
    f = fields.advected_field((8, 384, 384, 384), 3, device="cuda")
    host = f.cpu().numpy()
    del f
    torch.cuda.empty_cache()
    ref.set_threads(_threads(), "double")
    ref.reset_gain_lut("double")
    cs_ref = ref.compress(host, decomp=(3, 3, 3, 2), cb=(5, 5, 3, 1), rate=rates)
    ratemodel.load_default()
    bwc.reset_gain_state()
    c = bwc.Compressor(host, decomp=(3, 3, 3, 2), codeblocks=(5, 5, 3, 1), rate=rates)
    try:
        cs = bwc.compress_batch([c])[0]
    finally:
        c.close()
    assert len(cs) == len(cs_ref)
    assert cs == cs_ref
    out = bwc.decompress_array(cs)
    out_ref = ref.decompress(cs_ref, host.shape, host.dtype)
    assert n_bit_diffs(out, out_ref) == 0
