"""GPU path against the committed golden fixtures and the C restatement (no reference library
needed at run time).

Golden: every fixture's codestream is reproduced byte for byte through the C API, every
codeblock's tier-1 output matches, and decompressing the golden codestream gives the golden
field bit for bit.

Restatement: on fields larger than the fixtures, the GPU's normalised field, coefficients and
per-codeblock tier-1 output equal the restatement's, computed on the same input.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import ROOT
from parity import attach_stage_dump
from bigwhoop_b200 import bwc, fields

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(ROOT, "tests", "golden")
INDEX = json.load(open(os.path.join(GOLDEN, "cases.json")))
MAX_PASSES = {"double": 190, "single": 94}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", sorted(INDEX))
def test_golden_codestream_and_decompression(gpu, name):
    meta = INDEX[name]
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    precision = meta["precision"]
    f = g["field"]
    bwc.reset_gain_state(precision)
    c = bwc.Compressor(f, precision=precision, decomp=tuple(meta["decomp"]),
                       codeblocks=tuple(meta["codeblocks"]), rate=meta["rate"], qm=meta["qm"],
                       erres=meta["erres"])
    try:
        ncb = c.num_codeblocks()
        assert ncb == meta["codeblocks_n"]
        dump = attach_stage_dump(c, ncb, MAX_PASSES[precision])
        cs = c.compress()
    finally:
        c.close()
    assert sha(dump.normalized) == meta["normalized_sha"]
    assert sha(dump.transformed) == meta["transformed_sha"]
    for k in range(ncb):
        m = dump.codeblock(k)
        assert (m["K"], m["Z"]) == (g["K"][k], g["Z"][k]), k
        assert np.array_equal(m["L"], g["L"][k][:m["Z"]]), k
        assert np.array_equal(m["S"], g["S"][k][:m["Z"] + 1]), k
        lo, hi = int(g["cb_offsets"][k]), int(g["cb_offsets"][k + 1])
        n = int(g["L"][k][m["Z"] - 1]) if m["Z"] else 0
        assert bytes(dump.data[m["offset"]:m["offset"] + n]) == bytes(g["cb_data"][lo:lo + n]), k
    assert cs == g["codestream"].tobytes()
    bwc.reset_gain_state(precision)
    out = bwc.decompress_array(g["codestream"].tobytes(), precision)
    assert sha(out) == meta["output_sha"]


RESTATE_CASES = [
    # shape, dtype, precision, decomp, codeblocks, rate, erres
    ((48, 40, 56), np.float64, "double", (3, 3, 3, 0), (5, 5, 4, 0), "0.5,2", False),
    ((40, 44, 36), np.float32, "single", (3, 3, 2, 0), (5, 4, 4, 0), "1,4", False),
    ((6, 16, 20, 24), np.float64, "double", (2, 2, 2, 1), (4, 4, 3, 1), "2", True),
]


@pytest.mark.parametrize("case", RESTATE_CASES, ids=["double", "single", "4d_erres"])
def test_stages_match_restatement(gpu, case):
    from oracle import restated as rs
    shape, dtype, precision, decomp, cbs, rate, erres = case
    if not rs.available(precision):
        pytest.fail("restatement library missing: build with make -C oracle restate")
    f = fields.shock_field(shape[-3:], 9).astype(dtype)
    if len(shape) == 4:
        f = np.stack([fields.spectral_field(shape[1:], 30 + t).astype(dtype) for t in range(shape[0])])
    bwc.reset_gain_state(precision)
    c = bwc.Compressor(f, precision=precision, decomp=decomp, codeblocks=cbs, rate=rate, erres=erres)
    try:
        ncb = c.num_codeblocks()
        dump = attach_stage_dump(c, ncb, MAX_PASSES[precision])
        c.compress()
        geoms, subs = [], []
        for k in range(ncb):
            gg = np.zeros(10, np.uint64)
            assert c.L.bwc_b200_codeblock_geometry(c.codec, 0, k, gg.ctypes.data) == 0
            st = np.zeros(3)
            c.L.bwc_b200_subband_steps(c.codec, 0, k, st.ctypes.data)
            geoms.append(gg)
            subs.append(st)
    finally:
        c.close()
    qm = 62 if precision == "double" else 30
    dims = rs.dims_of(f.shape)
    work, _ = rs.fill_normalize(f, qm, precision)
    assert sha(work) == sha(dump.normalized)
    rs.dwt_forward(work, dims, decomp, precision)
    assert sha(work) == sha(dump.transformed)
    for k in range(ncb):
        st = subs[k]
        s2 = float(np.float32(st[1]) * np.float32(st[1])) if precision == "single" else st[1] * st[1]
        cb = rs.make_codeblock(geoms[k][:8], st[0], st[2] * s2, geoms[k][8], precision)
        K, Z, Ls, Ss, data = rs.t1_encode(work, dims, cb, erres, precision)
        m = dump.codeblock(k)
        assert (m["K"], m["Z"]) == (K, Z), k
        assert np.array_equal(m["L"], Ls), k
        assert np.array_equal(m["S"], Ss), k
        n = int(Ls[-1]) if Z else 0
        assert bytes(dump.data[m["offset"]:m["offset"] + n]) == data[:n], k
