"""bwc_b200_t1_encode_codeblock_static: tier-1 encoding of one codeblock with no allocation.

Callers that cannot call cudaMalloc (device memory owned by a framework's pool, services that
cannot take an allocation's synchronisation) use this entry point with buffers they own; the
library's working memory is a fixed static device area.  Its results must equal what
bwc_compress computes for the same codeblock, and what the reference library computes for it
(oracle/_ref) -- bit for bit, as everywhere in tier-1 -- on two calls in a row (the static area
keeps the previous call's contents), with and without error resilience.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import need_ref
from parity import attach_stage_dump
from bigwhoop_b200 import bwc, fields

pytestmark = pytest.mark.gpu

MAX_PASSES = {"double": 190, "single": 94}


def _entry(precision):
    lib = C.CDLL(bwc.lib_path(precision))   # private handle: argument types stay local
    f = lib.bwc_b200_t1_encode_codeblock_static
    flt = C.c_double if precision == "double" else C.c_float
    f.restype = C.c_int
    f.argtypes = ([C.c_void_p] + [C.c_uint64] * 4 + [C.POINTER(C.c_uint64), flt, C.c_double, C.c_uint8,
                  C.c_uint8] + [C.c_void_p] * 5 + [C.c_uint32, C.c_void_p, C.c_void_p])
    return f


@pytest.mark.parametrize("erres", [0, 1])
@pytest.mark.parametrize("precision", ["double", "single"])
def test_static_codeblock_encoder_matches_compress(gpu, precision, erres):
    import torch
    ref = need_ref(precision)
    dt = np.float64 if precision == "double" else np.float32
    mp = MAX_PASSES[precision]
    f = fields.shock_field((40, 48, 56), 5).astype(dt)
    kw = dict(precision=precision, decomp=(3, 3, 3, 0), cb=(5, 5, 4, 0), rate="1,4",
              erres=bool(erres))
    # the reference's own tier-1 output of every codeblock
    ref.reset_gain_lut(precision)
    rc = ref.RefCompressor(f, **kw)
    try:
        rc.normalize()
        rc.dwt()
        rc.t1()
        rcb = [rc.codeblock(k) for k in range(rc.num_codeblocks())]
    finally:
        rc.close()
    bwc.reset_gain_state(precision)
    c = bwc.Compressor(f, precision=precision, decomp=(3, 3, 3, 0), codeblocks=(5, 5, 4, 0),
                       rate="1,4", erres=bool(erres))
    try:
        ncb = c.num_codeblocks()
        assert ncb == len(rcb)
        dump = attach_stage_dump(c, ncb, mp)
        c.compress()
        geoms, subs = [], []
        for k in range(ncb):
            g = np.zeros(10, np.uint64)
            assert c.L.bwc_b200_codeblock_geometry(c.codec, 0, k, g.ctypes.data) == 0
            st = np.zeros(3)
            c.L.bwc_b200_subband_steps(c.codec, 0, k, st.ctypes.data)
            geoms.append(g)
            subs.append(st)
    finally:
        c.close()

    encode = _entry(precision)
    dims = tuple(int(v) for v in reversed(f.shape)) + (1,)
    coeffs = torch.from_numpy(dump.transformed.copy()).cuda()
    cap = 1 << 20
    K = torch.zeros(1, dtype=torch.uint8, device="cuda")
    Z = torch.zeros(1, dtype=torch.uint8, device="cuda")
    L = torch.zeros(mp, dtype=torch.int32, device="cuda")
    S = torch.zeros(mp + 1, dtype=torch.int16, device="cuda")
    data = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    checked = 0
    for rnd in range(2):   # two calls in a row for every codeblock
        for k in range(ncb):
            g, st = geoms[k], subs[k]
            s2 = float(np.float32(st[1]) * np.float32(st[1])) if precision == "single" else st[1] * st[1]
            box = (C.c_uint64 * 8)(*[int(v) for v in g[:8]])
            data.fill_(0xAB)
            rc = encode(coeffs.data_ptr(), *dims, box, st[0], st[2] * s2, int(g[8]), erres,
                        K.data_ptr(), Z.data_ptr(), L.data_ptr(), S.data_ptr(), data.data_ptr(),
                        cap, status.data_ptr(), None)
            assert rc == 0
            torch.cuda.synchronize()
            m = dump.codeblock(k)
            z = int(Z.item())
            assert int(status.item()) == 0, (rnd, k)
            assert (int(K.item()), z) == (m["K"], m["Z"]), (rnd, k)
            assert np.array_equal(L.cpu().numpy().view(np.uint32)[:z].astype(np.uint64), m["L"]), (rnd, k)
            assert np.array_equal(S.cpu().numpy().view(np.uint16)[:z + 1], m["S"]), (rnd, k)
            n = int(m["L"][-1]) if z else 0
            got = bytes(data[:n].cpu().numpy())
            assert got == bytes(dump.data[m["offset"]:m["offset"] + n]), (rnd, k)
            r = rcb[k]
            assert (int(K.item()), z) == (r.K, r.Z), (rnd, k)
            assert np.array_equal(L.cpu().numpy().view(np.uint32)[:z].astype(np.uint64), r.L), (rnd, k)
            assert np.array_equal(S.cpu().numpy().view(np.uint16)[:z + 1], r.S), (rnd, k)
            assert got == r.data, (rnd, k)
            checked += 1
    assert checked == 2 * ncb


def test_static_codeblock_encoder_rejects_oversize_codeblocks(gpu):
    import torch
    encode = _entry("double")
    coeffs = torch.zeros((16, 64, 64), dtype=torch.float64, device="cuda")
    out = torch.zeros(1 << 16, dtype=torch.uint8, device="cuda")
    box = (C.c_uint64 * 8)(0, 0, 0, 0, 64, 64, 16, 1)   # 64 x 16 x 16 = 16384 stripe columns
    p = out.data_ptr()
    rc = encode(coeffs.data_ptr(), 64, 64, 16, 1, box, 1.0, 1.0, 1, 0, p, p, p, p, p, 1024, p, None)
    assert rc == 1
