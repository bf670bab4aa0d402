"""Host-side parity with the reference (no GPU): geometry, energy-gain state, tier-2 rate
control, packet headers, codestream layout and codestream parsing.

The reference's own tier-1 output (codeblock lengths, slopes, coded bytes) is fed into this
library's tier-2 through bwc_b200_assemble_from_tier1; the codestream must be byte-identical to
the one the reference assembles from the same data.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import GPU, need_ref
from bigwhoop_b200 import bwc, fields

CASES = [
    # shape, precision, dtype, decomp, codeblocks, rate
    ((64, 64, 64), "double", np.float64, (3, 3, 3, 0), (4, 4, 4, 0), "2"),
    ((64, 64, 64), "double", np.float64, None, None, "0.5,1,2,4"),
    ((33, 47, 61), "double", np.float64, (2, 2, 2, 0), (5, 5, 4, 0), "1,2"),
    ((33, 47, 61), "single", np.float32, (2, 2, 2, 0), (5, 5, 4, 0), "1,2"),
    ((33, 47, 61), "double", np.float32, (2, 2, 2, 0), (5, 5, 4, 0), "0.25"),
    ((8, 20, 24, 30), "double", np.float64, (2, 2, 2, 1), (3, 3, 3, 1), "0.25,8"),
    ((40, 17, 90), "double", np.float64, (3, 2, 4, 0), (4, 3, 5, 0), "4,0.5"),
    ((1, 1, 300), "double", np.float64, (4, 0, 0, 0), (6, 0, 0, 0), "2"),
    # eight layers: tag-tree and length-code state carried through many final headers
    ((48, 40, 36), "double", np.float64, (2, 2, 2, 0), (4, 4, 3, 0),
     "0.125,0.25,0.5,1,1.5,2,3,6"),
]


def _field(shape, dtype, seed=3):
    return fields.spectral_field(shape, seed).astype(dtype)


def _assemble_both(f, precision, decomp, cb, rate, precincts=None, qm=None, erres=False):
    ref = need_ref(precision)
    ref.reset_gain_lut(precision)
    bwc.reset_gain_state(precision)
    rc = ref.RefCompressor(f, precision=precision, decomp=decomp, cb=cb, rate=rate,
                           precincts=precincts, qm=-1 if qm is None else qm, erres=erres)
    mc = bwc.Compressor(f, precision=precision, decomp=decomp, codeblocks=cb, rate=rate,
                        precincts=precincts, qm=qm, erres=erres)
    try:
        assert np.array_equal(ref.gain_lut(precision), bwc.gain_state(precision))
        ncb = rc.num_codeblocks()
        assert mc.num_codeblocks() == ncb
        L = mc.L
        for c in range(ncb):
            cbk = rc.codeblock(c, with_data=False)
            g = np.zeros(10, np.uint64)
            assert L.bwc_b200_codeblock_geometry(mc.codec, 0, c, g.ctypes.data) == 0
            assert np.array_equal(g, cbk.geom), (c, g, cbk.geom)
            st = np.zeros(3)
            L.bwc_b200_subband_steps(mc.codec, 0, c, st.ctypes.data)
            assert np.array_equal(st, cbk.subband), (c, st, cbk.subband)
        rc.normalize(); rc.dwt(); rc.t1()
        MP = ref.MAX_PASSES[precision]
        K = np.zeros(ncb, np.uint8); Z = np.zeros(ncb, np.uint8)
        Ls = np.zeros(ncb * MP, np.uint64); Ss = np.zeros(ncb * (MP + 1), np.uint16)
        offs = np.zeros(ncb, np.uint64); data = bytearray()
        for c in range(ncb):
            cbk = rc.codeblock(c)
            K[c], Z[c] = cbk.K, cbk.Z
            Ls[c * MP:c * MP + cbk.Z] = cbk.L
            Ss[c * (MP + 1):c * (MP + 1) + cbk.Z + 1] = cbk.S
            offs[c] = len(data)
            data += cbk.data
        smin, smax = rc.tile_slopes()
        stats = rc.stats()
        rc.t2()
        cs_ref = rc.assemble()
        dt = np.float64 if precision == "double" else np.float32
        mm = np.array(stats[:2], dt)
        buf = np.frombuffer(bytes(data) + b"\0" * 64, np.uint8).copy()
        out = np.zeros(len(cs_ref) + 4096, np.uint8)
        stream = L.bwc_init_stream(f.ctypes.data, out.ctypes.data, 0)
        n = L.bwc_b200_assemble_from_tier1(mc.codec, stream, K.ctypes.data, Z.ctypes.data,
                                           Ls.ctypes.data, Ss.ctypes.data, buf.ctypes.data,
                                           offs.ctypes.data, mm.ctypes.data, smin, smax)
        return cs_ref, bytes(out[:n])
    finally:
        rc.close()
        mc.close()


@pytest.mark.parametrize("shape,precision,dtype,decomp,cb,rate", CASES)
def test_tier2_codestream_identical(shape, precision, dtype, decomp, cb, rate):
    f = _field(shape, dtype)
    cs_ref, cs_me = _assemble_both(f, precision, decomp, cb, rate)
    assert len(cs_me) == len(cs_ref)
    assert cs_me == cs_ref


PRECINCT_CASES = [
    # shape, decomp, codeblocks, precincts (log2 sizes), rate: many precincts, so every
    # resolution has many packets
    ((64, 64, 64), (3, 3, 3, 0), (3, 3, 3, 0), (4, 4, 4, 0), "0.5,2"),
    ((33, 47, 61), (2, 2, 2, 0), (3, 3, 3, 0), (4, 4, 5, 0), "1"),
    ((8, 20, 24, 30), (2, 2, 2, 1), (2, 2, 2, 1), (3, 3, 3, 1), "0.25,4"),
    ((40, 36, 44), (2, 2, 2, 0), (3, 3, 3, 0), (4, 4, 4, 0), "0.1,0.3,0.6,1,2,5"),
]


@pytest.mark.parametrize("shape,decomp,cb,precincts,rate", PRECINCT_CASES)
def test_tier2_codestream_identical_with_precincts(shape, decomp, cb, precincts, rate):
    f = _field(shape, np.float64)
    cs_ref, cs_me = _assemble_both(f, "double", decomp, cb, rate, precincts=precincts)
    assert len(cs_me) == len(cs_ref)
    assert cs_me == cs_ref


@pytest.mark.parametrize("qm,erres", [(40, False), (None, True)])
def test_tier2_codestream_identical_with_precincts_qm_erres(qm, erres):
    f = _field((32, 32, 32), np.float64)
    cs_ref, cs_me = _assemble_both(f, "double", (3, 3, 3, 0), (3, 3, 3, 0), "1,3",
                                   precincts=(4, 4, 4, 0), qm=qm, erres=erres)
    assert cs_me == cs_ref


def test_tier2_codestream_identical_with_precincts_single_precision():
    f = _field((33, 47, 61), np.float32)
    cs_ref, cs_me = _assemble_both(f, "single", (2, 2, 2, 0), (3, 3, 3, 0), "1,2",
                                   precincts=(4, 4, 4, 0))
    assert cs_me == cs_ref


PARSE_CASES = [c + (None,) for c in CASES[:6]] + [
    ((64, 64, 64), "double", np.float64, (3, 3, 3, 0), (3, 3, 3, 0), "0.5,2", (4, 4, 4, 0)),
]


@pytest.mark.parametrize("shape,precision,dtype,decomp,cb,rate,precincts", PARSE_CASES)
def test_parse_identical(shape, precision, dtype, decomp, cb, rate, precincts):
    ref = need_ref(precision)
    f = _field(shape, dtype)
    ref.reset_gain_lut(precision)
    cs = ref.compress(f, precision=precision, decomp=decomp, cb=cb, rate=rate,
                      precincts=precincts)
    rd = ref.RefDecompressor(cs, f.shape, f.dtype, precision=precision)
    d = bwc.Decompressor(cs, precision=precision)
    try:
        L = bwc.load(precision)
        ncb = rd.L.rp_num_codeblocks(rd.h, 0)
        MP = ref.MAX_PASSES[precision]
        for c in range(ncb):
            m1 = np.zeros(3, np.int64); L1 = np.zeros(MP, np.uint64)
            rd.L.rp_dcodeblock(rd.h, 0, c, m1.ctypes.data, L1.ctypes.data)
            m2 = np.zeros(3, np.int64); L2 = np.zeros(MP, np.uint64)
            assert L.bwc_b200_parsed_codeblock(d.codec, 0, c, m2.ctypes.data, L2.ctypes.data) == 0
            assert np.array_equal(m1, m2), (c, m1, m2)
            assert np.array_equal(L1, L2), c
    finally:
        rd.close()
        d.close()


def test_gain_state_accumulates_like_reference():
    """Every configure_codec / bwc_set_decomp adds to the process-wide gain table."""
    ref = need_ref("double")
    ref.reset_gain_lut("double")
    bwc.reset_gain_state("double")
    f = _field((16, 16, 16), np.float64)
    for _ in range(3):
        rc = ref.RefCompressor(f, decomp=(2, 2, 2, 0), rate="2")
        mc = bwc.Compressor(f, decomp=(2, 2, 2, 0), rate="2")
        assert np.array_equal(ref.gain_lut("double"), bwc.gain_state("double"))
        rc.close()
        mc.close()
    g = bwc.gain_state("double")
    # six table initialisations: level-1 low-pass entry is six times a single one (to rounding)
    bwc.reset_gain_state("double")
    mc = bwc.Compressor(f, rate="2")   # one initialisation
    one = bwc.gain_state("double")
    mc.close()
    assert g[0, 1] == pytest.approx(6 * one[0, 1], rel=1e-12)


def test_fast_rate_control_probes_equal_the_plain_probes():
    """With BWC_B200_CHECK_PROBES set, every rate-control probe is also evaluated the plain way
    (create_quality_layer with estimation) and any difference fails the compression."""
    import os
    import subprocess
    import sys
    need_ref("double")
    env = dict(os.environ, BWC_B200_CHECK_PROBES="1")
    here = os.path.dirname(os.path.abspath(__file__))
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-k", "tier2_codestream_identical",
                        os.path.join(here, "test_host_parity.py")], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "mismatch" not in r.stderr


def test_rate_control_in_small_pieces():
    """The tier-2 probes split each packet into pieces of codeblocks evaluated in parallel;
    small fields fit in one piece, so here every piece holds two codeblocks
    (BWC_B200_T2_PIECE=2) and the probe self-check is on: codestreams must still equal the
    reference's and every probe the plain evaluation."""
    import os
    import subprocess
    import sys
    need_ref("double")
    env = dict(os.environ, BWC_B200_T2_PIECE="2", BWC_B200_CHECK_PROBES="1")
    here = os.path.dirname(os.path.abspath(__file__))
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-k", "tier2_codestream_identical",
                        os.path.join(here, "test_host_parity.py")], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "mismatch" not in r.stderr


TILE_CASES = [
    # shape, decomp, codeblocks, tile sizes (x, y, z, t), rate
    ((32, 32, 32), (2, 2, 2, 0), (3, 3, 3, 0), (16, 16, 16, 1), "1,4"),
    ((33, 47, 61), (2, 2, 2, 0), (4, 4, 4, 0), (32, 24, 20, 1), "2"),
    ((8, 20, 24, 30), (2, 2, 2, 1), (3, 3, 3, 1), (16, 12, 10, 4), "0.5,4"),
]


@pytest.mark.parametrize("shape,decomp,cb,tiles,rate", TILE_CASES)
def test_tier2_codestream_identical_with_tiles(shape, decomp, cb, tiles, rate):
    """Multi-tile fields: the reference's tier-1 results of every tile, fed to this library's
    host half (per-tile rate control, packets, the multi-tile codestream layout), give the
    reference's codestream byte for byte."""
    ref = need_ref("double")
    f = _field(shape, np.float64)
    ref.reset_gain_lut("double")
    bwc.reset_gain_state("double")
    rc = ref.RefCompressor(f, decomp=decomp, cb=cb, rate=rate, tiles=tiles)
    mc = bwc.Compressor(f, decomp=decomp, codeblocks=cb, rate=rate, tiles=tiles)
    try:
        nt = rc.num_tiles()
        assert nt > 1
        MP = ref.MAX_PASSES["double"]
        K, Z, Ls, Ss, offs, mm, slopes = [], [], [], [], [], [], []
        data = bytearray()
        for t in range(nt):
            rc.select_tile(t)
            rc.normalize(); rc.dwt(); rc.t1()
            for c in range(rc.num_codeblocks()):
                cbk = rc.codeblock(c)
                K.append(cbk.K); Z.append(cbk.Z)
                l = np.zeros(MP, np.uint64); l[:cbk.Z] = cbk.L
                s = np.zeros(MP + 1, np.uint16); s[:cbk.Z + 1] = cbk.S
                Ls.append(l); Ss.append(s)
                offs.append(len(data))
                data += cbk.data
            mm += list(rc.stats()[:2])
            slopes += list(rc.tile_slopes())
            rc.t2()
        cs_ref = rc.assemble()
        K = np.array(K, np.uint8); Z = np.array(Z, np.uint8)
        Ls = np.concatenate(Ls); Ss = np.concatenate(Ss)
        offs = np.array(offs, np.uint64); mm = np.array(mm, np.float64)
        slopes = np.array(slopes, np.uint16)
        buf = np.frombuffer(bytes(data) + b"\0" * 64, np.uint8).copy()
        out = np.zeros(len(cs_ref) + 4096, np.uint8)
        L = mc.L
        L.bwc_b200_assemble_tiles_from_tier1.restype = C.c_size_t
        L.bwc_b200_assemble_tiles_from_tier1.argtypes = [C.c_void_p] * 10
        stream = L.bwc_init_stream(f.ctypes.data, out.ctypes.data, 0)
        try:
            n = L.bwc_b200_assemble_tiles_from_tier1(
                mc.codec, stream, K.ctypes.data, Z.ctypes.data, Ls.ctypes.data, Ss.ctypes.data,
                buf.ctypes.data, offs.ctypes.data, mm.ctypes.data, slopes.ctypes.data)
        finally:
            C.CDLL(None).free(C.c_void_p(stream))
        assert n > 0
        assert bytes(out[:n]) == cs_ref
    finally:
        rc.close()
        mc.close()


@pytest.mark.parametrize("shape,decomp,cb,tiles,rate", TILE_CASES)
def test_parse_identical_with_tiles(shape, decomp, cb, tiles, rate):
    """A multi-tile reference codestream parses to the reference parser's codeblocks, tile by
    tile (missing bit planes, passes, truncation lengths); bwc_decompress then decodes on the
    device, so without a GPU it fails there."""
    ref = need_ref("double")
    f = _field(shape, np.float64)
    ref.reset_gain_lut("double")
    rc = ref.RefCompressor(f, decomp=decomp, cb=cb, rate=rate, tiles=tiles)
    try:
        cs = rc.compress()
    finally:
        rc.close()
    rd = ref.RefDecompressor(cs, f.shape, f.dtype)
    L = bwc.load("double")
    L.bwc_b200_parsed_codeblock_of_tile.restype = C.c_int
    L.bwc_b200_parsed_codeblock_of_tile.argtypes = [C.c_void_p, C.c_uint32, C.c_uint8,
                                                    C.c_uint64, C.c_void_p, C.c_void_p]
    buf = np.frombuffer(cs + b"\0" * 64, np.uint8).copy()
    out = np.zeros(f.size, np.float64)
    d = L.bwc_alloc_decoder()
    st = L.bwc_init_stream(buf.ctypes.data, out.ctypes.data, bwc.DECOMP)
    try:
        assert L.bwc_create_decompression(d, st, 0) == 0
        nt = rd.num_tiles()
        assert nt > 1
        meta = np.zeros(3, np.int64)
        Lz = np.zeros(ref.MAX_PASSES["double"], np.uint64)
        total = 0
        for t in range(nt):
            rd.select_tile(t)
            for c in range(rd.num_codeblocks()):
                (K, Kmsbs, Z), Lr = rd.codeblock_lengths(c)
                assert L.bwc_b200_parsed_codeblock_of_tile(d, t, 0, c, meta.ctypes.data,
                                                           Lz.ctypes.data) == 0
                assert tuple(int(v) for v in meta) == (K, Kmsbs, Z), (t, c)
                assert np.array_equal(Lz[:Z], Lr[:Z]), (t, c)
                total += 1
            assert L.bwc_b200_parsed_codeblock_of_tile(d, t, 0, rd.num_codeblocks(),
                                                       meta.ctypes.data, None) == 1
        assert total > 0
        if not GPU:
            assert L.bwc_decompress(d, st) == 1
    finally:
        rd.close()
        L.bwc_free_codec(d)
        C.CDLL(None).free(C.c_void_p(st))
