"""The oracle, pinned (no GPU needed).

1. The golden fixtures (tests/golden, produced by the reference library) are reproduced by the
   reference library built here, when it is present.
2. The C restatement of the hot path (oracle/restate) reproduces every golden value stage by
   stage: normalisation, forward transform, each codeblock's tier-1 output, and on the decoder
   side tier-1 decoding, the inverse transform and denormalisation.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import ROOT, need_ref

GOLDEN = os.path.join(ROOT, "tests", "golden")
INDEX = json.load(open(os.path.join(GOLDEN, "cases.json")))
NAMES = sorted(INDEX)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def load_case(name):
    return INDEX[name], dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def restated(precision):
    from oracle import restated as rs
    if not rs.available(precision):
        pytest.skip("restatement not built (make -C oracle restate)")
    return rs


def gain_step2(sub, precision):
    qt_step, gain = sub[1], sub[2]
    if precision == "single":
        s2 = float(np.float32(qt_step) * np.float32(qt_step))
    else:
        s2 = qt_step * qt_step
    return gain * s2


def qm_of(meta, precision):
    if meta["qm"] is not None:
        return meta["qm"]
    return 62 if precision == "double" else 30


@pytest.mark.parametrize("name", NAMES)
def test_reference_reproduces_golden(name):
    import sys
    sys.path.insert(0, GOLDEN)
    from make_golden import generate
    meta, g = load_case(name)
    need_ref(meta["precision"])
    arrays, meta2 = generate(name)
    assert np.array_equal(arrays["field"], g["field"]), "field generator changed"
    for k in ("codestream", "K", "Z", "L", "S", "cb_data", "dK", "dZ", "geom"):
        assert np.array_equal(arrays[k], g[k]), k
    for k in ("normalized_sha", "transformed_sha", "dequantized_sha", "reconstructed_sha", "output_sha"):
        assert meta2[k] == meta[k], k


@pytest.mark.parametrize("name", NAMES)
def test_restatement_encoder_matches_golden(name):
    meta, g = load_case(name)
    precision = meta["precision"]
    rs = restated(precision)
    f = g["field"]
    dims = rs.dims_of(f.shape)
    work, stats = rs.fill_normalize(f, qm_of(meta, precision), precision)
    assert np.array_equal(stats.astype(np.float64), g["stats"]), (stats, g["stats"])
    assert sha(work) == meta["normalized_sha"]
    rs.dwt_forward(work, dims, meta["decomp"], precision)
    assert sha(work) == meta["transformed_sha"]
    for c in range(meta["codeblocks_n"]):
        geo = g["geom"][c]
        cb = rs.make_codeblock(geo[:8], g["subband"][c][0], gain_step2(g["subband"][c], precision),
                               geo[8], precision)
        K, Z, Ls, Ss, data = rs.t1_encode(work, dims, cb, meta["erres"], precision)
        assert (K, Z) == (g["K"][c], g["Z"][c]), c
        assert np.array_equal(Ls, g["L"][c][:Z]), c
        assert np.array_equal(Ss, g["S"][c][:Z + 1]), c
        lo, hi = int(g["cb_offsets"][c]), int(g["cb_offsets"][c + 1])
        assert data[:hi - lo] == bytes(g["cb_data"][lo:hi]), c


@pytest.mark.parametrize("name", NAMES)
def test_restatement_decoder_matches_golden(name):
    meta, g = load_case(name)
    precision = meta["precision"]
    rs = restated(precision)
    f = g["field"]
    dims = rs.dims_of(f.shape)
    work = np.zeros(f.size, np.float64 if precision == "double" else np.float32)
    for c in range(meta["codeblocks_n"]):
        K, Z = int(g["dK"][c]), int(g["dZ"][c])
        if Z == 0:
            continue
        geo = g["geom"][c]
        cb = rs.make_codeblock(geo[:8], g["subband"][c][0], 0.0, geo[8], precision)
        lo = int(g["cb_offsets"][c])
        n = int(g["L"][c][Z - 1])
        rs.t1_decode(work, dims, cb, K, Z, bytes(g["cb_data"][lo:lo + n]), meta["erres"], precision)
    assert sha(work) == meta["dequantized_sha"]
    rs.dwt_inverse(work, dims, meta["decomp"], precision)
    assert sha(work) == meta["reconstructed_sha"]
    out = rs.denormalize(work, g["stats"][0], g["stats"][1], qm_of(meta, precision), f.dtype, precision)
    assert sha(out.reshape(f.shape)) == meta["output_sha"]


KERNEL_CASES = [
    # shape, precision, decomp (x, y, z, t), kernels (x, y, z, t): 0 CDF 9/7, 1 LeGall 5/3
    ((24, 20, 16), "double", (2, 2, 2, 0), (1, 1, 1, 0)),
    ((17, 23, 13), "double", (3, 2, 3, 0), (1, 0, 1, 0)),
    ((17, 23, 13), "single", (2, 2, 2, 0), (1, 1, 1, 0)),
    ((6, 10, 12, 14), "double", (2, 2, 2, 1), (1, 1, 1, 1)),
    ((1, 1, 300), "double", (4, 0, 0, 0), (1, 0, 0, 0)),
]


@pytest.mark.parametrize("shape,precision,decomp,kernels", KERNEL_CASES)
def test_restated_legall_transform_matches_reference(shape, precision, decomp, kernels):
    """The restatement's LeGall 5/3 lifting (alone or mixed with 9/7 per axis) against the
    reference library's own forward transform stage, bit for bit."""
    ref = need_ref(precision)
    rs = restated(precision)
    from bigwhoop_b200 import fields
    dt = np.float64 if precision == "double" else np.float32
    f = fields.spectral_field(shape, 7).astype(dt)
    cb = (3, 3, 3, 1) if len(shape) == 4 else (3, 3, 3, 0)
    rc = ref.RefCompressor(f, precision=precision, decomp=decomp, cb=cb, rate="2",
                           kernels=kernels)
    try:
        rc.normalize()
        ref_norm = rc.work()
        rc.dwt()
        ref_dwt = rc.work()
    finally:
        rc.close()
    work, _ = rs.fill_normalize(f, 62 if precision == "double" else 30, precision)
    assert sha(work) == sha(ref_norm)
    rs.dwt_forward(work, rs.dims_of(f.shape), decomp, precision, kernels=kernels)
    assert work.view(np.uint64 if precision == "double" else np.uint32).tolist() == \
        ref_dwt.view(np.uint64 if precision == "double" else np.uint32).tolist()
    # and the plain 9/7 transform is not what the reference computed
    if any(kernels[a] and decomp[a] for a in range(4)):
        plain, _ = rs.fill_normalize(f, 62 if precision == "double" else 30, precision)
        rs.dwt_forward(plain, rs.dims_of(f.shape), decomp, precision)
        assert sha(plain) != sha(ref_dwt)


@pytest.mark.parametrize("shape,precision,decomp,kernels", KERNEL_CASES[:4])
def test_restated_legall_inverse_matches_reference(shape, precision, decomp, kernels):
    """The restatement's inverse LeGall 5/3 lifting against the reference decoder's inverse
    transform stage, applied to the reference's own dequantised coefficients of a 5/3
    codestream, bit for bit."""
    ref = need_ref(precision)
    rs = restated(precision)
    from bigwhoop_b200 import fields
    dt = np.float64 if precision == "double" else np.float32
    f = fields.spectral_field(shape, 8).astype(dt)
    cb = (3, 3, 3, 1) if len(shape) == 4 else (3, 3, 3, 0)
    ref.reset_gain_lut(precision)
    rc = ref.RefCompressor(f, precision=precision, decomp=decomp, cb=cb, rate="4",
                           kernels=kernels)
    try:
        cs = rc.compress()
    finally:
        rc.close()
    rd = ref.RefDecompressor(cs, f.shape, f.dtype, precision=precision)
    try:
        rd.t1()
        coeffs = rd.work()
        rd.idwt()
        ref_rec = rd.work()
    finally:
        rd.close()
    rs.dwt_inverse(coeffs, rs.dims_of(f.shape), decomp, precision, kernels=kernels)
    u = np.uint64 if precision == "double" else np.uint32
    assert coeffs.view(u).tolist() == ref_rec.view(u).tolist()


TILE_DWT_CASES = [
    # shape (z, y, x) or (t, z, y, x), precision, decomp, tile sizes (x, y, z, t), kernels
    ((26, 30, 27), "double", (3, 3, 3, 0), (13, 15, 9, 1), (0, 0, 0, 0)),
    ((26, 30, 27), "single", (2, 2, 2, 0), (11, 17, 13, 1), (0, 0, 0, 0)),
    ((20, 18, 22), "double", (2, 2, 2, 0), (7, 9, 11, 1), (1, 0, 1, 0)),
    # 4D: the kernel setter is left out (None: the reference's default, CDF 9/7); with it, the
    # reference's own transform of a tiled 4D field crashed here
    ((8, 20, 24, 30), "double", (2, 2, 2, 1), (13, 11, 9, 4), None),
]


@pytest.mark.parametrize("shape,precision,decomp,tiles,kernels", TILE_DWT_CASES)
def test_restated_tile_transform_matches_reference(shape, precision, decomp, tiles, kernels):
    """Every tile of a multi-tile field, including tiles whose level regions start at odd
    coordinates (the reference's odd-start lifting and flush), transformed by the restatement
    as by the reference library's own forward transform stage, bit for bit."""
    ref = need_ref(precision)
    rs = restated(precision)
    from bigwhoop_b200 import fields
    dt = np.float64 if precision == "double" else np.float32
    f = fields.spectral_field(shape, 9).astype(dt)
    dims = tuple(reversed(shape)) + (1,) * (4 - len(shape))          # x, y, z, t
    f4 = f.reshape(tuple(reversed(dims)))                            # t, z, y, x
    cb = (2, 2, 2, 1) if len(shape) == 4 else (2, 2, 2, 0)
    rc = ref.RefCompressor(f, precision=precision, decomp=decomp, cb=cb, rate="2",
                           kernels=kernels, tiles=tiles)
    kernels = (0, 0, 0, 0) if kernels is None else kernels
    try:
        nt = rc.num_tiles()
        counts = [-(-dims[a] // tiles[a]) for a in range(4)]
        assert nt == int(np.prod(counts)) and nt > 1
        odd_starts = 0
        for t in range(nt):
            idx, r = [], t
            for a in range(4):
                idx.append(r % counts[a])
                r //= counts[a]
            origin = [idx[a] * tiles[a] for a in range(4)]
            ext = [min(tiles[a], dims[a] - origin[a]) for a in range(4)]
            odd_starts += any(o % 2 for o in origin)
            # the reference's fill_buffer takes a tile's time slices from slice 0, not from the
            # tile's first slice (libbwc.c:727-729 index with t, not TS0 + t): the same here
            sub = f4[0:ext[3], origin[2]:origin[2] + ext[2],
                     origin[1]:origin[1] + ext[1], origin[0]:origin[0] + ext[0]]
            n = int(np.prod(ext))
            rc.select_tile(t)
            rc.normalize()
            ref_norm = rc.work()[:n].copy()
            rc.dwt()
            ref_dwt = rc.work()[:n].copy()
            work, _ = rs.fill_normalize(np.ascontiguousarray(sub), 62 if precision == "double"
                                        else 30, precision)
            assert sha(work) == sha(ref_norm), t
            rs.dwt_forward_tile(work, ext, origin, decomp, precision, kernels=kernels)
            u = np.uint64 if precision == "double" else np.uint32
            assert np.array_equal(work.view(u), ref_dwt.view(u)), (t, origin, ext)
        assert odd_starts > 0
    finally:
        rc.close()


TILE_INV_CASES = [
    # tile sizes multiples of 2^levels: every region of every tile starts at an even coordinate
    ((26, 30, 27), "double", (3, 3, 3, 0), (16, 16, 8, 1), (0, 0, 0, 0)),
    ((26, 30, 27), "single", (2, 2, 2, 0), (12, 8, 16, 1), (0, 0, 0, 0)),
    ((20, 18, 22), "double", (2, 2, 2, 0), (8, 12, 4, 1), (1, 0, 1, 0)),
    ((8, 20, 24, 30), "double", (2, 2, 2, 1), (16, 12, 8, 4), None),
    # tiles starting at odd coordinates
    ((26, 30, 27), "double", (3, 3, 3, 0), (13, 15, 9, 1), (0, 0, 0, 0)),
    ((20, 18, 22), "double", (2, 2, 2, 0), (7, 9, 11, 1), (1, 0, 1, 0)),
]


def _tiles(dims, tiles):
    counts = [-(-dims[a] // tiles[a]) for a in range(4)]
    for t in range(int(np.prod(counts))):
        idx, r = [], t
        for a in range(4):
            idx.append(r % counts[a])
            r //= counts[a]
        origin = [idx[a] * tiles[a] for a in range(4)]
        yield t, origin, [min(tiles[a], dims[a] - origin[a]) for a in range(4)]


def _all_even(origin, ext, decomp):
    """every level region of the tile starts at an even coordinate and none has an odd length
    starting at an odd coordinate (where the reference reads an unwritten buffer sample)"""
    import math
    for a in range(4):
        for lv in range(decomp[a]):
            r0 = math.ceil(np.float32(origin[a]) / np.float32(2 ** lv))
            if r0 % 2:
                return False
    return True


@pytest.mark.parametrize("shape,precision,decomp,tiles,kernels", TILE_INV_CASES)
def test_restated_tile_inverse_matches_reference(shape, precision, decomp, tiles, kernels):
    """The inverse transform of the tiles of a multi-tile reference codestream, by the
    restatement as by the reference library's own inverse transform stage, bit for bit, for every
    tile whose level regions all start at even coordinates (all tiles of the aligned tilings)."""
    ref = need_ref(precision)
    rs = restated(precision)
    from bigwhoop_b200 import fields
    dt = np.float64 if precision == "double" else np.float32
    f = fields.spectral_field(shape, 9).astype(dt)
    dims = tuple(reversed(shape)) + (1,) * (4 - len(shape))
    cb = (2, 2, 2, 1) if len(shape) == 4 else (2, 2, 2, 0)
    ref.reset_gain_lut(precision)
    cs = ref.compress(f, precision=precision, decomp=decomp, cb=cb, rate="4", kernels=kernels,
                      tiles=tiles)
    kernels = (0, 0, 0, 0) if kernels is None else kernels
    rd = ref.RefDecompressor(cs, f.shape, f.dtype, precision=precision)
    checked = 0
    try:
        assert rd.num_tiles() > 1
        for t, origin, ext in _tiles(dims, tiles):
            if not _all_even(origin, ext, decomp):
                continue
            n = int(np.prod(ext))
            rd.select_tile(t)
            rd.t1()
            deq = rd.work()[:n].copy()
            rd.idwt()
            rec = rd.work()[:n].copy()
            rs.dwt_inverse_tile(deq, ext, origin, decomp, precision, kernels=kernels)
            u = np.uint64 if precision == "double" else np.uint32
            assert np.array_equal(deq.view(u), rec.view(u)), (t, origin, ext)
            checked += 1
    finally:
        rd.close()
    assert checked >= 1


def test_reference_tile_inverse_depends_on_its_thread_count():
    """Documents why tiles starting at odd coordinates are not compared with the reference's
    decompression: its inverse transform of an odd-length line starting at an odd coordinate lifts
    a sample of its per-thread line buffer that the fill did not write, so its output changes
    with the number of OpenMP threads (this library and the restatement use zero there)."""
    ref = need_ref("double")
    from bigwhoop_b200 import fields
    f = fields.spectral_field((26, 30, 27), 9)
    ref.reset_gain_lut("double")
    cs = ref.compress(f, decomp=(3, 3, 3, 0), cb=(2, 2, 2, 0), rate="4", tiles=(13, 15, 9, 1))
    outs = []
    try:
        for th in (1, 3):
            ref.set_threads(th, "double")
            outs.append(ref.decompress(cs, f.shape, f.dtype))
    finally:
        ref.set_threads(os.cpu_count() or 1, "double")
    assert np.count_nonzero(outs[0].view(np.uint64) != outs[1].view(np.uint64)) > 0
