"""GPU parity for multi-tile fields: bwc_set_tiles splits the field into tiles that are coded one
after another (libbwc.c:3231-3358 for compression, :3561-3667 for decompression), each with its
own normalisation, transform, tier-1 and rate control.

Compression is compared with the reference library byte for byte on every tiling, those whose
tiles start at odd coordinates included.  Decompression is compared with the reference library
bit for bit where every level region of every tile starts at an even coordinate; where a tile
starts at an odd coordinate, the reference's inverse transform reads a buffer sample it never
wrote (its result then depends on its OpenMP thread count), and the expected field is built
from the reference's own stages with the restated inverse transform in their place, which
takes that sample as zero, as this library does.
"""
import numpy as np
import pytest

from conftest import need_ref, need_restated
from bigwhoop_b200 import bwc, fields

pytestmark = pytest.mark.gpu

CASES = [
    # id, shape (z, y, x) or (t, z, y, x), field dtype, precision, decomp, codeblocks,
    # tile sizes (x, y, z, t), rate, kernels
    ("3d_even_tiles", (32, 32, 32), np.float64, "double", (2, 2, 2, 0), (3, 3, 3, 0),
     (16, 16, 16, 1), "1,4", None),
    ("3d_ragged_tiles", (33, 47, 61), np.float64, "double", (2, 2, 2, 0), (4, 4, 4, 0),
     (32, 24, 20, 1), "2", None),
    ("3d_odd_tiles", (26, 30, 27), np.float64, "double", (3, 3, 3, 0), (3, 3, 3, 0),
     (13, 15, 9, 1), "1,2", None),
    ("3d_odd_tiles_single", (26, 30, 27), np.float32, "single", (2, 2, 2, 0), (3, 3, 3, 0),
     (11, 17, 13, 1), "1", None),
    # float32 input to a double codec on even tiles (the reference library aborted with a heap
    # error here when such a field had ragged tiles, e.g. 26 x 30 x 27 in 16 x 16 x 8 tiles)
    ("3d_even_tiles_f32_input", (32, 32, 32), np.float32, "double", (2, 2, 2, 0), (3, 3, 3, 0),
     (16, 16, 16, 1), "0.5,4", None),
    ("3d_odd_tiles_5_3", (20, 18, 22), np.float64, "double", (2, 2, 2, 0), (3, 3, 3, 0),
     (7, 9, 11, 1), "2", (1, 0, 1, 0)),
    ("3d_even_tiles_5_3", (20, 18, 22), np.float64, "double", (2, 2, 2, 0), (3, 3, 3, 0),
     (8, 12, 4, 1), "2", (1, 0, 1, 0)),
    # time tiles: the second starts at time step 4 and, as in the reference, reads and writes
    # time steps 0..3 of the field (its fill and flush index time from the field's first step)
    ("4d_time_tiles", (8, 20, 24, 30), np.float64, "double", (2, 2, 2, 1), (3, 3, 3, 1),
     (16, 12, 8, 4), "0.5,4", None),
    ("4d_odd_tiles", (8, 20, 24, 30), np.float64, "double", (2, 2, 2, 1), (3, 3, 3, 1),
     (13, 11, 9, 4), "1", None),
]


def _dims(shape):
    return tuple(reversed(shape)) + (1,) * (4 - len(shape))


def _tiles(dims, tiles):
    counts = [-(-dims[a] // tiles[a]) for a in range(4)]
    for t in range(int(np.prod(counts))):
        idx, r = [], t
        for a in range(4):
            idx.append(r % counts[a])
            r //= counts[a]
        origin = [idx[a] * tiles[a] for a in range(4)]
        yield t, origin, [min(tiles[a], dims[a] - origin[a]) for a in range(4)]


def _all_even(dims, tiles, decomp):
    """every level region of every tile starts at an even coordinate"""
    for _, origin, _ in _tiles(dims, tiles):
        for a in range(4):
            for lv in range(decomp[a]):
                if -(-origin[a] // (1 << lv)) % 2:
                    return False
    return True


def _field(case):
    _, shape, dt, *_ = case
    return fields.spectral_field(shape, 31).astype(dt)


def _ref_compress(ref, f, case):
    _, shape, dt, precision, decomp, cb, tiles, rate, kernels = case
    ref.reset_gain_lut(precision)
    return ref.compress(f, precision=precision, decomp=decomp, cb=cb, rate=rate, tiles=tiles,
                        kernels=kernels)


def _expected_decompression(ref, cs, f, case):
    """the reference's tier-1 decoding and output stage per tile, with the restated inverse
    transform (unwritten buffer sample taken as zero) between them"""
    _, shape, dt, precision, decomp, cb, tiles, rate, kernels = case
    rs = need_restated(precision)
    rd = ref.RefDecompressor(cs, f.shape, f.dtype, precision=precision)
    try:
        for t, origin, ext in _tiles(_dims(shape), tiles):
            n = int(np.prod(ext))
            rd.select_tile(t)
            rd.t1()
            w = rd.work()[:n].copy()
            rs.dwt_inverse_tile(w, ext, origin, decomp, precision,
                                kernels=(0, 0, 0, 0) if kernels is None else kernels)
            rd.set_work(w)
            rd.finish()
        return rd.out.copy()
    finally:
        rd.close()


def _decompress(cs, f, precision):
    d = bwc.Decompressor(cs, precision=precision, out=np.zeros(f.shape, f.dtype))
    try:
        return d.decompress().copy()
    finally:
        d.close()


def _bits(a):
    a = np.ascontiguousarray(a).reshape(-1)
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_tiled_compression_matches_reference(gpu, case):
    _, shape, dt, precision, decomp, cb, tiles, rate, kernels = case
    ref = need_ref(precision)
    f = _field(case)
    cs_ref = _ref_compress(ref, f, case)
    bwc.reset_gain_state(precision)
    mc = bwc.Compressor(f, precision=precision, decomp=decomp, codeblocks=cb, rate=rate,
                        tiles=tiles, kernels=kernels)
    try:
        cs = mc.compress()
    finally:
        mc.close()
    assert len(cs) == len(cs_ref)
    assert cs == cs_ref


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_tiled_decompression(gpu, case):
    _, shape, dt, precision, decomp, cb, tiles, rate, kernels = case
    ref = need_ref(precision)
    f = _field(case)
    cs = _ref_compress(ref, f, case)
    out = _decompress(cs, f, precision)
    expected = _expected_decompression(ref, cs, f, case)
    assert int(np.count_nonzero(_bits(out) != _bits(expected))) == 0
    if _all_even(_dims(shape), tiles, decomp):
        full = ref.decompress(cs, f.shape, f.dtype, precision)
        assert int(np.count_nonzero(_bits(out) != _bits(full))) == 0


def test_tiled_fields_in_a_batch(gpu):
    """bwc_b200_compress_batch over tiled and untiled fields: each codestream equals the one the
    reference writes for that field alone (the gain table reset before each, on both sides)."""
    ref = need_ref("double")
    picks = [CASES[1], CASES[2], CASES[7]]
    fs = [_field(c) for c in picks] + [fields.spectral_field((30, 20, 40), 5)]
    untiled = ("untiled", (30, 20, 40), np.float64, "double", (2, 2, 2, 0), (3, 3, 3, 0),
               None, "2", None)
    cases = picks + [untiled]
    expected = [_ref_compress(ref, f, c) for f, c in zip(fs, cases)]
    for warm in range(2):
        comps = []
        try:
            for f, c in zip(fs, cases):
                bwc.reset_gain_state("double")
                _, shape, dt, precision, decomp, cb, tiles, rate, kernels = c
                comps.append(bwc.Compressor(f, precision=precision, decomp=decomp,
                                            codeblocks=cb, rate=rate, tiles=tiles,
                                            kernels=kernels))
            got = bwc.compress_batch(comps)
        finally:
            for m in comps:
                m.close()
        assert [len(g) for g in got] == [len(e) for e in expected], warm
        assert got == expected, warm
