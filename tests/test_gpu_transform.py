"""Forward transform paths against the reference: the bulk-copy z-streaming kernel (rows on
16-byte boundaries), the register z-streaming kernel (grids from one CTA, whose runs cross tiles
and time slices, to one per SM; odd and even row widths, partial edge tiles, 4D fields, both
precisions) and the 3D tile kernel must give the reference's coefficients bit for bit, and so
the same codestream.  Tuning modes: 0 tile kernel, 2 bulk-copy kernel wherever rows allow it
(else register streaming), 3 register streaming only, 1 the default choice."""
import numpy as np
import pytest

from conftest import need_ref
from parity import compare_stages
from bigwhoop_b200 import bwc, fields

pytestmark = pytest.mark.gpu

CLEAN = dict(normalized=0, transformed=0, codeblocks=0, flags=0, codestream=0)

CASES = [
    # id, shape (t, z, y, x order of numpy), dtype, precision, decomp, codeblocks, rate
    ("odd_extents", (33, 47, 61), np.float64, "double", (2, 2, 2, 0), (5, 5, 4, 0), "1,2"),
    ("odd_extents_single", (33, 47, 61), np.float32, "single", (2, 2, 2, 0), (5, 5, 4, 0), "1,2"),
    ("even_width_edge_tiles", (100, 70, 130), np.float64, "double", (3, 3, 3, 0), (5, 5, 4, 0), "1"),
    ("odd_width_edge_tiles", (99, 71, 129), np.float64, "double", (3, 3, 3, 0), (5, 5, 4, 0), "1"),
    ("uneven_decomp", (40, 17, 90), np.float64, "double", (3, 2, 4, 0), (4, 3, 5, 0), "4,0.5"),
    ("4d", (8, 20, 24, 30), np.float64, "double", (2, 2, 2, 1), (3, 3, 3, 1), "0.25,8"),
    ("4d_single", (6, 12, 16, 18), np.float32, "single", (1, 2, 2, 1), (3, 3, 3, 1), "1,4"),
    # rows on 16-byte boundaries in FP32 (width a multiple of 4), ragged edge tiles and levels
    ("aligned_rows_single", (50, 36, 76), np.float32, "single", (3, 3, 3, 0), (5, 5, 4, 0), "1,2"),
    # extents below one tile, repeated reflection, odd level extents from level 1 on
    ("small_levels", (9, 33, 18), np.float64, "double", (1, 2, 1, 0), (3, 3, 3, 0), "2"),
]
TUNINGS = [(0, 0), (2, 0), (2, 1), (2, 7), (2, 50), (3, 0), (3, 1), (3, 7), (1, 0)]   # (mode, CTAs)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_transform_paths_match_reference(gpu, case):
    _, shape, dtype, precision, decomp, cb, rate = case
    ref = need_ref(precision)
    f = fields.spectral_field(shape, 5).astype(dtype)
    streams = set()
    try:
        for mode, zlen in TUNINGS:
            bwc.set_transform_tuning(mode, zlen, precision)
            rep, cs, cs_ref = compare_stages(f, ref, precision=precision, decomp=decomp, cb=cb,
                                             rate=rate)
            assert rep == CLEAN, (mode, zlen, rep)
            streams.add(cs)
    finally:
        bwc.set_transform_tuning(1, 0, precision)
    assert len(streams) == 1
