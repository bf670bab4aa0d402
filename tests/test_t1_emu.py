"""The tier-1 encoder's kernel logic on the CPU (no GPU needed).

The CUDA kernels' bodies -- the block-wide context modelling (t1_model.cuh), the MQ lane
coder, whole and in its two halves, with its finish (t1_mq.cuh, t1_common.cuh) -- are also
built for the host
(lib/emu/<precision>/libt1emu.so, 256 host threads standing in for the CUDA block).  Their
output is compared, codeblock by codeblock, with the C restatement of the reference encoder:

* every coded decision (context and value), pass by pass, against the restatement's trace;
* K, Z, truncation lengths, log slopes and the coded bytes against the restatement and, for the
  golden cases, against the reference's own values stored in tests/golden.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")
INDEX = json.load(open(os.path.join(GOLDEN, "cases.json")))
MAX_PASSES = {"double": 190, "single": 94}


def emu(precision):
    path = os.path.join(ROOT, "bigwhoop_b200", "lib", "emu", precision, "libt1emu.so")
    if not os.path.exists(path):
        from bigwhoop_b200 import build
        build.build_emu(precisions=(precision,))
    L = C.CDLL(path)
    fl = C.c_double if precision == "double" else C.c_float
    vp = C.c_void_p
    L.t1emu_encode.restype = C.c_longlong
    L.t1emu_encode.argtypes = [vp, vp, vp, fl, C.c_double, C.c_int, C.c_int, vp, vp, vp, vp, vp,
                               C.c_uint64, vp, vp, vp, C.c_uint32, vp]
    L.t1emu_transpose8.restype = C.c_ulonglong
    L.t1emu_transpose8.argtypes = [C.c_ulonglong]
    return L


def restated(precision):
    from oracle import restated as rs
    if not rs.available(precision):
        pytest.skip("restatement not built (make -C oracle restate)")
    return rs


def run_emu(L, work, dims, box, qt_eff, gain_step2, cls, erres, precision):
    mp = MAX_PASSES[precision]
    n = int(np.prod([box[4 + a] - box[a] for a in range(4)]))
    K = np.zeros(1, np.uint8)
    Z = np.zeros(1, np.uint8)
    pc = np.zeros(mp, np.uint32)
    dm = np.zeros(mp, np.int64)
    cap = n * 80 + 4096
    sym = np.zeros(cap, np.uint8)
    Ls = np.zeros(mp, np.uint32)
    Ss = np.zeros(mp + 1, np.uint16)
    bcap = n * 10 + 4096
    data = np.zeros(bcap, np.uint8)
    flags = np.zeros(1, np.uint32)
    d = np.asarray(dims, np.uint64)
    b = np.asarray(box, np.uint64)
    total = L.t1emu_encode(work.ctypes.data, d.ctypes.data, b.ctypes.data, qt_eff, gain_step2, cls,
                           int(erres), K.ctypes.data, Z.ctypes.data, pc.ctypes.data, dm.ctypes.data,
                           sym.ctypes.data, cap, Ls.ctypes.data, Ss.ctypes.data, data.ctypes.data,
                           bcap, flags.ctypes.data)
    assert total >= 0
    z = int(Z[0])
    return dict(K=int(K[0]), Z=z, counts=pc[:z].astype(np.uint64), symbols=sym[:total].copy(),
                L=Ls[:z].astype(np.uint64), S=Ss[:z + 1].copy(), data=data, flags=int(flags[0]),
                dmse=dm[:z].copy(), bcap=bcap)


def run_split(L, m, gain_step2, precision):
    """the same decisions through the coder in two halves (t1emu_mq_split)"""
    mp = MAX_PASSES[precision]
    vp = C.c_void_p
    L.t1emu_mq_split.restype = C.c_int
    L.t1emu_mq_split.argtypes = [vp, vp, C.c_int, C.c_int, vp, C.c_double, vp, vp, vp,
                                 C.c_uint32, vp]
    z = m["Z"]
    pc = np.zeros(mp, np.uint32)
    pc[:z] = m["counts"]
    dm = np.zeros(mp, np.int64)
    dm[:z] = m["dmse"]
    sym = np.concatenate([m["symbols"], np.zeros(16, np.uint8)])
    Ls = np.zeros(mp, np.uint32)
    Ss = np.zeros(mp + 1, np.uint16)
    data = np.zeros(m["bcap"], np.uint8)
    flags = np.zeros(1, np.uint32)
    rc = L.t1emu_mq_split(sym.ctypes.data, pc.ctypes.data, m["K"], z, dm.ctypes.data, gain_step2,
                          Ls.ctypes.data, Ss.ctypes.data, data.ctypes.data, m["bcap"],
                          flags.ctypes.data)
    assert rc == 0
    return dict(L=Ls[:z].astype(np.uint64), S=Ss[:z + 1].copy(), data=data, flags=int(flags[0]))


def test_transpose8_moves_bit_8k_plus_j_to_8j_plus_k():
    L = emu("double")
    rng = np.random.default_rng(0)
    for _ in range(200):
        x = int(rng.integers(0, 2**63)) * 2 + int(rng.integers(0, 2))
        y = L.t1emu_transpose8(x)
        for k in range(8):
            for j in range(8):
                assert ((x >> (8 * k + j)) & 1) == ((y >> (8 * j + k)) & 1)


def _compare(L, rs, work, dims, box, qt_eff, gain_step2, hb, erres, precision, golden=None):
    cls = rs.load(precision).rs_context_class(int(hb))
    cb = rs.make_codeblock(box, qt_eff, gain_step2, hb, precision)
    K, Z, trace, ends = rs.t1_symbols(work, dims, cb, erres, precision)
    Kr, Zr, Lr, Sr, data_r = rs.t1_encode(work, dims, cb, erres, precision)
    m = run_emu(L, work, dims, box, qt_eff, gain_step2, cls, erres, precision)
    # flag 2 (hull stack underflow: the reference would read below its stack) is a property of
    # the data; the restatement stops there the same way
    assert m["flags"] & ~2 == 0, m["flags"]
    assert (m["K"], m["Z"]) == (K, Z)
    counts = np.diff(np.concatenate([[0], ends])).astype(np.uint64)
    assert np.array_equal(m["counts"], counts), (m["counts"][:12], counts[:12])
    assert np.array_equal(m["symbols"], trace)
    assert np.array_equal(m["L"], Lr)
    assert np.array_equal(m["S"], Sr)
    n = int(Lr[-1]) if Z else 0
    assert bytes(m["data"][:n]) == data_r[:n]
    if K:
        # the coder in two halves gives the same truncation lengths, slopes and bytes
        sp = run_split(L, m, gain_step2, precision)
        assert sp["flags"] == m["flags"]
        assert np.array_equal(sp["L"], m["L"])
        assert np.array_equal(sp["S"], m["S"])
        assert bytes(sp["data"][:n + 16]) == bytes(m["data"][:n + 16])
    if golden is not None:
        gK, gZ, gL, gS, gdata = golden
        assert (m["K"], m["Z"]) == (gK, gZ)
        assert np.array_equal(m["L"], gL[:gZ])
        assert np.array_equal(m["S"], gS[:gZ + 1])
        assert bytes(m["data"][:len(gdata)]) == gdata


@pytest.mark.parametrize("name", sorted(INDEX))
def test_kernel_logic_matches_golden_codeblocks(name):
    meta = INDEX[name]
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    precision = meta["precision"]
    rs = restated(precision)
    L = emu(precision)
    f = g["field"]
    dims = rs.dims_of(f.shape)
    qm = meta["qm"] if meta["qm"] is not None else (62 if precision == "double" else 30)
    work, _ = rs.fill_normalize(f, qm, precision)
    rs.dwt_forward(work, dims, meta["decomp"], precision)
    for c in range(meta["codeblocks_n"]):
        geo = g["geom"][c]
        sub = g["subband"][c]
        if precision == "single":
            s2 = float(np.float32(sub[1]) * np.float32(sub[1]))
        else:
            s2 = sub[1] * sub[1]
        lo, hi = int(g["cb_offsets"][c]), int(g["cb_offsets"][c + 1])
        gold = (int(g["K"][c]), int(g["Z"][c]), g["L"][c], g["S"][c], bytes(g["cb_data"][lo:hi]))
        _compare(L, rs, work, dims, [int(v) for v in geo[:8]], sub[0], sub[2] * s2, int(geo[8]),
                 meta["erres"], precision, gold)


CASES = [
    # shape (z, y, x), codeblock box within the transformed field, highband, erres
    ((16, 32, 32), (0, 0, 0, 0, 32, 32, 16, 1), 0, 0),      # one 32x32x16 codeblock (4096 columns)
    ((16, 32, 32), (0, 0, 0, 0, 32, 32, 16, 1), 7, 1),      # diagonal class, error resilience
    ((20, 30, 37), (3, 5, 2, 0), 3, 0),                     # odd box: partial stripes, W not /16
    ((9, 13, 11), (0, 0, 0, 0, 11, 13, 9, 1), 1, 0),
    ((6, 7, 5), (1, 2, 1, 0, 4, 7, 6, 1), 2, 1),
    ((4, 64, 64), (0, 0, 0, 0, 64, 64, 4, 1), 5, 0),        # 64 x 64 x 4: wide rows
    ((40, 4, 3), (0, 0, 0, 0, 3, 4, 40, 1), 4, 0),          # W = 3: stripe above in the same thread
]


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("case", CASES, ids=[str(i) for i in range(len(CASES))])
def test_kernel_logic_matches_restatement(case, precision):
    rs = restated(precision)
    L = emu(precision)
    from bigwhoop_b200 import fields
    shape, box, hb, erres = case
    f = fields.shock_field(shape, 77)
    dims = rs.dims_of(shape)
    work, _ = rs.fill_normalize(f, 62 if precision == "double" else 30, precision)
    rs.dwt_forward(work, dims, (1, 1, 1, 0), precision)
    if len(box) == 4:
        x0, y0, z0, t0 = box
        box = (x0, y0, z0, t0, min(dims[0], x0 + 32), min(dims[1], y0 + 23), min(dims[2], z0 + 9), 1)
    qt = 1.0 / 8.0 if precision == "double" else 1.0 / 4.0
    _compare(L, rs, work, dims, list(box), qt, 0.37, hb, erres, precision)


# ---- decoder -----------------------------------------------------------------------------------

def emu_decode(L, work, dims, box, qt_eff, cls, erres, K, Z, data):
    L.t1emu_decode.restype = C.c_int
    fl = C.c_double if work.dtype == np.float64 else C.c_float
    L.t1emu_decode.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, fl, C.c_int, C.c_int, C.c_int,
                               C.c_int, C.c_char_p, C.c_uint32]
    d = np.asarray(dims, np.uint64)
    b = np.asarray(box, np.uint64)
    rc = L.t1emu_decode(work.ctypes.data, d.ctypes.data, b.ctypes.data, qt_eff, cls, int(erres),
                        int(K), int(Z), bytes(data), len(data))
    assert rc == 0


@pytest.mark.parametrize("name", sorted(INDEX))
def test_decoder_logic_matches_golden(name):
    """Every codeblock of the golden codestream decoded by the decoder's kernel bodies gives the
    reference's dequantised field (its hash is stored in the fixture)."""
    import hashlib
    meta = INDEX[name]
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    precision = meta["precision"]
    rs = restated(precision)
    L = emu(precision)
    f = g["field"]
    dims = rs.dims_of(f.shape)
    work = np.zeros(f.size, np.float64 if precision == "double" else np.float32)
    for c in range(meta["codeblocks_n"]):
        K, Z = int(g["dK"][c]), int(g["dZ"][c])
        if Z == 0:
            continue
        geo = g["geom"][c]
        cls = rs.load(precision).rs_context_class(int(geo[8]))
        lo = int(g["cb_offsets"][c])
        n = int(g["L"][c][Z - 1])
        emu_decode(L, work, dims, [int(v) for v in geo[:8]], g["subband"][c][0], cls,
                   meta["erres"], K, Z, g["cb_data"][lo:lo + n])
    assert hashlib.sha256(work.tobytes()).hexdigest() == meta["dequantized_sha"]


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("case", CASES, ids=[str(i) for i in range(len(CASES))])
def test_decoder_logic_matches_restatement_at_every_truncation(case, precision):
    """Codeblocks truncated after every kind of pass (significance, refinement, cleanup), as the
    quality layers cut them, decode like the restated decoder."""
    rs = restated(precision)
    L = emu(precision)
    from bigwhoop_b200 import fields
    shape, box, hb, erres = case
    f = fields.shock_field(shape, 78)
    dims = rs.dims_of(shape)
    work, _ = rs.fill_normalize(f, 62 if precision == "double" else 30, precision)
    rs.dwt_forward(work, dims, (1, 1, 1, 0), precision)
    if len(box) == 4:
        x0, y0, z0, t0 = box
        box = (x0, y0, z0, t0, min(dims[0], x0 + 32), min(dims[1], y0 + 23), min(dims[2], z0 + 9), 1)
    box = list(box)
    qt = 1.0 if precision == "double" else 1.0 / 4.0
    cls = rs.load(precision).rs_context_class(int(hb))
    cb = rs.make_codeblock(box, qt, 0.37, hb, precision)
    K, Z, Ls, _, data = rs.t1_encode(work, dims, cb, erres, precision)
    assert Z > 6
    dt = np.float64 if precision == "double" else np.float32
    for z in sorted({1, 2, 3, 4, 5, Z // 3, Z // 2, Z - 2, Z - 1, Z}):
        n = int(Ls[z - 1])
        ours = np.zeros(int(np.prod(dims)), dt)
        theirs = np.zeros_like(ours)
        emu_decode(L, ours, dims, box, qt, cls, erres, K, z, data[:n])
        rs.t1_decode(theirs, dims, cb, K, z, data[:n], erres, precision)
        assert np.array_equal(ours.view(np.uint64 if dt == np.float64 else np.uint32),
                              theirs.view(np.uint64 if dt == np.float64 else np.uint32)), z
