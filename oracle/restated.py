"""ctypes binding of the C restatement (oracle/restate/bwc_restate.c) -- test infrastructure.

Only the test suite, the smoke check and the benchmark's CPU-baseline leg use this module; the
product library never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MAX_PASSES = 190
_libs = {}


class RsCodeblock(C.Structure):
    _fields_ = [("x0", C.c_uint64), ("y0", C.c_uint64), ("z0", C.c_uint64), ("t0", C.c_uint64),
                ("x1", C.c_uint64), ("y1", C.c_uint64), ("z1", C.c_uint64), ("t1", C.c_uint64),
                ("qt_eff", C.c_double), ("gain_step2", C.c_double), ("cls", C.c_int)]


class RsCodeblockSingle(C.Structure):
    _fields_ = [("x0", C.c_uint64), ("y0", C.c_uint64), ("z0", C.c_uint64), ("t0", C.c_uint64),
                ("x1", C.c_uint64), ("y1", C.c_uint64), ("z1", C.c_uint64), ("t1", C.c_uint64),
                ("qt_eff", C.c_float), ("gain_step2", C.c_double), ("cls", C.c_int)]


def lib_path(precision="double"):
    return os.path.join(HERE, "_build", "librestate_%s.so" % ("d" if precision == "double" else "s"))


def available(precision="double"):
    return os.path.exists(lib_path(precision))


def load(precision="double"):
    if precision in _libs:
        return _libs[precision]
    L = C.CDLL(lib_path(precision))
    vp, u64 = C.c_void_p, C.c_uint64
    fl = C.c_double if precision == "double" else C.c_float
    L.rs_precision_bits.restype = C.c_int
    L.rs_fill_normalize.argtypes = [vp, C.c_int, u64, C.c_uint8, vp, vp]
    L.rs_denormalize.argtypes = [vp, u64, fl, fl, C.c_uint8, vp, C.c_int]
    L.rs_dwt_forward.argtypes = [vp, vp, vp]
    L.rs_dwt_inverse.argtypes = [vp, vp, vp]
    L.rs_dwt_forward_kernels.argtypes = [vp, vp, vp, vp]
    L.rs_dwt_inverse_kernels.argtypes = [vp, vp, vp, vp]
    L.rs_dwt_forward_tile.argtypes = [vp, vp, vp, vp, vp]
    L.rs_dwt_inverse_tile.argtypes = [vp, vp, vp, vp, vp]
    L.rs_context_class.restype = C.c_int
    L.rs_context_class.argtypes = [C.c_uint32]
    L.rs_t1_encode.restype = C.c_int64
    L.rs_t1_encode.argtypes = [vp, vp, vp, C.c_int, vp, vp, vp, vp, vp, u64]
    L.rs_set_symbol_trace.argtypes = [vp, u64, vp]
    L.rs_symbol_trace_count.restype = u64
    L.rs_t1_decode.restype = C.c_int
    L.rs_t1_decode.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int, vp, u64]
    _libs[precision] = L
    return L


def _dtype(precision):
    return np.float64 if precision == "double" else np.float32


def dims_of(shape):
    """(nX, nY, nZ, nTS) of a C-ordered array whose last axis is x."""
    d = tuple(int(v) for v in reversed(shape))
    return np.array(d + (1,) * (4 - len(d)), dtype=np.uint64)


def fill_normalize(field, qm, precision="double"):
    L = load(precision)
    f = np.ascontiguousarray(field)
    work = np.zeros(f.size, dtype=_dtype(precision))
    stats = np.zeros(4, dtype=_dtype(precision))
    L.rs_fill_normalize(f.ctypes.data, int(f.dtype == np.float64), f.size, qm, work.ctypes.data,
                        stats.ctypes.data)
    return work, stats


def denormalize(work, pmin, pmax, qm, out_dtype, precision="double"):
    L = load(precision)
    out = np.zeros(work.size, dtype=out_dtype)
    L.rs_denormalize(work.ctypes.data, work.size, pmin, pmax, qm, out.ctypes.data,
                     int(np.dtype(out_dtype) == np.float64))
    return out


def dwt_forward(work, dims, decomp, precision="double", kernels=None):
    """kernels: per axis (x, y, z, t), 0 CDF 9/7 (default), 1 LeGall 5/3"""
    dec = np.array(decomp, dtype=np.uint8)
    d = np.asarray(dims, np.uint64)
    if kernels is None:
        load(precision).rs_dwt_forward(work.ctypes.data, d.ctypes.data, dec.ctypes.data)
    else:
        k = np.array(kernels, dtype=np.uint8)
        load(precision).rs_dwt_forward_kernels(work.ctypes.data, d.ctypes.data, dec.ctypes.data,
                                               k.ctypes.data)
    return work


def dwt_inverse(work, dims, decomp, precision="double", kernels=None):
    dec = np.array(decomp, dtype=np.uint8)
    d = np.asarray(dims, np.uint64)
    if kernels is None:
        load(precision).rs_dwt_inverse(work.ctypes.data, d.ctypes.data, dec.ctypes.data)
    else:
        k = np.array(kernels, dtype=np.uint8)
        load(precision).rs_dwt_inverse_kernels(work.ctypes.data, d.ctypes.data, dec.ctypes.data,
                                               k.ctypes.data)
    return work


def make_codeblock(box, qt_eff, gain_step2, highband, precision="double"):
    L = load(precision)
    T = RsCodeblock if precision == "double" else RsCodeblockSingle
    return T(*[int(v) for v in box], qt_eff, gain_step2, L.rs_context_class(int(highband)))


def t1_encode(work, dims, cb, erres=False, precision="double"):
    """(K, Z, L[Z], S[Z+1], coded bytes of the whole codeword)."""
    L = load(precision)
    K = np.zeros(1, np.uint8)
    Z = np.zeros(1, np.uint8)
    Ls = np.zeros(MAX_PASSES, np.uint64)
    Ss = np.zeros(MAX_PASSES + 1, np.uint16)
    n = int((cb.x1 - cb.x0) * (cb.y1 - cb.y0) * (cb.z1 - cb.z0) * (cb.t1 - cb.t0))
    cap = n * 10 + 4096
    data = np.zeros(cap, np.uint8)
    nb = L.rs_t1_encode(work.ctypes.data, np.asarray(dims, np.uint64).ctypes.data, C.byref(cb),
                        int(erres), K.ctypes.data, Z.ctypes.data, Ls.ctypes.data, Ss.ctypes.data,
                        data.ctypes.data, cap)
    if nb < 0:
        raise RuntimeError("restated tier-1 encoder ran out of space")
    z = int(Z[0])
    return int(K[0]), z, Ls[:z].copy(), Ss[:z + 1].copy(), bytes(data[:nb])


def t1_symbols(work, dims, cb, erres=False, precision="double"):
    """The coded decisions of one codeblock in coding order, one byte each
    (context << 1 | decision), and the decision count at the end of every pass."""
    L = load(precision)
    n = int((cb.x1 - cb.x0) * (cb.y1 - cb.y0) * (cb.z1 - cb.z0) * (cb.t1 - cb.t0))
    cap = n * 80 + 4096
    buf = np.zeros(cap, np.uint8)
    ends = np.zeros(MAX_PASSES, np.uint64)
    L.rs_set_symbol_trace(buf.ctypes.data, cap, ends.ctypes.data)
    try:
        K, Z, _, _, _ = t1_encode(work, dims, cb, erres, precision)
        total = int(L.rs_symbol_trace_count())
    finally:
        L.rs_set_symbol_trace(None, 0, None)
    assert total <= cap
    return K, Z, buf[:total].copy(), ends[:Z].copy()


def t1_decode(work, dims, cb, K, Z, data, erres=False, precision="double"):
    L = load(precision)
    buf = np.frombuffer(bytes(data) + b"\0" * 16, dtype=np.uint8).copy()
    rc = L.rs_t1_decode(work.ctypes.data, np.asarray(dims, np.uint64).ctypes.data, C.byref(cb),
                        int(erres), int(K), int(Z), buf.ctypes.data, len(data))
    assert rc == 0
    return work


def dwt_inverse_tile(work, dims, origin, decomp, precision="double", kernels=(0, 0, 0, 0)):
    """inverse transform of one tile: dims its extent, origin its first sample (x, y, z, t)"""
    d = np.asarray(dims, np.uint64)
    o = np.asarray(origin, np.uint64)
    dec = np.array(decomp, dtype=np.uint8)
    k = np.array(kernels, dtype=np.uint8)
    load(precision).rs_dwt_inverse_tile(work.ctypes.data, d.ctypes.data, o.ctypes.data,
                                        dec.ctypes.data, k.ctypes.data)
    return work


def dwt_forward_tile(work, dims, origin, decomp, precision="double", kernels=(0, 0, 0, 0)):
    """forward transform of one tile: dims its extent, origin its first sample (x, y, z, t)"""
    d = np.asarray(dims, np.uint64)
    o = np.asarray(origin, np.uint64)
    dec = np.array(decomp, dtype=np.uint8)
    k = np.array(kernels, dtype=np.uint8)
    load(precision).rs_dwt_forward_tile(work.ctypes.data, d.ctypes.data, o.ctypes.data,
                                        dec.ctypes.data, k.ctypes.data)
    return work
