"""TEST INFRASTRUCTURE ONLY: ctypes access to the reference library built by oracle/Makefile.

``oracle/_ref/{double,single}/libbwc_ref.so`` is the unmodified BigWhoop libbwc compiled from
its own sources plus ``ref_probe.c``.  This module drives it the way a user of libbwc does
(bwc_alloc_coder -> setters -> bwc_create_compression -> bwc_compress, and the decompression
calls), and exposes the probe's stage-by-stage entry points so tests can read intermediate
results.  Only tests, ``__graft_entry__.smoke`` and bench.py's CPU-baseline arm use it.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MAX_PASSES = {"double": 64 * 3 - 2, "single": 32 * 3 - 2}

_libs = {}


def lib_path(precision="double"):
    return os.path.join(HERE, "_ref", precision, "libbwc_ref.so")


def available(precision="double"):
    return os.path.exists(lib_path(precision))


def load(precision="double"):
    if precision in _libs:
        return _libs[precision]
    path = lib_path(precision)
    if not os.path.exists(path):
        raise FileNotFoundError(f"reference library not built: {path} (run make -C oracle)")
    L = C.CDLL(path, mode=C.RTLD_LOCAL)
    vp, u64, u8p = C.c_void_p, C.c_uint64, C.POINTER(C.c_uint8)
    L.rp_open_compress.restype = vp
    L.rp_open_compress.argtypes = [vp, u64, u64, u64, u64, C.c_uint8, C.c_int, u8p, u8p,
                                   C.c_int, C.c_int, C.c_char_p, vp]
    L.rp_compress_full.restype = C.c_size_t
    L.rp_compress_full.argtypes = [vp]
    L.rp_set_precincts.argtypes = [u8p]
    L.rp_set_kernels.argtypes = [u8p]
    L.rp_set_tiles.argtypes = [C.POINTER(C.c_uint64)]
    L.rp_select_tile.restype = C.c_int
    L.rp_select_tile.argtypes = [vp, C.c_int]
    L.rp_num_tiles.restype = u64
    L.rp_num_tiles.argtypes = [vp]
    for n in ("rp_stage_normalize", "rp_stage_dwt", "rp_stage_t1", "rp_dstage_t1",
              "rp_dstage_idwt", "rp_dstage_finish"):
        getattr(L, n).restype = C.c_int
        getattr(L, n).argtypes = [vp, C.c_int]
    L.rp_stage_t2.restype = C.c_int
    L.rp_stage_t2.argtypes = [vp]
    L.rp_stage_assemble.restype = C.c_size_t
    L.rp_stage_assemble.argtypes = [vp]
    L.rp_copy_work.restype = u64
    L.rp_copy_work.argtypes = [vp, vp]
    L.rp_set_work.restype = C.c_int
    L.rp_set_work.argtypes = [vp, vp, u64]
    L.rp_param_stats.argtypes = [vp, C.c_int, vp]
    L.rp_num_codeblocks.restype = u64
    L.rp_num_codeblocks.argtypes = [vp, C.c_int]
    L.rp_codeblock.restype = C.c_int
    L.rp_codeblock.argtypes = [vp, C.c_int, u64, vp, vp, vp, vp, vp, u64]
    L.rp_codeblock_subband.argtypes = [vp, C.c_int, u64, vp]
    L.rp_tile_slopes.argtypes = [vp, vp]
    L.rp_codec_control.argtypes = [vp, vp]
    L.rp_close.argtypes = [vp]
    L.rp_open_decompress.restype = vp
    L.rp_open_decompress.argtypes = [vp, vp, C.c_uint8]
    L.rp_decompress_full.restype = C.c_int
    L.rp_decompress_full.argtypes = [vp]
    L.rp_dcodeblock.restype = C.c_int
    L.rp_dcodeblock.argtypes = [vp, C.c_int, u64, vp, vp]
    L.rp_reset_gain_lut.argtypes = []
    L.rp_get_gain_lut.argtypes = [vp]
    L.rp_set_threads.argtypes = [C.c_int]
    L.rp_max_threads.restype = C.c_int
    L.rp_prec_bytes.restype = C.c_int
    _libs[precision] = L
    return L


def _u8arr(v):
    if v is None:
        return None
    a = (C.c_uint8 * 4)(*[int(x) for x in v])
    return a


@dataclass
class Codeblock:
    geom: np.ndarray      # X0,Y0,Z0,TS0,X1,Y1,Z1,TS1,highband,Kmax
    K: int
    Kmsbs: int
    Z: int
    L: np.ndarray         # Z lengths
    S: np.ndarray         # Z+1 log slopes
    data: bytes
    subband: np.ndarray   # effective step, step, dwt gain


class RefCompressor:
    """One reference compression, optionally run stage by stage."""

    def __init__(self, field, *, precision="double", decomp=None, cb=None, qm=-1, erres=False,
                 rate="2", n_par=None, precincts=None, kernels=None, tiles=None):
        self.L = load(precision)
        self.precision = precision
        f = np.ascontiguousarray(field)
        if f.dtype not in (np.float32, np.float64):
            raise TypeError("field must be float32 or float64")
        self.field = f
        if n_par is None:
            n_par = 1
            dims = f.shape
        else:
            dims = f.shape[1:]
        dims = tuple(reversed(dims))          # x fastest
        dims = dims + (1,) * (4 - len(dims))
        self.dims = dims
        self.n_par = n_par
        self.h = None
        self.out = np.zeros(f.nbytes + (1 << 16), dtype=np.uint8)
        rate_b = None if rate is None else rate.encode()
        self.L.rp_set_precincts(_u8arr(precincts))
        self.L.rp_set_kernels(_u8arr(kernels))   # (x, y, z, t): 0 CDF 9/7, 1 LeGall 5/3
        # tile sizes (x, y, z, t)
        tl = None if tiles is None else (C.c_uint64 * 4)(*[int(v) for v in tiles])
        self.L.rp_set_tiles(tl)
        try:
            self.h = self._open(f, dims, n_par, decomp, cb, qm, erres, rate_b)
        finally:
            self.L.rp_set_precincts(None)
            self.L.rp_set_kernels(None)
            self.L.rp_set_tiles(None)
        if not self.h:
            raise RuntimeError("reference rejected the configuration")

    def _open(self, f, dims, n_par, decomp, cb, qm, erres, rate_b):
        return self.L.rp_open_compress(
            f.ctypes.data, dims[0], dims[1], dims[2], dims[3], n_par,
            8 if f.dtype == np.float64 else 4, _u8arr(decomp), _u8arr(cb), int(qm), int(erres),
            rate_b, self.out.ctypes.data)

    def close(self):
        if self.h:
            self.L.rp_close(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def compress(self):
        n = self.L.rp_compress_full(self.h)
        return bytes(self.out[:n])

    # ---- stages -------------------------------------------------------------------------
    def normalize(self, p=0):
        assert self.L.rp_stage_normalize(self.h, p) == 0

    def dwt(self, p=0):
        assert self.L.rp_stage_dwt(self.h, p) == 0

    def t1(self, p=0):
        assert self.L.rp_stage_t1(self.h, p) == 0

    def t2(self):
        assert self.L.rp_stage_t2(self.h) == 0

    def assemble(self):
        n = self.L.rp_stage_assemble(self.h)
        return bytes(self.out[:n])

    def work(self):
        n = int(np.prod(self.dims))
        dt = np.float64 if self.precision == "double" else np.float32
        buf = np.zeros(n, dtype=dt)
        self.L.rp_copy_work(self.h, buf.ctypes.data)
        return buf

    def stats(self, p=0):
        out = np.zeros(4)
        self.L.rp_param_stats(self.h, p, out.ctypes.data)
        return out

    def num_codeblocks(self, p=0):
        return int(self.L.rp_num_codeblocks(self.h, p))

    def codeblock(self, c, p=0, with_data=True):
        mp = MAX_PASSES[self.precision]
        geom = np.zeros(10, dtype=np.uint64)
        meta = np.zeros(3, dtype=np.int64)
        Ls = np.zeros(mp, dtype=np.uint64)
        Ss = np.zeros(mp + 1, dtype=np.uint16)
        cap = 1 << 24
        data = np.zeros(cap if with_data else 1, dtype=np.uint8)
        rc = self.L.rp_codeblock(self.h, p, c, geom.ctypes.data, meta.ctypes.data, Ls.ctypes.data,
                                 Ss.ctypes.data, data.ctypes.data if with_data else None,
                                 cap if with_data else 0)
        assert rc == 0, rc
        K, Kmsbs, Z = (int(v) for v in meta)
        sb = np.zeros(3)
        self.L.rp_codeblock_subband(self.h, p, c, sb.ctypes.data)
        nbytes = int(Ls[Z - 1]) if Z > 0 else 0
        return Codeblock(geom, K, Kmsbs, Z, Ls[:Z].copy(), Ss[:Z + 1].copy(),
                         bytes(data[:nbytes]) if with_data else b"", sb)

    def num_tiles(self):
        return int(self.L.rp_num_tiles(self.h))

    def select_tile(self, t):
        """stage functions and per-codeblock queries work on tile t from here on"""
        assert self.L.rp_select_tile(self.h, t) == 0

    def tile_slopes(self):
        out = np.zeros(2, dtype=np.uint16)
        self.L.rp_tile_slopes(self.h, out.ctypes.data)
        return int(out[0]), int(out[1])

    def control(self):
        out = np.zeros(29, dtype=np.uint64)
        self.L.rp_codec_control(self.h, out.ctypes.data)
        return out


class RefDecompressor:
    def __init__(self, codestream, out_shape, out_dtype, *, precision="double", layer=0):
        self.L = load(precision)
        self.precision = precision
        self.h = None
        self.cs = np.frombuffer(bytes(codestream), dtype=np.uint8).copy()
        self.out = np.zeros(out_shape, dtype=out_dtype)
        self.h = self.L.rp_open_decompress(self.cs.ctypes.data, self.out.ctypes.data, layer)
        if not self.h:
            raise RuntimeError("reference rejected the codestream")

    def close(self):
        if self.h:
            self.L.rp_close(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def decompress(self):
        assert self.L.rp_decompress_full(self.h) == 0
        return self.out

    # stage by stage: t1 (decode + dequantise into a zeroed buffer), idwt, finish (denormalise
    # and write the output)
    def t1(self, p=0):
        assert self.L.rp_dstage_t1(self.h, p) == 0

    def idwt(self, p=0):
        assert self.L.rp_dstage_idwt(self.h, p) == 0

    def finish(self, p=0):
        assert self.L.rp_dstage_finish(self.h, p) == 0
        return self.out

    def work(self):
        dt = np.float64 if self.L.rp_prec_bytes() == 8 else np.float32
        n = int(np.prod(self.out.shape))
        buf = np.zeros(n, dtype=dt)
        self.L.rp_copy_work(self.h, buf.ctypes.data)
        return buf

    def set_work(self, buf):
        """replaces the start of the working buffer with ``buf`` (values of the codec's
        precision), e.g. a transform computed elsewhere, before finish()"""
        b = np.ascontiguousarray(buf)
        assert self.L.rp_set_work(self.h, b.ctypes.data, b.size) == 0

    def num_tiles(self):
        return int(self.L.rp_num_tiles(self.h))

    def select_tile(self, t):
        """codeblock queries and stages work on tile t from here on"""
        assert self.L.rp_select_tile(self.h, t) == 0

    def num_codeblocks(self, p=0):
        return int(self.L.rp_num_codeblocks(self.h, p))

    def codeblock_lengths(self, c, p=0):
        """(K, Kmsbs, Z) and the truncation lengths of codeblock c as parsed"""
        meta = np.zeros(3, dtype=np.int64)
        Ls = np.zeros(MAX_PASSES[self.precision], dtype=np.uint64)
        assert self.L.rp_dcodeblock(self.h, p, c, meta.ctypes.data, Ls.ctypes.data) == 0
        return tuple(int(v) for v in meta), Ls

    def codeblock(self, c, p=0):
        """(K, Kmsbs, Z) of codeblock c as parsed from the codestream."""
        meta = np.zeros(3, dtype=np.int64)
        assert self.L.rp_dcodeblock(self.h, p, c, meta.ctypes.data, None) == 0
        return tuple(int(v) for v in meta)


def reset_gain_lut(precision="double"):
    load(precision).rp_reset_gain_lut()


def gain_lut(precision="double"):
    out = np.zeros(30)
    load(precision).rp_get_gain_lut(out.ctypes.data)
    return out.reshape(3, 10)


def set_threads(n, precision="double"):
    load(precision).rp_set_threads(int(n))


def compress(field, **kw):
    rc = RefCompressor(field, **kw)
    try:
        return rc.compress()
    finally:
        rc.close()


def decompress(codestream, shape, dtype, precision="double", layer=0):
    rd = RefDecompressor(codestream, shape, dtype, precision=precision, layer=layer)
    try:
        return rd.decompress().copy()
    finally:
        rd.close()
