"""ctypes binding of the B200 libbwc (include/bwc.h, include/bwc_b200.h).

Mirrors the reference's Python interface (src/interfaces/python/bwc.py: init_stream,
alloc_coder, alloc_decoder, free_codec, set_* setters, create_compression, compress,
create_decompression, decompress) with argument types that match the C prototypes, and adds
array-level helpers:

    cs = compress_array(field, rate="2", decomp=(3, 3, 3, 0), codeblocks=(4, 4, 4, 0))
    out = decompress_array(cs)

`precision` selects the library build: "double" (bwc_float = double, the reference's default
build) or "single".  The libraries are built in-tree by ``python -m bigwhoop_b200.build``; a
missing library raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os
from enum import IntEnum

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MAX_PASSES = {"double": 64 * 3 - 2, "single": 32 * 3 - 2}

_libs = {}


class DWT(IntEnum):
    CDF_9_7 = 0
    LEGALL_5_3 = 1
    HAAR = 2


class PROG(IntEnum):
    LRCP = 0
    RLCP = 1
    RPCL = 2
    PCRL = 3
    CPRL = 4


class QT(IntEnum):
    NONE = 0
    DERIVED = 1


class TILE(IntEnum):
    SIZEOF = 0
    NUMBOF = 1


COMP, DECOMP = 0, 1


def lib_path(precision="double"):
    """The library of one precision build; BWC_B200_LIB_DIR points at another build tree
    (holding double/libbwc.so and single/libbwc.so)."""
    base = os.environ.get("BWC_B200_LIB_DIR") or os.path.join(HERE, "lib")
    return os.path.join(base, precision, "libbwc.so")


class bwc_gl_inf(C.Structure):
    _fields_ = [("nX", C.c_uint64), ("nY", C.c_uint64), ("nZ", C.c_uint64), ("nTS", C.c_uint64),
                ("nPar", C.c_uint8), ("data_prec", C.c_int), ("codec_prec", C.c_int)]


class bwc_gl_ctrl(C.Structure):
    _fields_ = [("CSsgc", C.c_uint16), ("error_resilience", C.c_uint8),
                ("tileSizeX", C.c_uint64), ("tileSizeY", C.c_uint64),
                ("tileSizeZ", C.c_uint64), ("tileSizeTS", C.c_uint64), ("nTiles", C.c_uint64),
                ("precSizeX", C.c_uint8), ("precSizeY", C.c_uint8), ("precSizeZ", C.c_uint8),
                ("precSizeTS", C.c_uint8), ("cbX", C.c_uint8), ("cbY", C.c_uint8),
                ("cbZ", C.c_uint8), ("cbTS", C.c_uint8), ("KernelX", C.c_int),
                ("KernelY", C.c_int), ("KernelZ", C.c_int), ("KernelTS", C.c_int),
                ("decompX", C.c_uint8), ("decompY", C.c_uint8), ("decompZ", C.c_uint8),
                ("decompTS", C.c_uint8), ("nDecomp", C.c_uint8), ("qt_exponent", C.c_uint32),
                ("qt_mantissa", C.c_uint32), ("Qm", C.c_uint8), ("bitrate", C.POINTER(C.c_float)),
                ("nLayers", C.c_uint8), ("useLayer", C.c_uint8), ("guard_bits", C.c_uint8),
                ("headerSize", C.c_uint64), ("codestreamSize", C.c_uint64),
                ("quantization_style", C.c_int), ("progression", C.c_int)]


class bwc_span(C.Structure):
    _fields_ = [("size", C.c_uint64), ("position", C.c_uint64),
                ("access", C.c_void_p), ("memory", C.c_void_p)]


class bwc_header(C.Structure):
    _fields_ = [("info", bwc_gl_inf), ("control", bwc_gl_ctrl), ("aux", bwc_span),
                ("com", bwc_span)]


class bwc_codec(C.Structure):
    _fields_ = [("info", bwc_gl_inf), ("control", bwc_gl_ctrl), ("tile", C.c_void_p),
                ("mode", C.c_int)]


def _stage_dump_type(precision):
    fl = C.c_double if precision == "double" else C.c_float

    class bwc_b200_stage_dump(C.Structure):
        _fields_ = [("normalized", C.POINTER(fl)), ("transformed", C.POINTER(fl)),
                    ("K", C.c_void_p), ("Z", C.c_void_p), ("L", C.c_void_p), ("S", C.c_void_p),
                    ("bytes", C.c_void_p), ("bytes_cap", C.c_uint64),
                    ("byte_offsets", C.c_void_p), ("stats", C.POINTER(fl)), ("flags", C.c_void_p)]

    class bwc_b200_decode_dump(C.Structure):
        _fields_ = [("dequantized", C.POINTER(fl)), ("reconstructed", C.POINTER(fl))]

    return bwc_b200_stage_dump, bwc_b200_decode_dump


def load(precision="double"):
    if precision in _libs:
        return _libs[precision]
    path = lib_path(precision)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (python -m bigwhoop_b200.build)")
    L = C.CDLL(path, mode=C.RTLD_LOCAL)
    vp, u8, u64 = C.c_void_p, C.c_uint8, C.c_uint64
    cp = C.POINTER(bwc_codec)
    sig = {
        "bwc_init_stream": (vp, [vp, vp, C.c_int]),
        "bwc_set_com": (C.c_uint8, [vp, C.c_char_p, C.c_uint16]),
        "bwc_set_aux": (C.c_uint8, [vp, C.c_char_p, C.c_uint32]),
        "bwc_alloc_coder": (cp, [u64, u64, u64, u64, u8, C.c_int]),
        "bwc_alloc_decoder": (cp, []),
        "bwc_free_codec": (None, [cp]),
        "bwc_set_error_resilience": (None, [cp]),
        "set_quant_style": (None, [cp, C.c_int]),
        "set_quant_step_size": (None, [cp, C.c_double]),
        "set_progression": (None, [cp, C.c_int]),
        "set_kernels": (None, [cp, C.c_int, C.c_int, C.c_int, C.c_int]),
        "bwc_set_decomp": (None, [cp, u8, u8, u8, u8]),
        "bwc_set_precincts": (None, [cp, u8, u8, u8, u8]),
        "bwc_set_codeblocks": (None, [cp, u8, u8, u8, u8]),
        "bwc_set_qm": (None, [cp, u8]),
        "bwc_set_tiles": (None, [cp, u64, u64, u64, u64, C.c_int]),
        "bwc_open_header": (C.POINTER(bwc_header), [vp]),
        "bwc_close_header": (None, [C.POINTER(bwc_header)]),
        "bwc_create_compression": (C.c_uint8, [cp, vp, C.c_char_p]),
        "bwc_compress": (C.c_size_t, [cp, vp]),
        "bwc_create_decompression": (C.c_uint8, [cp, vp, u8]),
        "bwc_decompress": (C.c_uint8, [cp, vp]),
        "bwc_b200_precision_bits": (C.c_int, []),
        "bwc_b200_reset_gain_state": (None, []),
        "bwc_b200_get_gain_state": (None, [vp]),
        "bwc_b200_num_codeblocks": (u64, [cp, u8]),
        "bwc_b200_set_stage_dump": (None, [cp, vp]),
        "bwc_b200_set_decode_dump": (None, [cp, vp]),
        "bwc_b200_last_timings": (C.c_int, [cp, vp, C.c_int]),
        "bwc_b200_codeblock_geometry": (C.c_int, [cp, u8, u64, vp]),
        "bwc_b200_subband_steps": (C.c_int, [cp, u8, u64, vp]),
        "bwc_b200_parsed_codeblock": (C.c_int, [cp, u8, u64, vp, vp]),
        "bwc_b200_assemble_from_tier1": (C.c_size_t, [cp, vp, vp, vp, vp, vp, vp, vp, vp,
                                                      C.c_uint16, C.c_uint16]),
        "bwc_b200_compress_batch": (C.c_uint8, [vp, vp, C.c_uint32, vp]),
        "bwc_b200_last_batch_timings": (C.c_int, [vp, C.c_int]),
        "bwc_b200_set_rate_model": (C.c_int, [vp]),
        "bwc_b200_mq_lanes": (C.c_int, [C.c_uint32]),
        "bwc_b200_set_transform_tuning": (None, [C.c_int, C.c_int]),
        "bwc_b200_rate_features": (C.c_int, [cp, u8, vp]),
        "bwc_b200_rate_stats": (C.c_int, [cp, u8, vp]),
        "bwc_b200_mlp_forward": (C.c_int, [vp, vp, C.c_uint32, vp]),
        "bwc_b200_mlp_gradient": (C.c_int, [vp, vp, vp, C.c_uint32, vp, vp]),
        "bwc_b200_mlp_train": (C.c_int, [vp, vp, vp, C.c_uint32, C.c_uint32, C.c_uint32,
                                         C.c_float, u64, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    if L.bwc_b200_precision_bits() != (63 if precision == "double" else 31):
        raise RuntimeError(f"{path} is not the {precision}-precision build")
    _libs[precision] = L
    return L


# ---- reference-style function interface -----------------------------------------------------
def init_stream(inpbuf, outbuf, mode, precision="double"):
    ip = inpbuf.ctypes.data if hasattr(inpbuf, "ctypes") else inpbuf
    op = outbuf.ctypes.data if hasattr(outbuf, "ctypes") else outbuf
    return load(precision).bwc_init_stream(ip, op, mode)


def alloc_coder(nX, nY, nZ, nTS, nPar, prec, precision="double"):
    return load(precision).bwc_alloc_coder(nX, nY, nZ, nTS, nPar, prec)


def alloc_decoder(precision="double"):
    return load(precision).bwc_alloc_decoder()


def free_codec(codec, precision="double"):
    load(precision).bwc_free_codec(codec)


def set_codeblocks(codec, cbX, cbY, cbZ, cbTS, precision="double"):
    load(precision).bwc_set_codeblocks(codec, cbX, cbY, cbZ, cbTS)


def set_decomp(codec, decompX, decompY, decompZ, decompTS, precision="double"):
    load(precision).bwc_set_decomp(codec, decompX, decompY, decompZ, decompTS)


def set_qm(codec, Qm, precision="double"):
    load(precision).bwc_set_qm(codec, Qm)


def set_tiles(codec, tilesX, tilesY, tilesZ, tilesTS, instr, precision="double"):
    load(precision).bwc_set_tiles(codec, tilesX, tilesY, tilesZ, tilesTS, int(instr))


def set_precincts(codec, pX, pY, pZ, pTS, precision="double"):
    load(precision).bwc_set_precincts(codec, pX, pY, pZ, pTS)


def create_compression(codec, stream, rate_control, precision="double"):
    rc = None if rate_control is None else C.create_string_buffer(rate_control.encode())
    return load(precision).bwc_create_compression(codec, stream, rc)


def compress(codec, stream, precision="double"):
    return load(precision).bwc_compress(codec, stream)


def create_decompression(codec, stream, layer, precision="double"):
    return load(precision).bwc_create_decompression(codec, stream, layer)


def decompress(codec, stream, precision="double"):
    return load(precision).bwc_decompress(codec, stream)


def set_transform_tuning(mode=1, ctas=0, precision="double"):
    """Forward transform path for levels that transform x, y and z: 0 = 3D tile kernel only,
    1 = the bulk-copy z-streaming kernel wherever rows start on 16-byte boundaries, else the
    register z-streaming kernel where it pays (default), 2 = as 1 with the register kernel
    wherever x, y, z >= 8, 3 = the register z-streaming kernel wherever x, y, z >= 8 (never the
    bulk-copy one); ``ctas`` > 0 fixes the streaming kernels' grids.  Coefficients are
    identical."""
    load(precision).bwc_b200_set_transform_tuning(int(mode), int(ctas))


def reset_gain_state(precision="double"):
    load(precision).bwc_b200_reset_gain_state()


def gain_state(precision="double"):
    out = np.zeros(30)
    load(precision).bwc_b200_get_gain_state(out.ctypes.data)
    return out.reshape(3, 10)


# ---- array helpers -----------------------------------------------------------------------------
def field_dims(field, n_par=None):
    """(nX, nY, nZ, nTS) of a C-ordered array whose last axis is x; n_par leading fields."""
    shape = field.shape if n_par is None else field.shape[1:]
    dims = tuple(int(v) for v in reversed(shape))
    return dims + (1,) * (4 - len(dims))


class Compressor:
    """One bwc compression, set up like a libbwc user does; the field may be a numpy array or
    a CUDA device pointer (``device_ptr=(ptr, shape, dtype)``)."""

    def __init__(self, field=None, *, precision="double", rate="2", decomp=None, codeblocks=None,
                 precincts=None, qm=None, erres=False, n_par=None, device_ptr=None,
                 out=None, tiles=None, kernels=None):
        self.L = load(precision)
        self.precision = precision
        if device_ptr is not None:
            ptr, shape, dtype = device_ptr
            dims = tuple(int(v) for v in reversed(shape if n_par is None else shape[1:]))
            dims = dims + (1,) * (4 - len(dims))
            inp = ptr
            nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
            self.field = None
        else:
            self.field = np.ascontiguousarray(field)
            dtype = self.field.dtype
            dims = field_dims(self.field, n_par)
            inp = self.field.ctypes.data
            nbytes = self.field.nbytes
        if np.dtype(dtype) not in (np.float32, np.float64):
            raise TypeError("fields must be float32 or float64")
        self.dims = dims
        prec = 8 if np.dtype(dtype) == np.float64 else 4
        self.codec = self.L.bwc_alloc_coder(dims[0], dims[1], dims[2], dims[3], n_par or 1, prec)
        if not self.codec:
            raise RuntimeError("bwc_alloc_coder failed")
        if erres:
            self.L.bwc_set_error_resilience(self.codec)
        if decomp is not None:
            self.L.bwc_set_decomp(self.codec, *decomp)
        if precincts is not None:
            self.L.bwc_set_precincts(self.codec, *precincts)
        if codeblocks is not None:
            self.L.bwc_set_codeblocks(self.codec, *codeblocks)
        if qm is not None:
            self.L.bwc_set_qm(self.codec, qm)
        if tiles is not None:   # tile sizes (x, y, z, t)
            self.L.bwc_set_tiles(self.codec, *[int(v) for v in tiles], 0)
        if kernels is not None:   # wavelet per axis (x, y, z, t): 0 CDF 9/7, 1 LeGall 5/3
            self.L.set_kernels(self.codec, *[int(v) for v in kernels])
        if out is None:
            # not zero-filled: compress() reads back only the bytes the library wrote
            self.out = np.empty(nbytes + (1 << 16), dtype=np.uint8)
            outp = self.out.ctypes.data
        else:
            self.out = out
            outp = out.ctypes.data if hasattr(out, "ctypes") else out
        self.stream = self.L.bwc_init_stream(inp, outp, COMP)
        self._rate = None if rate is None else C.create_string_buffer(rate.encode())
        if self.L.bwc_create_compression(self.codec, self.stream, self._rate):
            self.close()
            raise RuntimeError("bwc_create_compression failed")

    def num_codeblocks(self, param=0):
        return int(self.L.bwc_b200_num_codeblocks(self.codec, param))

    def compress(self):
        n = self.L.bwc_compress(self.codec, self.stream)
        if n == 0:
            raise RuntimeError("bwc_compress failed")
        if isinstance(self.out, np.ndarray):
            return bytes(self.out[:n])
        return n

    def timings(self):
        out = np.zeros(12)
        k = self.L.bwc_b200_last_timings(self.codec, out.ctypes.data, 12)
        return out[:k]

    def close(self):
        if getattr(self, "codec", None):
            self.L.bwc_free_codec(self.codec)
            self.codec = None
        if getattr(self, "stream", None):
            C.CDLL(None).free(C.c_void_p(self.stream))
            self.stream = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def compress_array(field, **kw):
    c = Compressor(field, **kw)
    try:
        return c.compress()
    finally:
        c.close()


def open_header(codestream, precision="double"):
    L = load(precision)
    buf = np.frombuffer(bytes(codestream), dtype=np.uint8).copy()
    h = L.bwc_open_header(buf.ctypes.data)
    if not h:
        raise RuntimeError("bwc_open_header failed")
    info = h.contents.info
    ctrl = h.contents.control
    res = dict(nX=info.nX, nY=info.nY, nZ=info.nZ, nTS=info.nTS, nPar=info.nPar,
               data_prec=info.data_prec, codec_prec=info.codec_prec, nLayers=ctrl.nLayers,
               bitrate=[ctrl.bitrate[i] for i in range(ctrl.nLayers)],
               codestreamSize=ctrl.codestreamSize)
    L.bwc_close_header(h)
    return res


class Decompressor:
    def __init__(self, codestream, *, precision="double", layer=0, out=None):
        self.L = load(precision)
        self.precision = precision
        self.cs = np.frombuffer(bytes(codestream), dtype=np.uint8).copy()
        hdr = open_header(self.cs, precision)
        self.shape = tuple(int(v) for v in (hdr["nTS"], hdr["nZ"], hdr["nY"], hdr["nX"]))
        if hdr["nPar"] > 1:
            self.shape = (hdr["nPar"],) + self.shape
        self.dtype = np.float64 if hdr["data_prec"] == 8 else np.float32
        # zero-filled: a tiling in time leaves time steps unwritten (the reference writes each
        # tile's time steps from the field's first one)
        self.out = np.zeros(self.shape, dtype=self.dtype) if out is None else out
        self.codec = self.L.bwc_alloc_decoder()
        outp = self.out.ctypes.data if hasattr(self.out, "ctypes") else self.out
        self.stream = self.L.bwc_init_stream(self.cs.ctypes.data, outp, DECOMP)
        if self.L.bwc_create_decompression(self.codec, self.stream, layer):
            self.close()
            raise RuntimeError("bwc_create_decompression failed")

    def decompress(self):
        if self.L.bwc_decompress(self.codec, self.stream):
            raise RuntimeError("bwc_decompress failed")
        return self.out

    def timings(self):
        out = np.zeros(12)
        k = self.L.bwc_b200_last_timings(self.codec, out.ctypes.data, 12)
        return out[:k]

    def close(self):
        if getattr(self, "codec", None):
            self.L.bwc_free_codec(self.codec)
            self.codec = None
        if getattr(self, "stream", None):
            C.CDLL(None).free(C.c_void_p(self.stream))
            self.stream = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def compress_batch(compressors):
    """Compress several prepared `Compressor`s with one bwc_b200_compress_batch call.  All must
    use the same precision build.  Returns a list with each codestream (bytes) when the
    compressor writes to host memory, else its length."""
    if not compressors:
        return []
    prec = compressors[0].precision
    if any(c.precision != prec for c in compressors):
        raise ValueError("a batch runs in one precision build")
    L = load(prec)
    n = len(compressors)
    codecs = (C.c_void_p * n)(*[C.cast(c.codec, C.c_void_p).value for c in compressors])
    streams = (C.c_void_p * n)(*[c.stream for c in compressors])
    sizes = (C.c_size_t * n)()
    if L.bwc_b200_compress_batch(codecs, streams, n, sizes):
        raise RuntimeError("bwc_b200_compress_batch failed")
    out = []
    for c, sz in zip(compressors, sizes):
        out.append(bytes(c.out[:sz]) if isinstance(c.out, np.ndarray) else int(sz))
    return out


def batch_timings(precision="double"):
    """[0] set-up/uploads, [1] transforms, [2] tier-1, [3] tier-2, [4] gather/outputs, [5] call
    (ms); [6] graphs captured and [7] graph launches so far."""
    out = np.zeros(8)
    k = load(precision).bwc_b200_last_batch_timings(out.ctypes.data, 8)
    return out[:k]


def decompress_array(codestream, precision="double", layer=0):
    d = Decompressor(codestream, precision=precision, layer=layer)
    try:
        return d.decompress()
    finally:
        d.close()
