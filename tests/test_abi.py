"""The drop-in boundary, checked without a GPU: the libraries load, export every function that
include/*.h declares, lay out the caller-visible structs exactly like the reference's types.h,
and behave like the reference on host-only calls (setters, header probe, bad arguments).
"""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, need_ref
from bigwhoop_b200 import bwc

INCLUDE = os.path.join(ROOT, "include")
# the reference's private headers, copied there by the oracle's recipe (make -C oracle)
REF_INC = os.path.join(ROOT, "oracle", "_ref", "include")


def _declared_functions(header):
    text = open(os.path.join(INCLUDE, header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    text = re.sub(r"typedef[^;]*;", "", text)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", text)
    return sorted(set(n for n in names if n not in ("if", "while", "sizeof")))


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("header", ["bwc.h", "bwc_b200.h"])
def test_library_exports_every_declared_function(precision, header):
    lib = C.CDLL(bwc.lib_path(precision))
    names = _declared_functions(header)
    assert len(names) >= (22 if header == "bwc.h" else 10), names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_precision_builds_differ():
    d = C.CDLL(bwc.lib_path("double"))
    s = C.CDLL(bwc.lib_path("single"))
    assert d.bwc_b200_precision_bits() == 63 and s.bwc_b200_precision_bits() == 31


LAYOUT_FIELDS = {
    "bwc_span": ["size", "position", "access", "memory"],
    "bwc_gl_inf": ["nX", "nY", "nZ", "nTS", "nPar", "data_prec", "codec_prec"],
    "bwc_stream": ["codestream.aux", "codestream.com", "inp", "out", "mode"],
    "bwc_gl_ctrl": ["CSsgc", "error_resilience", "tileSizeX", "tileSizeY", "tileSizeZ",
                    "tileSizeTS", "nTiles", "precSizeX", "precSizeY", "precSizeZ", "precSizeTS",
                    "cbX", "cbY", "cbZ", "cbTS", "KernelX", "KernelY", "KernelZ", "KernelTS",
                    "decompX", "decompY", "decompZ", "decompTS", "nDecomp", "qt_exponent",
                    "qt_mantissa", "Qm", "bitrate", "nLayers", "useLayer", "guard_bits",
                    "headerSize", "codestreamSize", "quantization_style", "progression"],
    "bwc_header": ["info", "control", "aux", "com"],
    "bwc_codec": ["info", "control", "tile", "mode"],
}


def _layout_program(include_line):
    lines = ["#include <stdio.h>", "#include <stddef.h>", include_line, "int main(void) {"]
    for t, fs in LAYOUT_FIELDS.items():
        lines.append(f'  printf("{t} %zu\\n", sizeof({t}));')
        for f in fs:
            lines.append(f'  printf("{t}.{f} %zu\\n", offsetof({t}, {f}));')
    lines.append("  return 0; }")
    return "\n".join(lines)


def _run_layout(include_line, flags):
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(src, "w").write(_layout_program(include_line))
        subprocess.run(["gcc", "-std=gnu11", src, "-o", exe] + flags, check=True,
                       capture_output=True)
        return subprocess.run([exe], check=True, capture_output=True, text=True).stdout


@pytest.mark.parametrize("precision", ["double", "single"])
def test_struct_layout_matches_reference_types(precision):
    if not os.path.exists(os.path.join(REF_INC, "types.h")):
        pytest.skip("reference headers not present")
    define = "-DBWC_DOUBLE_PRECISION" if precision == "double" else "-DBWC_SINGLE_PRECISION"
    ours = _run_layout('#include "bwc.h"', ["-I", INCLUDE] +
                       (["-DBWC_SINGLE_PRECISION"] if precision == "single" else []))
    theirs = _run_layout('#include "types.h"', ["-I", REF_INC, define])
    assert ours == theirs


# ---- host-only behaviour, compared with the reference library -----------------------------------

def _lib(precision="double"):
    return bwc.load(precision)


def _codec_fields(lib, codec):
    """info and control of a codec as plain values (the bitrate pointer left out)."""
    cd = C.cast(codec, C.POINTER(bwc.bwc_codec)).contents
    out = {}
    for part in ("info", "control"):
        s = getattr(cd, part)
        for name, _ in s._fields_:
            if name != "bitrate":
                out[f"{part}.{name}"] = getattr(s, name)
    return out


SETTER_SEQUENCES = [
    [],
    [("bwc_set_codeblocks", 5, 5, 4, 0), ("bwc_set_decomp", 4, 4, 4, 0)],
    [("bwc_set_codeblocks", 16, 4, 4, 0)],          # a codeblock exponent above the limit
    [("bwc_set_codeblocks", 12, 12, 0, 0)],         # exponents summing above the limit
    [("bwc_set_decomp", 70, 1, 1, 0)],              # more levels than allowed
    [("bwc_set_decomp", 3, 2, 1, 0), ("bwc_set_qm", 40)],
    [("bwc_set_precincts", 3, 3, 3, 0), ("bwc_set_codeblocks", 2, 2, 2, 0)],
    [("bwc_set_precincts", 1, 1, 1, 0)],
    [("bwc_set_qm", 70)],
    [("bwc_set_error_resilience",)],
]


@pytest.mark.parametrize("dims", [(64, 64, 64, 1), (33, 1, 7, 1), (16, 16, 16, 9), (1, 1, 1, 1)])
@pytest.mark.parametrize("seq", range(len(SETTER_SEQUENCES)))
def test_setters_match_reference(dims, seq):
    """The same setter calls leave the same info/control values (including rejected inputs,
    which the reference answers with a warning and its defaults)."""
    ref = need_ref("double")
    # private handles: the argument types set here must not leak into the shared bindings
    Lr = C.CDLL(ref.lib_path("double"))
    Lm = C.CDLL(bwc.lib_path("double"))
    for L in (Lr, Lm):
        L.bwc_alloc_coder.restype = C.c_void_p
        L.bwc_alloc_coder.argtypes = [C.c_uint64] * 4 + [C.c_uint8, C.c_int]
    results = []
    for L in (Lr, Lm):
        c = L.bwc_alloc_coder(*dims, 1, 8)
        try:
            for call in SETTER_SEQUENCES[seq]:
                fn = getattr(L, call[0])
                fn.restype = None
                fn.argtypes = [C.c_void_p] + [C.c_uint8] * (len(call) - 1)
                fn(c, *call[1:])
            results.append(_codec_fields(L, c))
        finally:
            L.bwc_free_codec.argtypes = [C.c_void_p]
            L.bwc_free_codec(c)
    assert results[0] == results[1]


def test_open_header_matches_reference_codestream():
    ref = need_ref("double")
    from bigwhoop_b200 import fields
    f = fields.spectral_field((20, 18, 16), 5)
    ref.reset_gain_lut("double")
    cs = ref.compress(f, decomp=(2, 2, 2, 0), cb=(3, 3, 3, 0), rate="0.5,2")
    h = bwc.open_header(cs)
    assert (h["nX"], h["nY"], h["nZ"], h["nTS"], h["nPar"]) == (16, 18, 20, 1, 1)
    assert h["data_prec"] == 8 and h["nLayers"] == 2
    assert h["bitrate"] == [0.5, 2.0]
    assert h["codestreamSize"] == len(cs)


def test_open_header_rejects_garbage():
    L = _lib()
    junk = np.frombuffer(bytes(range(256)) * 4, dtype=np.uint8).copy()
    assert not L.bwc_open_header(junk.ctypes.data)


RATES = [b"abc", b"-1", b"0", b"65", b"64", b"2", b"1,2", b"2,1", b"0.5,,1", b"", b"1 2",
         b"0.1,0.2,0.3,0.4,0.5,0.6,0.7,0.8,0.9,1", b"1e1", b"4,4"]


@pytest.mark.parametrize("rate", RATES)
def test_create_compression_rate_parsing_matches_reference(rate):
    """Return code and parsed layer rates of bwc_create_compression, against the reference."""
    ref = need_ref("double")
    f = np.zeros((8, 8, 8))
    out = np.zeros(1 << 16, np.uint8)
    res = []
    for path in (ref.lib_path("double"), bwc.lib_path("double")):
        L = C.CDLL(path)
        L.bwc_alloc_coder.restype = C.c_void_p
        L.bwc_alloc_coder.argtypes = [C.c_uint64] * 4 + [C.c_uint8, C.c_int]
        L.bwc_init_stream.restype = C.c_void_p
        L.bwc_init_stream.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.bwc_create_compression.restype = C.c_uint8
        L.bwc_create_compression.argtypes = [C.c_void_p, C.c_void_p, C.c_char_p]
        L.bwc_free_codec.argtypes = [C.c_void_p]
        c = L.bwc_alloc_coder(8, 8, 8, 1, 1, 8)
        s = L.bwc_init_stream(f.ctypes.data, out.ctypes.data, bwc.COMP)
        try:
            rc = L.bwc_create_compression(c, s, C.create_string_buffer(rate))
            ctrl = C.cast(c, C.POINTER(bwc.bwc_codec)).contents.control
            layers = [ctrl.bitrate[i] for i in range(ctrl.nLayers)] if rc == 0 else None
            res.append((rc, layers))
        finally:
            L.bwc_free_codec(c)
            C.CDLL(None).free(C.c_void_p(s))
    assert res[0] == res[1]


def test_create_decompression_rejects_truncated_codestream():
    ref = need_ref("double")
    from bigwhoop_b200 import fields
    f = fields.spectral_field((12, 12, 12), 6)
    ref.reset_gain_lut("double")
    cs = ref.compress(f, decomp=(1, 1, 1, 0), cb=(3, 3, 3, 0), rate="4")
    L = _lib()
    for cut in (3, 20, len(cs) // 2):
        buf = np.zeros(len(cs) + 64, np.uint8)
        buf[:cut] = np.frombuffer(cs[:cut], np.uint8)
        out = np.zeros(f.size, np.float64)
        c = L.bwc_alloc_decoder()
        s = L.bwc_init_stream(buf.ctypes.data, out.ctypes.data, bwc.DECOMP)
        try:
            assert L.bwc_create_decompression(c, s, 0) == 1, cut
        finally:
            L.bwc_free_codec(c)
            C.CDLL(None).free(C.c_void_p(s))


@pytest.mark.parametrize("case", ["kernel_haar", "no_quantisation", "kernel_5_3"])
def test_create_compression_accepts_5_3_and_refuses_haar_and_no_quantisation(case):
    """The LeGall 5/3 kernel is accepted; the Haar kernel and bwc_qt_none are refused by
    bwc_create_compression with return code 1 (the default configuration of the same field is
    accepted)."""
    f = np.zeros((16, 16, 16))
    out = np.zeros(1 << 16, np.uint8)
    L = C.CDLL(bwc.lib_path("double"))
    L.bwc_alloc_coder.restype = C.c_void_p
    L.bwc_alloc_coder.argtypes = [C.c_uint64] * 4 + [C.c_uint8, C.c_int]
    L.bwc_init_stream.restype = C.c_void_p
    L.bwc_init_stream.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    L.bwc_create_compression.restype = C.c_uint8
    L.bwc_create_compression.argtypes = [C.c_void_p, C.c_void_p, C.c_char_p]
    L.bwc_free_codec.argtypes = [C.c_void_p]
    L.bwc_set_tiles.argtypes = [C.c_void_p] + [C.c_uint64] * 4 + [C.c_int]
    L.set_kernels.argtypes = [C.c_void_p] + [C.c_int] * 4
    L.set_quant_style.argtypes = [C.c_void_p, C.c_int]
    for configure in (False, True):
        c = L.bwc_alloc_coder(16, 16, 16, 1, 1, 8)
        s = L.bwc_init_stream(f.ctypes.data, out.ctypes.data, bwc.COMP)
        try:
            if configure:
                if case == "kernel_5_3":
                    L.set_kernels(c, 1, 1, 1, 1)
                elif case == "kernel_haar":
                    L.set_kernels(c, 2, 2, 2, 2)
                else:
                    L.set_quant_style(c, 0)
            rc = L.bwc_create_compression(c, s, C.create_string_buffer(b"2"))
            refused = configure and case != "kernel_5_3"
            assert rc == (1 if refused else 0), (case, configure)
        finally:
            L.bwc_free_codec(c)
            C.CDLL(None).free(C.c_void_p(s))


@pytest.mark.parametrize("case", ["default", "kernel_5_3", "kernel_haar_in_header"])
def test_create_decompression_checks_the_wavelet_of_the_codestream(case):
    """Reference codestreams made with the 9/7 and the 5/3 kernel are accepted by
    bwc_create_decompression; one whose header names the Haar kernel is refused (return code
    1).  The reference's own bwc_compress crashes (segmentation fault, some runs) with the Haar
    kernel or without quantisation on this input, so the Haar header is made by rewriting the
    kernel byte of the 5/3 codestream's SGC marker."""
    need_ref("double")
    from oracle import ref
    from bigwhoop_b200 import fields
    f = fields.spectral_field((16, 16, 16), 3)
    out = np.zeros(1 << 20, np.uint8)
    R = C.CDLL(ref.lib_path("double"))
    R.bwc_alloc_coder.restype = C.c_void_p
    R.bwc_alloc_coder.argtypes = [C.c_uint64] * 4 + [C.c_uint8, C.c_int]
    R.bwc_init_stream.restype = C.c_void_p
    R.bwc_init_stream.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    R.bwc_create_compression.restype = C.c_uint8
    R.bwc_create_compression.argtypes = [C.c_void_p, C.c_void_p, C.c_char_p]
    R.bwc_compress.restype = C.c_size_t
    R.bwc_compress.argtypes = [C.c_void_p, C.c_void_p]
    R.bwc_free_codec.argtypes = [C.c_void_p]
    R.set_kernels.argtypes = [C.c_void_p] + [C.c_int] * 4
    c = R.bwc_alloc_coder(16, 16, 16, 1, 1, 8)
    s = R.bwc_init_stream(f.ctypes.data, out.ctypes.data, bwc.COMP)
    try:
        if case != "default":
            R.set_kernels(c, 1, 1, 1, 1)
        assert R.bwc_create_compression(c, s, C.create_string_buffer(b"4")) == 0
        n = R.bwc_compress(c, s)
        assert n > 0
    finally:
        R.bwc_free_codec(c)
        C.CDLL(None).free(C.c_void_p(s))
    cs = np.zeros(n + 64, np.uint8)
    cs[:n] = out[:n]
    if case == "kernel_haar_in_header":
        # the kernel byte (x << 6 | y << 4 | z << 2 | t) of the SGC marker: 5/3 everywhere is
        # 0x55; Haar everywhere is 0xAA
        pos = bytes(cs[:256]).find(b"\x55")
        assert pos > 0
        cs[pos] = 0xAA
    L = _lib()
    rec = np.zeros(f.size, np.float64)
    d = L.bwc_alloc_decoder()
    st = L.bwc_init_stream(cs.ctypes.data, rec.ctypes.data, bwc.DECOMP)
    try:
        rc = L.bwc_create_decompression(d, st, 0)
    finally:
        L.bwc_free_codec(d)
        C.CDLL(None).free(C.c_void_p(st))
    assert rc == (1 if case == "kernel_haar_in_header" else 0), case


def test_compress_takes_multi_tile_fields_to_the_device(capfd):
    """A codec of two tiles is set up (its host half is tested against the reference in
    tests/test_host_parity.py) and bwc_compress takes it to the device: with no GPU it fails
    there, naming the CUDA call, and it refuses nothing for the tiling (the tiled codestreams
    are compared with the reference in tests/test_gpu_tiles.py)."""
    f = np.zeros((16, 16, 16))
    out = np.zeros(1 << 16, np.uint8)
    L = C.CDLL(bwc.lib_path("double"))
    L.bwc_alloc_coder.restype = C.c_void_p
    L.bwc_alloc_coder.argtypes = [C.c_uint64] * 4 + [C.c_uint8, C.c_int]
    L.bwc_init_stream.restype = C.c_void_p
    L.bwc_init_stream.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    L.bwc_create_compression.restype = C.c_uint8
    L.bwc_create_compression.argtypes = [C.c_void_p, C.c_void_p, C.c_char_p]
    L.bwc_compress.restype = C.c_size_t
    L.bwc_compress.argtypes = [C.c_void_p, C.c_void_p]
    L.bwc_free_codec.argtypes = [C.c_void_p]
    L.bwc_set_tiles.argtypes = [C.c_void_p] + [C.c_uint64] * 4 + [C.c_int]
    c = L.bwc_alloc_coder(16, 16, 16, 1, 1, 8)
    s = L.bwc_init_stream(f.ctypes.data, out.ctypes.data, bwc.COMP)
    try:
        L.bwc_set_tiles(c, 8, 16, 16, 1, 0)   # bwc_tile_sizeof: two 8 x 16 x 16 tiles
        assert L.bwc_create_compression(c, s, C.create_string_buffer(b"2")) == 0
        capfd.readouterr()
        n = L.bwc_compress(c, s)
        err = capfd.readouterr().err
        assert "tile" not in err
        assert n > 0 or "CUDA failure" in err
    finally:
        L.bwc_free_codec(c)
        C.CDLL(None).free(C.c_void_p(s))
