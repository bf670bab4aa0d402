"""GPU parity: the CUDA path, called through the drop-in C API, against the reference library
compiled from its own sources (oracle/_ref).

Every case checks, stage by stage: the normalised field and the wavelet coefficients bit for
bit, each codeblock's tier-1 output (K, Z, truncation lengths, log slopes, coded bytes), the
final codestream byte for byte, and the decompressed field bit for bit.
"""
import numpy as np
import pytest

from conftest import need_ref
from parity import bits, compare_stages, n_bit_diffs
from bigwhoop_b200 import bwc, fields

pytestmark = pytest.mark.gpu

CASES = [
    # id, shape, field dtype, precision, decomp, codeblocks, rate, extra
    ("cfg0_64cube_cb16_2bpv", (64, 64, 64), np.float64, "double", (3, 3, 3, 0), (4, 4, 4, 0), "2", {}),
    ("64cube_defaults_4layers", (64, 64, 64), np.float64, "double", None, None, "0.5,1,2,4", {}),
    ("odd_extents", (33, 47, 61), np.float64, "double", (2, 2, 2, 0), (5, 5, 4, 0), "1,2", {}),
    ("odd_extents_single", (33, 47, 61), np.float32, "single", (2, 2, 2, 0), (5, 5, 4, 0), "1,2", {}),
    ("f32_input_double_codec", (33, 47, 61), np.float32, "double", (2, 2, 2, 0), (5, 5, 4, 0), "0.25", {}),
    ("4d", (8, 20, 24, 30), np.float64, "double", (2, 2, 2, 1), (3, 3, 3, 1), "0.25,8", {}),
    ("4d_single", (6, 12, 16, 18), np.float32, "single", (1, 2, 2, 1), (3, 3, 3, 1), "1,4", {}),
    ("uneven_decomp", (40, 17, 90), np.float64, "double", (3, 2, 4, 0), (4, 3, 5, 0), "4,0.5", {}),
    ("1d_line", (1, 1, 300), np.float64, "double", (4, 0, 0, 0), (6, 0, 0, 0), "2", {}),
    ("qm40", (32, 32, 32), np.float64, "double", (3, 3, 3, 0), (4, 4, 4, 0), "1,3", {"qm": 40}),
    ("erres", (32, 32, 32), np.float64, "double", (3, 3, 3, 0), (4, 4, 4, 0), "1,3", {"erres": True}),
    ("high_rate", (24, 24, 24), np.float64, "double", (2, 2, 2, 0), (3, 3, 3, 0), "32", {}),
    ("high_rate_single", (24, 24, 24), np.float32, "single", (2, 2, 2, 0), (3, 3, 3, 0), "16", {}),
    ("tiny", (3, 5, 7), np.float64, "double", (1, 1, 1, 0), (2, 2, 2, 0), "2", {}),
    # 64 x 64 x 8 codeblocks (8192 stripe columns): the wide modelling kernel
    ("wide_codeblocks", (32, 128, 128), np.float64, "double", (2, 2, 2, 0), (6, 6, 3, 0), "1,2", {}),
    ("wide_codeblocks_single", (16, 128, 160), np.float32, "single", (1, 1, 1, 0), (6, 6, 3, 0), "4", {}),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_stage_and_codestream_parity(gpu, case):
    _, shape, dtype, precision, decomp, cb, rate, extra = case
    ref = need_ref(precision)
    f = fields.spectral_field(shape, 11).astype(dtype)
    rep, cs, cs_ref = compare_stages(f, ref, precision=precision, decomp=decomp, cb=cb, rate=rate,
                                     **extra)
    assert rep == dict(normalized=0, transformed=0, codeblocks=0, flags=0, codestream=0), rep
    out = bwc.decompress_array(cs, precision)
    out_ref = ref.decompress(cs_ref, f.shape, f.dtype, precision)
    assert n_bit_diffs(out, out_ref) == 0


KERNEL_CASES = [
    # id, shape, precision, decomp, codeblocks, rate, kernels (x, y, z, t): 0 CDF 9/7, 1 LeGall 5/3
    ("legall_3d", (40, 36, 44), "double", (3, 3, 3, 0), (4, 4, 4, 0), "1,4", (1, 1, 1, 1)),
    ("legall_mixed", (33, 47, 61), "double", (2, 3, 2, 0), (5, 5, 4, 0), "0.5,2", (1, 0, 1, 1)),
    ("legall_single", (24, 40, 32), "single", (2, 2, 2, 0), (4, 4, 4, 0), "2,8", (0, 1, 1, 1)),
    ("legall_4d", (6, 20, 16, 24), "double", (2, 2, 2, 1), (3, 3, 3, 1), "1,4", (1, 1, 1, 1)),
    ("legall_line", (1, 1, 300), "double", (4, 0, 0, 0), (6, 0, 0, 0), "2", (1, 1, 1, 1)),
]


@pytest.mark.parametrize("case", KERNEL_CASES, ids=[c[0] for c in KERNEL_CASES])
def test_legall_5_3_parity(gpu, case):
    """The LeGall 5/3 kernel, alone and mixed with 9/7 per axis: stage by stage, codestream and
    decompression against the reference."""
    _, shape, precision, decomp, cb, rate, kernels = case
    ref = need_ref(precision)
    dt = np.float64 if precision == "double" else np.float32
    f = fields.spectral_field(shape, 15).astype(dt)
    rep, cs, cs_ref = compare_stages(f, ref, precision=precision, decomp=decomp, cb=cb, rate=rate,
                                     kernels=kernels)
    assert rep == dict(normalized=0, transformed=0, codeblocks=0, flags=0, codestream=0), rep
    out = bwc.decompress_array(cs, precision)
    out_ref = ref.decompress(cs_ref, f.shape, f.dtype, precision)
    assert n_bit_diffs(out, out_ref) == 0


def test_many_precincts(gpu):
    """16^3 precincts over 8^3 codeblocks: many packets per resolution, stage by stage and the
    decompressed field."""
    ref = need_ref("double")
    f = fields.spectral_field((64, 64, 64), 11)
    rep, cs, cs_ref = compare_stages(f, ref, decomp=(3, 3, 3, 0), cb=(3, 3, 3, 0),
                                     precincts=(4, 4, 4, 0), rate="0.5,2")
    assert rep == dict(normalized=0, transformed=0, codeblocks=0, flags=0, codestream=0), rep
    out = bwc.decompress_array(cs)
    assert n_bit_diffs(out, ref.decompress(cs_ref, f.shape, f.dtype)) == 0


def test_shock_field_with_constant_quarter(gpu):
    """Shock fronts and a constant quarter (all-zero codeblocks: K = 0) at 128^3, 4 layers."""
    ref = need_ref("double")
    f = fields.shock_field((128, 128, 128), 1)
    rep, cs, cs_ref = compare_stages(f, ref, decomp=(4, 4, 4, 0), cb=(5, 5, 4, 0), rate="0.5,1,2,4")
    assert rep == dict(normalized=0, transformed=0, codeblocks=0, flags=0, codestream=0), rep
    out = bwc.decompress_array(cs)
    assert n_bit_diffs(out, ref.decompress(cs_ref, f.shape, f.dtype)) == 0


def test_shock_field_single_precision(gpu):
    ref = need_ref("single")
    f = fields.shock_field((96, 80, 64), 4, dtype=np.float32)
    rep, cs, cs_ref = compare_stages(f, ref, precision="single", decomp=(3, 3, 3, 0),
                                     cb=(5, 5, 4, 0), rate="0.5,2")
    assert rep == dict(normalized=0, transformed=0, codeblocks=0, flags=0, codestream=0), rep
    out = bwc.decompress_array(cs, "single")
    assert n_bit_diffs(out, ref.decompress(cs_ref, f.shape, f.dtype, "single")) == 0


@pytest.mark.parametrize("precision", ["double", "single"])
def test_decompress_each_layer(gpu, precision):
    """bwc_create_decompression(layer): decoding a prefix of the quality layers."""
    ref = need_ref(precision)
    dt = np.float64 if precision == "double" else np.float32
    f = fields.spectral_field((40, 36, 44), 12).astype(dt)
    ref.reset_gain_lut(precision)
    cs = ref.compress(f, precision=precision, decomp=(3, 3, 3, 0), cb=(4, 4, 4, 0), rate="0.25,1,4")
    for layer in range(0, 4):
        ref.reset_gain_lut(precision)
        bwc.reset_gain_state(precision)
        out = bwc.decompress_array(cs, precision, layer=layer)
        out_ref = ref.decompress(cs, f.shape, f.dtype, precision, layer=layer)
        assert n_bit_diffs(out, out_ref) == 0, layer


def test_multi_parameter(gpu):
    """nPar = 2: two fields coded into one codestream."""
    ref = need_ref("double")
    f = np.stack([fields.spectral_field((20, 24, 28), 21), fields.spectral_field((20, 24, 28), 22)])
    kw = dict(decomp=(2, 2, 2, 0), rate="1,2")
    ref.reset_gain_lut("double")
    bwc.reset_gain_state("double")
    cs_ref = ref.compress(f, cb=(4, 4, 4, 0), n_par=2, **kw)
    cs = bwc.compress_array(f, codeblocks=(4, 4, 4, 0), n_par=2, **kw)
    assert cs == cs_ref
    out = bwc.decompress_array(cs)
    assert n_bit_diffs(out, ref.decompress(cs_ref, f.shape, f.dtype)) == 0


def test_device_buffers_match_host_buffers(gpu):
    """Device-resident input and output (CUDA pointers in bwc_stream) give the same bytes."""
    import torch
    f = fields.spectral_field((48, 40, 56), 13)
    kw = dict(decomp=(3, 3, 3, 0), codeblocks=(4, 4, 4, 0), rate="0.5,2")
    bwc.reset_gain_state()
    cs_host = bwc.compress_array(f, **kw)
    t = torch.from_numpy(f).cuda()
    out_dev = torch.zeros(f.nbytes + (1 << 16), dtype=torch.uint8, device="cuda")
    bwc.reset_gain_state()
    c = bwc.Compressor(device_ptr=(t.data_ptr(), f.shape, f.dtype), out=out_dev.data_ptr(), **kw)
    try:
        n = c.compress()
    finally:
        c.close()
    assert bytes(out_dev[:n].cpu().numpy()) == cs_host
    # decompression into device memory
    rec = torch.zeros(f.shape, dtype=torch.float64, device="cuda")
    d = bwc.Decompressor(cs_host, out=rec.data_ptr())
    try:
        d.decompress()
    finally:
        d.close()
    assert n_bit_diffs(rec.cpu().numpy(), bwc.decompress_array(cs_host)) == 0


def test_pageable_host_buffers_match_device_buffers(gpu):
    """Inputs and outputs in pageable host memory large enough to go through the library's
    page-locked staging chunks (32 MiB) in several pieces, the last one partial: the same bytes
    as device-resident and page-locked buffers, both ways."""
    import torch
    f = fields.shock_field((200, 256, 264), 5, device="cuda")   # 103 MiB FP64
    host = f.cpu().numpy()
    kw = dict(decomp=(3, 3, 3, 0), codeblocks=(5, 5, 4, 0), rate="2,28")
    bwc.reset_gain_state()
    cs_host = bwc.compress_array(host, **kw)
    assert len(cs_host) > (36 << 20)   # the codestream too spans two staging chunks
    out_dev = torch.zeros(host.nbytes + (1 << 20), dtype=torch.uint8, device="cuda")
    bwc.reset_gain_state()
    c = bwc.Compressor(device_ptr=(f.data_ptr(), host.shape, host.dtype), out=out_dev.data_ptr(),
                       **kw)
    try:
        n = c.compress()
    finally:
        c.close()
    assert bytes(out_dev[:n].cpu().numpy()) == cs_host
    pinned_in = f.cpu().pin_memory()
    pinned_out = torch.zeros(host.nbytes + (1 << 20), dtype=torch.uint8).pin_memory()
    bwc.reset_gain_state()
    c = bwc.Compressor(device_ptr=(pinned_in.data_ptr(), host.shape, host.dtype),
                       out=pinned_out.data_ptr(), **kw)
    try:
        n = c.compress()
    finally:
        c.close()
    assert bytes(pinned_out[:n].numpy()) == cs_host
    rec_host = bwc.decompress_array(cs_host)
    rec_dev = torch.zeros(host.shape, dtype=torch.float64, device="cuda")
    d = bwc.Decompressor(cs_host, out=rec_dev.data_ptr())
    try:
        d.decompress()
    finally:
        d.close()
    assert n_bit_diffs(rec_dev.cpu().numpy(), rec_host) == 0
    del f, rec_dev, out_dev
    torch.cuda.empty_cache()


def test_repeated_calls_are_deterministic(gpu):
    f = fields.shock_field((64, 72, 80), 3)
    outs = []
    for _ in range(3):
        bwc.reset_gain_state()
        outs.append(bwc.compress_array(f, decomp=(3, 3, 3, 0), codeblocks=(5, 5, 4, 0), rate="1,2"))
    assert outs[0] == outs[1] == outs[2]


def test_gain_state_accumulates_like_reference(gpu):
    """The reference's subband-gain table is process-global and grows on every setup; a second
    compression without a reset must still match the reference's second compression."""
    ref = need_ref("double")
    f = fields.spectral_field((24, 28, 32), 14)
    kw = dict(decomp=(2, 2, 2, 0), rate="2")
    ref.reset_gain_lut("double")
    bwc.reset_gain_state("double")
    r1 = ref.compress(f, cb=(4, 4, 4, 0), **kw)
    r2 = ref.compress(f, cb=(4, 4, 4, 0), **kw)
    m1 = bwc.compress_array(f, codeblocks=(4, 4, 4, 0), **kw)
    m2 = bwc.compress_array(f, codeblocks=(4, 4, 4, 0), **kw)
    assert (m1, m2) == (r1, r2)


def test_constant_field(gpu):
    """A constant field: every codeblock is empty."""
    ref = need_ref("double")
    f = np.full((16, 16, 16), 3.25)
    kw = dict(decomp=(2, 2, 2, 0), rate="2")
    ref.reset_gain_lut("double")
    bwc.reset_gain_state("double")
    cs_ref = ref.compress(f, cb=(3, 3, 3, 0), **kw)
    cs = bwc.compress_array(f, codeblocks=(3, 3, 3, 0), **kw)
    assert cs == cs_ref
    assert n_bit_diffs(bwc.decompress_array(cs), ref.decompress(cs_ref, f.shape, f.dtype)) == 0


def test_full_size_round_trip_properties(gpu):
    """512^3 FP32 shock field (0.5 GiB) through the single-precision build: determinism, layer
    budgets and reconstruction quality improving with every layer."""
    f = fields.shock_field((512, 512, 512), 1, dtype=np.float32, device="cuda")
    import torch
    host = f.cpu().numpy()
    rates = [0.5, 1, 2, 4]
    kw = dict(precision="single", decomp=(4, 4, 4, 0), codeblocks=(5, 5, 4, 0),
              rate=",".join(str(r) for r in rates))
    bwc.reset_gain_state("single")
    cs1 = bwc.compress_array(host, **kw)
    bwc.reset_gain_state("single")
    cs2 = bwc.compress_array(host, **kw)
    assert cs1 == cs2
    n = host.size
    assert len(cs1) <= int(np.ceil(rates[-1] * n / 8)) + 4096
    hdr = bwc.open_header(cs1, "single")
    assert hdr["nLayers"] == 4 and (hdr["nX"], hdr["nY"], hdr["nZ"]) == (512, 512, 512)
    rng = float(host.max() - host.min())
    out = bwc.decompress_array(cs1, "single")
    mse = float(np.mean((out.astype(np.float64) - host) ** 2))
    psnr = 20 * np.log10(rng / (2 * np.sqrt(mse)))
    assert psnr > 60, psnr
    # The reference records the requested layer (codestream.c:1480-1493) but never reads it,
    # so every layer index decodes all layers; so does this library.
    out1 = bwc.decompress_array(cs1, "single", layer=1)
    assert n_bit_diffs(out1, out) == 0
    del f
    torch.cuda.empty_cache()
