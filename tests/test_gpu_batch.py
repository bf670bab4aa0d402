"""Batched compression (bwc_b200_compress_batch) against one bwc_compress call per field.

Fields of uneven shapes, input dtypes, decomposition depths, rates and error-resilience
settings are compressed once field by field and once as a batch; every codestream must be
byte-identical.  Codecs are set up in the same order both times, because the reference's
process-wide subband-gain table (which each set-up extends) enters the step sizes.
"""
import numpy as np
import pytest

from bigwhoop_b200 import bwc, fields

pytestmark = pytest.mark.gpu

SPECS = [
    # shape, dtype, decomp, codeblocks, rate, erres
    ((33, 47, 61), np.float64, (2, 2, 2, 0), (5, 5, 4, 0), "1,2", False),
    ((40, 36, 44), np.float32, (3, 3, 3, 0), (5, 5, 4, 0), "0.25", False),
    ((17, 70, 35), np.float64, (2, 3, 2, 0), (4, 4, 4, 0), "4", True),
    ((64, 64, 64), np.float32, (4, 4, 4, 0), (5, 5, 4, 0), "0.5,1,2,4", False),
    ((5, 12, 14, 16), np.float64, (1, 1, 1, 1), (3, 3, 3, 1), "2", False),
    ((12, 13, 14), np.float64, (1, 1, 1, 0), (3, 3, 3, 0), "8", False),
]


def _field(i, spec):
    shape, dtype = spec[0], spec[1]
    if len(shape) == 4:
        return np.stack([fields.spectral_field(shape[1:], 40 + i * 10 + t) for t in range(shape[0])]).astype(dtype)
    return fields.shock_field(shape, 40 + i).astype(dtype)


def _compressor(f, spec, **kw):
    _, _, decomp, cb, rate, erres = spec
    return bwc.Compressor(f, decomp=decomp, codeblocks=cb, rate=rate, erres=erres, **kw)


@pytest.mark.parametrize("repeat", [1, 2])
def test_batch_equals_per_field_calls(gpu, repeat):
    fs = [_field(i, sp) for i, sp in enumerate(SPECS)]
    bwc.reset_gain_state()
    plain = []
    for f, sp in zip(fs, SPECS):
        c = _compressor(f, sp)
        try:
            plain.append(c.compress())
        finally:
            c.close()
    counts = []
    for _ in range(repeat):
        bwc.reset_gain_state()
        comps = [_compressor(f, sp) for f, sp in zip(fs, SPECS)]
        try:
            batch = bwc.compress_batch(comps)
        finally:
            for c in comps:
                c.close()
        for i, (a, b) in enumerate(zip(plain, batch)):
            assert a == b, i
        t = bwc.batch_timings()
        assert len(t) == 8 and t[5] > 0
        counts.append((t[6], t[7]))
    if repeat == 2:
        # the same batch again replays the captured transform graph
        assert counts[1][0] == counts[0][0] and counts[1][1] == counts[0][1] + 1


def test_batch_with_device_buffers(gpu):
    import torch
    fs = [_field(i, sp) for i, sp in enumerate(SPECS[:3])]
    bwc.reset_gain_state()
    plain = []
    for f, sp in zip(fs, SPECS):
        c = _compressor(f, sp)
        try:
            plain.append(c.compress())
        finally:
            c.close()
    bwc.reset_gain_state()
    dev_in = [torch.from_numpy(f).cuda() for f in fs]
    dev_out = [torch.zeros(f.nbytes + (1 << 16), dtype=torch.uint8, device="cuda") for f in fs]
    comps = [_compressor(None, sp, device_ptr=(t.data_ptr(), f.shape, f.dtype), out=o.data_ptr())
             for f, t, o, sp in zip(fs, dev_in, dev_out, SPECS)]
    try:
        sizes = bwc.compress_batch(comps)
    finally:
        for c in comps:
            c.close()
    for i, (p, n, o) in enumerate(zip(plain, sizes, dev_out)):
        assert bytes(o[:n].cpu().numpy()) == p, i
