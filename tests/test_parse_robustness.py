"""Corrupt codestreams through the host-side parser (bwc_open_header and
bwc_create_decompression): every call returns (accepting or refusing the input) instead of
crashing, aborting on an exception or running without end.  The inputs are the reference's own
golden codestreams with bytes flipped, overwritten or cut off, seeded.  Each run goes in a child
process, so that a crash shows as a failed test."""
import os
import subprocess
import sys

import pytest

from conftest import ROOT

CHILD = r'''
import sys, ctypes as C
sys.path.insert(0, ROOT)
import numpy as np
from bigwhoop_b200 import bwc
cs0 = np.load(FIXTURE)["codestream"].astype(np.uint8)
L = bwc.load("double")
rng = np.random.default_rng(SEED)
out = np.zeros(1 << 22, np.uint8)
counts = [0, 0]
for it in range(ITERS):
    cs = cs0.copy()
    kind = it % 4
    if kind == 0:      # flipped bits anywhere
        for _ in range(rng.integers(1, 4)):
            cs[rng.integers(0, len(cs))] ^= np.uint8(1 << rng.integers(0, 8))
    elif kind == 1:    # overwritten bytes in the headers
        for _ in range(rng.integers(1, 3)):
            cs[rng.integers(0, min(len(cs), 200))] = rng.integers(0, 256)
    elif kind == 2:    # cut off
        cs = cs[:rng.integers(1, len(cs))]
    else:              # overwritten bytes in packet headers and bodies
        k = rng.integers(0, len(cs) - 8)
        cs[k:k + 8] = rng.integers(0, 256, 8).astype(np.uint8)
    buf = np.zeros(len(cs) + 64, np.uint8)
    buf[:len(cs)] = cs
    h = L.bwc_open_header(buf.ctypes.data)
    if h:
        L.bwc_close_header(h)
    d = L.bwc_alloc_decoder()
    st = L.bwc_init_stream(buf.ctypes.data, out.ctypes.data, bwc.DECOMP)
    counts[int(L.bwc_create_decompression(d, st, 0) != 0)] += 1
    L.bwc_free_codec(d)
    C.CDLL(None).free(C.c_void_p(st))
print("ok", counts)
'''


@pytest.mark.parametrize("fixture,seed", [("d_odd_4layers", 11), ("d_4d_erres", 12),
                                          ("d_shock_quarter", 13)])
def test_corrupt_codestreams_are_refused_or_parsed(fixture, seed):
    path = os.path.join(ROOT, "tests", "golden", fixture + ".npz")
    code = f"ROOT = {ROOT!r}\nFIXTURE = {path!r}\nSEED = {seed}\nITERS = 400\n" + CHILD
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=240)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.startswith("ok"), r.stdout[-500:]
    accepted, refused = eval(r.stdout.split("ok", 1)[1])
    assert refused > 0 and accepted > 0
