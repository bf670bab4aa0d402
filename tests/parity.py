"""Shared checks for the GPU parity tests: run one configuration through the reference library
(built from its sources under oracle/_ref) and through this library's C API, stage by stage.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from bigwhoop_b200 import bwc


def bits(a):
    a = np.ascontiguousarray(a).reshape(-1)
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


def n_bit_diffs(a, b):
    return int(np.count_nonzero(bits(a) != bits(b)))


@dataclass
class StageDump:
    """Host buffers the library fills during one compression (bwc_b200_stage_dump)."""
    normalized: np.ndarray
    transformed: np.ndarray
    K: np.ndarray
    Z: np.ndarray
    L: np.ndarray
    S: np.ndarray
    data: np.ndarray
    offsets: np.ndarray
    stats: np.ndarray
    flags: np.ndarray
    max_passes: int
    keep: list = field(default_factory=list)

    def codeblock(self, c):
        mp = self.max_passes
        z = int(self.Z[c])
        return dict(K=int(self.K[c]), Z=z, L=self.L[c * mp:c * mp + z].astype(np.uint64),
                    S=self.S[c * (mp + 1):c * (mp + 1) + z + 1].copy(), offset=int(self.offsets[c]))


def attach_stage_dump(comp: bwc.Compressor, ncb: int, max_passes: int) -> StageDump:
    precision = comp.precision
    dt = np.float64 if precision == "double" else np.float32
    n = int(np.prod(comp.dims))
    d = StageDump(normalized=np.zeros(n, dt), transformed=np.zeros(n, dt),
                  K=np.zeros(ncb, np.uint8), Z=np.zeros(ncb, np.uint8),
                  L=np.zeros(ncb * max_passes, np.uint32), S=np.zeros(ncb * (max_passes + 1), np.uint16),
                  data=np.zeros(n * (dt().itemsize + 1) + 4096, np.uint8), offsets=np.zeros(ncb, np.uint64),
                  stats=np.zeros(4, dt), flags=np.zeros(ncb, np.uint32), max_passes=max_passes)
    D, _ = bwc._stage_dump_type(precision)
    fp = C.POINTER(C.c_double if precision == "double" else C.c_float)
    cs = D(d.normalized.ctypes.data_as(fp), d.transformed.ctypes.data_as(fp), d.K.ctypes.data,
           d.Z.ctypes.data, d.L.ctypes.data, d.S.ctypes.data, d.data.ctypes.data, d.data.size,
           d.offsets.ctypes.data, d.stats.ctypes.data_as(fp), d.flags.ctypes.data)
    d.keep.append(cs)
    comp.L.bwc_b200_set_stage_dump(comp.codec, C.byref(cs))
    return d


def compare_stages(f, ref, *, precision="double", decomp=None, cb=None, rate="2", qm=None,
                   erres=False, precincts=None, kernels=None):
    """Compress ``f`` with both libraries, stage by stage.  Returns a dict of mismatch counts
    (all zero on parity) plus both codestreams."""
    mp = ref.MAX_PASSES[precision]
    ref.reset_gain_lut(precision)
    bwc.reset_gain_state(precision)
    rc = ref.RefCompressor(f, precision=precision, decomp=decomp, cb=cb, rate=rate,
                           qm=-1 if qm is None else qm, erres=erres, precincts=precincts,
                           kernels=kernels)
    try:
        rc.normalize()
        a = rc.work()
        rc.dwt()
        b = rc.work()
        rc.t1()
        ncb = rc.num_codeblocks()
        rcb = [rc.codeblock(c) for c in range(ncb)]
        rc.t2()
        cs_ref = rc.assemble()
    finally:
        rc.close()
    mc = bwc.Compressor(f, precision=precision, decomp=decomp, codeblocks=cb, rate=rate, qm=qm,
                        erres=erres, precincts=precincts, kernels=kernels)
    try:
        assert mc.num_codeblocks() == ncb
        dump = attach_stage_dump(mc, ncb, mp)
        cs = mc.compress()
    finally:
        mc.close()
    bad = []
    for c in range(ncb):
        r = rcb[c]
        m = dump.codeblock(c)
        ok = (m["K"] == r.K and m["Z"] == r.Z and np.array_equal(m["L"], r.L)
              and np.array_equal(m["S"], r.S)
              and bytes(dump.data[m["offset"]:m["offset"] + len(r.data)]) == r.data)
        if not ok:
            bad.append(c)
    return dict(normalized=n_bit_diffs(dump.normalized, a), transformed=n_bit_diffs(dump.transformed, b),
                codeblocks=len(bad), flags=int(np.count_nonzero(dump.flags)),
                codestream=int(cs != cs_ref)), cs, cs_ref
