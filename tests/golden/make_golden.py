"""Generates the golden fixtures of this directory from the reference library.

    python tests/golden/make_golden.py        (needs oracle/_ref: make -C oracle ref)

Each case stores its input field (so that no fixture depends on the host's libm) and what the
reference library, compiled from its own sources, produces for it stage by stage:

  normalised field and wavelet coefficients (SHA-256 of their bits), min/max/alpha/beta,
  every codeblock's geometry, subband parameters, K, Z, truncation lengths, log slopes and
  coded bytes, the codestream, and on the decoder side every codeblock's parsed (K, Z), the
  dequantised coefficients, the inverse transform and the decompressed field (SHA-256).

The reference's subband-gain table is process-global and grows with every codec set up
(dwt.c:808-1066); it is reset before every case so that each fixture stands alone.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from bigwhoop_b200 import fields  # noqa: E402

CASES = {
    # name: (shape, field dtype, precision, decomp, codeblocks, rate, qm, erres, generator)
    "d_3lv_cb16_2bpv": ((20, 24, 32), "f8", "double", (3, 3, 3, 0), (4, 4, 4, 0), "2", None, False, "spectral"),
    "d_odd_4layers": ((13, 17, 23), "f8", "double", (2, 2, 2, 0), (3, 3, 3, 0), "0.5,1,2,4", None, False, "spectral"),
    "s_single_2layers": ((16, 18, 20), "f4", "single", (2, 2, 2, 0), (3, 3, 2, 0), "1,4", None, False, "spectral"),
    "d_4d_erres": ((4, 8, 10, 12), "f8", "double", (1, 1, 1, 1), (3, 3, 3, 1), "2,8", None, True, "spectral"),
    "d_f32in_qm40": ((12, 14, 16), "f4", "double", (2, 2, 2, 0), (3, 3, 3, 0), "3", 40, False, "spectral"),
    "d_shock_quarter": ((24, 24, 24), "f8", "double", (2, 2, 2, 0), (4, 4, 4, 0), "0.25,1", None, False, "shock"),
    "s_high_rate": ((10, 12, 14), "f4", "single", (1, 2, 2, 0), (2, 3, 3, 0), "24", None, False, "spectral"),
}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def make_field(name, shape, dtype, gen):
    seed = 100 + sorted(CASES).index(name)
    if gen == "shock":
        return fields.shock_field(shape, seed).astype(dtype)
    return fields.spectral_field(shape, seed).astype(dtype)


def generate(name):
    from oracle import ref
    shape, dtype, precision, decomp, cb, rate, qm, erres, gen = CASES[name]
    f = make_field(name, shape, np.dtype(dtype), gen)
    mp = ref.MAX_PASSES[precision]
    ref.reset_gain_lut(precision)
    rc = ref.RefCompressor(f, precision=precision, decomp=decomp, cb=cb, rate=rate,
                           qm=-1 if qm is None else qm, erres=erres)
    try:
        rc.normalize()
        normalized = rc.work()
        stats = rc.stats()
        rc.dwt()
        transformed = rc.work()
        rc.t1()
        ncb = rc.num_codeblocks()
        geom = np.zeros((ncb, 10), np.uint64)
        sub = np.zeros((ncb, 3))
        K = np.zeros(ncb, np.uint8)
        Z = np.zeros(ncb, np.uint8)
        Ls = np.zeros((ncb, mp), np.uint64)
        Ss = np.zeros((ncb, mp + 1), np.uint16)
        offs = np.zeros(ncb + 1, np.uint64)
        data = bytearray()
        for c in range(ncb):
            cbk = rc.codeblock(c)
            geom[c] = cbk.geom
            sub[c] = cbk.subband
            K[c], Z[c] = cbk.K, cbk.Z
            Ls[c, :cbk.Z] = cbk.L
            Ss[c, :cbk.Z + 1] = cbk.S
            offs[c] = len(data)
            data += cbk.data
        offs[ncb] = len(data)
        rc.t2()
        cs = rc.assemble()
    finally:
        rc.close()
    ref.reset_gain_lut(precision)
    rd = ref.RefDecompressor(cs, f.shape, f.dtype, precision=precision)
    try:
        rd.t1()
        dequant = rd.work()
        dK = np.zeros(ncb, np.uint8)
        dZ = np.zeros(ncb, np.uint8)
        for c in range(ncb):
            k, _, z = rd.codeblock(c)
            dK[c], dZ[c] = k, z
        rd.idwt()
        recon = rd.work()
        out = rd.finish().copy()
    finally:
        rd.close()
    arrays = dict(field=f, stats=stats, geom=geom, subband=sub, K=K, Z=Z, L=Ls, S=Ss,
                  cb_offsets=offs, cb_data=np.frombuffer(bytes(data), np.uint8),
                  codestream=np.frombuffer(cs, np.uint8), dK=dK, dZ=dZ)
    meta = dict(shape=list(shape), dtype=dtype, precision=precision, decomp=list(decomp),
                codeblocks=list(cb), rate=rate, qm=qm, erres=erres, generator=gen,
                normalized_sha=sha(normalized), transformed_sha=sha(transformed),
                dequantized_sha=sha(dequant), reconstructed_sha=sha(recon), output_sha=sha(out),
                codestream_sha=hashlib.sha256(cs).hexdigest(), codeblocks_n=int(ncb))
    return arrays, meta


def main():
    index = {}
    for name in CASES:
        arrays, meta = generate(name)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        index[name] = meta
        print(name, meta["codeblocks_n"], "codeblocks,", arrays["codestream"].size, "bytes")
    with open(os.path.join(HERE, "cases.json"), "w") as fh:
        json.dump(index, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
