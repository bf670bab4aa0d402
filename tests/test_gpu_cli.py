"""The reference's command-line tool (bwccmdl.c with its EAS3 reader eas3.c, unchanged) on this
library: the same two source files compiled against include/bwc.h and linked once with the
reference library (oracle/_ref/cli/bwc-ref) and once with this library (oracle/_ref/cli/bwc-b200),
by `make -C oracle cli`.  Both binaries compress the same EAS3 file with the same options and
must write the same codestream file byte for byte; both decompress the reference's codestream
and must write the same EAS3 file byte for byte.

The EAS3 writer below restates the layout the tool's reader expects (eas3.c:439-760 header,
:981-1140 field): a 20-byte tag holding "EAS3_I8R8", 22 big-endian 64-bit header words
(file type, accuracy, time steps, parameters, the three extents, the attribute, geometry and
user-data modes and sizes), the time-step numbers, the time-step, parameter and axis attribute
names (10 bytes each), then the field as big-endian doubles, x fastest.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

from bigwhoop_b200 import fields

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "oracle", "_ref", "cli")

# header word values as the reader compares them (its mode constants are big-endian 1, 2, ...)
EAS3_TYPE, ACCURACY_DOUBLE, ALL_ATTR, NO_GEOMETRY, NO_USER_DATA = 2, 2, 2, 1, 1
ATTRLEN = 10


def write_eas3(path, f):
    f = np.ascontiguousarray(f, np.float64)
    nt, nz, ny, nx = (1,) * (4 - f.ndim) + f.shape
    words = [EAS3_TYPE, ACCURACY_DOUBLE, nt, 1, nx, ny, nz, ALL_ATTR] + [NO_GEOMETRY] * 5
    words += [0] * 5 + [NO_USER_DATA, 0, 0, 0]
    assert len(words) == 22
    with open(path, "wb") as fp:
        fp.write(b"EAS3_I8R8".ljust(20, b" "))
        fp.write(struct.pack(">22Q", *words))
        fp.write(struct.pack(">%dQ" % nt, *range(nt)))
        fp.write(b"".join(("t%d" % i).encode().ljust(ATTRLEN) for i in range(nt)))
        fp.write(b"u".ljust(ATTRLEN))
        fp.write(b"".join(a.ljust(ATTRLEN) for a in (b"x", b"y", b"z")))
        fp.write(f.astype(">f8").tobytes())


def _tools():
    tools = {k: os.path.join(CLI, "bwc-" + k) for k in ("ref", "b200")}
    for t in tools.values():
        if not os.path.exists(t):
            pytest.skip("command-line tool not built (make -C oracle cli)")
    return tools


def _run(tool, *args):
    r = subprocess.run([tool, *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (tool, args, r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


CASES = [
    # id, field shape (z, y, x) or (t, z, y, x), options of the tool
    ("defaults_2_layers", (48, 40, 56), ["-b", "1,4"]),
    ("levels_codeblocks_qm_erres", (40, 36, 44), ["-b", "2", "-d", "3", "-c", "4", "-m", "40", "-e"]),
    ("tiles", (48, 40, 56), ["-b", "0.5,2", "-t", "32", "-d", "2", "-c", "4"]),
    ("4d", (8, 20, 24, 30), ["-b", "0.5,4", "-d", "2,2,2,1", "-c", "3"]),
    ("compression_ratio", (48, 40, 56), ["-r", "20"]),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_cli_on_this_library_writes_the_reference_files(gpu, tmp_path, case):
    _, shape, opts = case
    tools = _tools()
    f = fields.spectral_field(shape, 17)
    src = str(tmp_path / "field.eas")
    write_eas3(src, f)
    cs = {}
    for k, tool in tools.items():
        out = str(tmp_path / ("field_%s.bwc" % k))
        _run(tool, "-C", src, "-O", out, *opts)
        cs[k] = open(out, "rb").read()
    assert len(cs["b200"]) == len(cs["ref"])
    assert cs["b200"] == cs["ref"]
    rec = {}
    for k, tool in tools.items():
        out = str(tmp_path / ("rec_%s.eas" % k))
        _run(tool, "-D", str(tmp_path / "field_ref.bwc"), "-O", out)
        rec[k] = open(out, "rb").read()
    assert rec["b200"] == rec["ref"]
    # the analysis mode (decompression and PSNR against the input) on this library
    report = _run(tools["b200"], "-A", str(tmp_path / "field_ref.bwc"), "-R", src)
    assert "Peak Signal-to-Noise Ratio" in report
