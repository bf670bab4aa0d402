"""The MQ autotuner: a tuned size class is recorded (process-wide and in BWC_B200_TUNE_FILE),
later processes start from the file, and tuning never changes a codestream."""
import hashlib
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SCRIPT = r"""
import hashlib, sys
sys.path.insert(0, %r)
from bigwhoop_b200 import bwc, fields
f = fields.shock_field((64, 96, 160), 7)
bwc.reset_gain_state()
c = bwc.Compressor(f, decomp=(3, 3, 3, 0), codeblocks=(4, 4, 4, 0), rate="1,4")
ncb = c.num_codeblocks()
cs = c.compress()
c.close()
print(hashlib.sha256(cs).hexdigest(), ncb, bwc.load().bwc_b200_mq_lanes(ncb))
""" % ROOT


def _run(env):
    r = subprocess.run([sys.executable, "-c", SCRIPT], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    h, ncb, lanes = r.stdout.split()[-3:]
    return h, int(ncb), int(lanes)


def test_autotune_records_and_keeps_bytes(gpu, tmp_path):
    tune = tmp_path / "tune.txt"
    base = dict(os.environ)
    h0, ncb, lanes0 = _run(dict(base, BWC_B200_AUTOTUNE="0"))
    assert ncb >= 64
    h1, _, lanes1 = _run(dict(base, BWC_B200_TUNE_FILE=str(tune)))
    assert h1 == h0
    lines = tune.read_text().split("\n")
    assert any(line.strip() for line in lines)
    key, val = lines[0].split()
    assert int(val) == lanes1 and 1 <= lanes1 <= 32
    # a later process starts from the file (and so does not tune again)
    h2, _, lanes2 = _run(dict(base, BWC_B200_TUNE_FILE=str(tune)))
    assert h2 == h0 and lanes2 == lanes1
    assert len([l for l in tune.read_text().split("\n") if l.strip()]) == 1
