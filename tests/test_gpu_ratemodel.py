"""The learned rate-control warm start on the GPU.

* the CUDA forward pass and gradient equal the numpy restatement (float32 against float64, so
  within 1e-4 relative to the largest gradient entry);
* training with the CUDA kernels lowers the loss;
* codestreams are byte-identical with and without a model, and with the trained model the
  rate control needs fewer rounds of dependent probes than the plain bisection.
"""
import os

import numpy as np
import pytest

from bigwhoop_b200 import bwc, fields, ratemodel

pytestmark = pytest.mark.gpu


def test_forward_and_gradient_match_cpu(gpu):
    rng = np.random.default_rng(4)
    p = ratemodel.init_params(2)
    X = rng.random((40, 34)).astype(np.float32)
    t = rng.random(40).astype(np.float32)
    y = ratemodel.forward(p, X)
    y_ref, _ = ratemodel.cpu_forward(p, X)
    assert np.max(np.abs(y - y_ref)) < 1e-4 * max(1.0, np.max(np.abs(y_ref)))
    g, loss = ratemodel.gradient(p, X, t)
    g_ref, loss_ref = ratemodel.cpu_gradient(p, X, t)
    assert np.max(np.abs(g - g_ref)) < 1e-4 * np.max(np.abs(g_ref))
    assert abs(loss - loss_ref) < 1e-4 * max(1.0, loss_ref)


def test_training_lowers_the_loss(gpu):
    rng = np.random.default_rng(5)
    X = rng.random((256, 34)).astype(np.float32)
    t = (0.3 + 0.4 * X[:, 0] - 0.2 * X[:, 5] * X[:, 9]).astype(np.float32)
    p0 = ratemodel.init_params(3)
    _, l0 = ratemodel.gradient(p0, X, t)
    p, hist = ratemodel.train(p0, X, t, epochs=200, batch=32, lr=3e-3, seed=1)
    _, l1 = ratemodel.gradient(p, X, t)
    assert l1 < 0.1 * l0, (l0, l1)
    assert hist[-1] < hist[0]
    # deterministic: the same seed gives the same weights
    p2, _ = ratemodel.train(p0, X, t, epochs=200, batch=32, lr=3e-3, seed=1)
    assert np.array_equal(p, p2)


def _compress_with_stats(f, rate, precision="double"):
    bwc.reset_gain_state(precision)
    c = bwc.Compressor(f, precision=precision, decomp=(4, 4, 4, 0), codeblocks=(5, 5, 4, 0), rate=rate)
    try:
        cs = c.compress()
        nl = len(rate.split(","))
        st = np.array([ratemodel.stats(c, l) for l in range(nl)])
    finally:
        c.close()
    return cs, st


def test_warm_start_keeps_bytes_and_saves_rounds(gpu):
    if not os.path.exists(ratemodel.DEFAULT_MODEL):
        pytest.fail("trained model missing: python -m bigwhoop_b200.ratemodel")
    model = np.load(ratemodel.DEFAULT_MODEL)
    probes, rounds = 0, 0
    for seed, rate in [(3001, "0.5"), (3002, "2"), (3003, "6"), (3004, "0.5,1,2,4")]:
        f = fields.shock_field((128, 128, 128), seed, dtype=np.float32, device="cuda").cpu().numpy()
        ratemodel.set_model(None)
        cs_plain, st_plain = _compress_with_stats(f, rate)
        ratemodel.set_model(model)
        try:
            cs_warm, st_warm = _compress_with_stats(f, rate)
        finally:
            ratemodel.set_model(None)
        assert cs_warm == cs_plain
        assert np.array_equal(st_warm[:, 0], st_plain[:, 0])     # same final thresholds
        assert np.array_equal(st_warm[:, 1], st_plain[:, 1])     # same probes
        # plain: one new probe per round (a slope the search revisits is not evaluated again)
        assert np.all(st_plain[:, 2] <= st_plain[:, 1])
        assert np.all(st_warm[:, 3] >= 0)                        # a prediction was made
        probes += st_plain[:, 2].sum()
        rounds += st_warm[:, 2].sum()
    assert rounds < probes, (rounds, probes)
