"""The learned warm start of rate control: data, training, evaluation.

The library's rate control (PCRD) bisects, per quality layer, over a 16-bit log-slope
threshold.  A small network (34 -> 64 -> 64 -> 1, FP32) predicts the final threshold from a
histogram of the codeblocks' pass slopes, the layer's bits per value and the field size; the
library then evaluates the probe path the prediction implies at once and replays the exact
search over those results, so the bytes never change -- only the number of dependent probe
rounds does (see include/bwc_b200.h, "Rate-control warm start").

Everything here runs the library's own code: training data come from exact rate control on
synthetic fields (batched compression on the GPU), and the network is trained with the
library's hand-written CUDA forward/backward/Adam kernels (bwc_b200_mlp_train).

    python -m bigwhoop_b200.ratemodel            # make the data set, train, evaluate, save

writes bigwhoop_b200/data/pcrd_dataset.npz and bigwhoop_b200/data/pcrd_mlp.npy.
"""
from __future__ import annotations

import argparse
import ctypes as C
import os

import numpy as np

from . import bwc, fields

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "data")
N_IN, N_HID, N_PARAMS = 34, 64, 6465
DEFAULT_MODEL = os.path.join(DATA, "pcrd_mlp.npy")
DEFAULT_DATA = os.path.join(DATA, "pcrd_dataset.npz")


def init_params(seed=0):
    """He-initialised parameters in the library's layout (W1, b1, W2, b2, W3, b3)."""
    rng = np.random.default_rng(seed)
    w1 = rng.normal(0, np.sqrt(2.0 / N_IN), (N_HID, N_IN))
    w2 = rng.normal(0, np.sqrt(2.0 / N_HID), (N_HID, N_HID))
    w3 = rng.normal(0, np.sqrt(1.0 / N_HID), N_HID)
    p = np.concatenate([w1.ravel(), np.zeros(N_HID), w2.ravel(), np.zeros(N_HID), w3, [0.5]])
    assert p.size == N_PARAMS
    return p.astype(np.float32)


def _lib(precision="double"):
    return bwc.load(precision)


def forward(params, X, precision="double"):
    X = np.ascontiguousarray(X, np.float32)
    y = np.zeros(X.shape[0], np.float32)
    p = np.ascontiguousarray(params, np.float32)
    assert _lib(precision).bwc_b200_mlp_forward(p.ctypes.data, X.ctypes.data, X.shape[0], y.ctypes.data) == 0
    return y


def gradient(params, X, t, precision="double"):
    X = np.ascontiguousarray(X, np.float32)
    t = np.ascontiguousarray(t, np.float32)
    p = np.ascontiguousarray(params, np.float32)
    g = np.zeros(N_PARAMS, np.float32)
    loss = np.zeros(1, np.float32)
    assert _lib(precision).bwc_b200_mlp_gradient(p.ctypes.data, X.ctypes.data, t.ctypes.data,
                                                 X.shape[0], g.ctypes.data, loss.ctypes.data) == 0
    return g, float(loss[0])


def train(params, X, t, epochs=400, batch=64, lr=2e-3, seed=0, precision="double"):
    p = np.array(params, np.float32, copy=True)
    X = np.ascontiguousarray(X, np.float32)
    t = np.ascontiguousarray(t, np.float32)
    hist = np.zeros(epochs, np.float32)
    assert _lib(precision).bwc_b200_mlp_train(p.ctypes.data, X.ctypes.data, t.ctypes.data, X.shape[0],
                                              epochs, batch, lr, seed, hist.ctypes.data) == 0
    return p, hist


def set_model(params, precision="double"):
    """Use `params` for warm starts in this process (None: plain bisection)."""
    L = _lib(precision)
    if params is None:
        L.bwc_b200_set_rate_model(None)
    else:
        p = np.ascontiguousarray(params, np.float32)
        L.bwc_b200_set_rate_model(p.ctypes.data)


def load_default(precision="double"):
    set_model(np.load(DEFAULT_MODEL), precision)


def features(comp, layer=0):
    out = np.zeros(N_IN, np.float32)
    assert comp.L.bwc_b200_rate_features(comp.codec, layer, out.ctypes.data) == 0
    return out


def stats(comp, layer=0):
    """final threshold, probes, rounds of dependent probes, predicted threshold, slope range."""
    out = np.zeros(6)
    assert comp.L.bwc_b200_rate_stats(comp.codec, layer, out.ctypes.data) == 0
    return out


# ---- data --------------------------------------------------------------------------------------

def cpu_forward(params, X):
    """numpy restatement of the network (for checking the CUDA kernels)."""
    p = np.asarray(params, np.float64)
    w1 = p[:N_HID * N_IN].reshape(N_HID, N_IN)
    o = N_HID * N_IN
    b1 = p[o:o + N_HID]; o += N_HID
    w2 = p[o:o + N_HID * N_HID].reshape(N_HID, N_HID); o += N_HID * N_HID
    b2 = p[o:o + N_HID]; o += N_HID
    w3 = p[o:o + N_HID]; o += N_HID
    b3 = p[o]
    a1 = X @ w1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ w2.T + b2
    h2 = np.maximum(a2, 0)
    return h2 @ w3 + b3, (a1, h1, a2, h2, w1, w2, w3)


def cpu_gradient(params, X, t):
    X = np.asarray(X, np.float64)
    y, (a1, h1, a2, h2, w1, w2, w3) = cpu_forward(params, X)
    n = X.shape[0]
    dy = 2.0 * (y - t) / n
    g_w3 = dy @ h2
    g_b3 = dy.sum()
    d2 = np.outer(dy, w3) * (a2 > 0)
    g_w2 = d2.T @ h1
    g_b2 = d2.sum(0)
    d1 = (d2 @ w2) * (a1 > 0)
    g_w1 = d1.T @ X
    g_b1 = d1.sum(0)
    g = np.concatenate([g_w1.ravel(), g_b1, g_w2.ravel(), g_b2, g_w3, [g_b3]])
    return g, float(np.mean((y - t) ** 2))


def field_specs(seeds, seed_targets=7):
    rng = np.random.default_rng(seed_targets)
    return [(int(s), float(rng.uniform(0.1, 8.0))) for s in seeds]


def make_samples(specs, shape=(128, 128, 128), batch=32, precision="double", log=print):
    """Features and exact final thresholds of one-layer compressions of config-1 fields (FP32),
    computed by batched compression on the GPU."""
    X, t, S = [], [], []
    for b0 in range(0, len(specs), batch):
        chunk = specs[b0:b0 + batch]
        fs = [fields.shock_field(shape, s, dtype=np.float32, device="cuda").cpu().numpy() for s, _ in chunk]
        bwc.reset_gain_state(precision)
        comps = [bwc.Compressor(f, precision=precision, decomp=(4, 4, 4, 0), codeblocks=(5, 5, 4, 0),
                                rate="%.6f" % r) for f, (_, r) in zip(fs, chunk)]
        try:
            bwc.compress_batch(comps)
            for c in comps:
                X.append(features(c))
                st = stats(c)
                t.append(st[0] / 65536.0)
                S.append(st)
        finally:
            for c in comps:
                c.close()
        if log:
            log(f"  {min(b0 + batch, len(specs))}/{len(specs)} fields")
    return np.array(X, np.float32), np.array(t, np.float32), np.array(S)


def evaluate(specs, params, shape=(128, 128, 128), batch=32, precision="double"):
    """Compress every field with and without the model: the codestreams must be identical;
    returns (final thresholds, predicted thresholds, plain probe counts, warm-start rounds)."""
    final, pred, probes, rounds = [], [], [], []
    for b0 in range(0, len(specs), batch):
        chunk = specs[b0:b0 + batch]
        fs = [fields.shock_field(shape, s, dtype=np.float32, device="cuda").cpu().numpy() for s, _ in chunk]
        out = {}
        for use in (False, True):
            set_model(params if use else None, precision)
            bwc.reset_gain_state(precision)
            comps = [bwc.Compressor(f, precision=precision, decomp=(4, 4, 4, 0),
                                    codeblocks=(5, 5, 4, 0), rate="%.6f" % r) for f, (_, r) in zip(fs, chunk)]
            try:
                cs = bwc.compress_batch(comps)
                out[use] = (cs, [stats(c) for c in comps])
            finally:
                for c in comps:
                    c.close()
        set_model(None, precision)
        if out[False][0] != out[True][0]:
            raise AssertionError("warm start changed a codestream")
        for sp, sw in zip(out[False][1], out[True][1]):
            final.append(sp[0])
            pred.append(sw[3])
            probes.append(sp[1])
            rounds.append(sw[2])
    return np.array(final), np.array(pred), np.array(probes), np.array(rounds)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-fields", type=int, default=2000)
    ap.add_argument("--eval-fields", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=600)
    ap.add_argument("--reuse-data", action="store_true")
    ap.add_argument("--out", default=DATA, help="directory for pcrd_dataset.npz, pcrd_mlp.npy")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    data_path = os.path.join(a.out, "pcrd_dataset.npz")
    model_path = os.path.join(a.out, "pcrd_mlp.npy")
    if a.reuse_data and os.path.exists(data_path):
        d = np.load(data_path)
        Xtr, ttr, Xev, tev = d["X_train"], d["t_train"], d["X_eval"], d["t_eval"]
    else:
        tr = field_specs(range(1000, 1000 + a.train_fields))
        ev = field_specs(range(3000, 3000 + a.eval_fields), seed_targets=8)
        Xtr, ttr, _ = make_samples(tr)
        Xev, tev, _ = make_samples(ev)
        np.savez_compressed(data_path, X_train=Xtr, t_train=ttr, X_eval=Xev, t_eval=tev,
                            train_specs=np.array(tr), eval_specs=np.array(ev))
    p0 = init_params(0)
    p, hist = train(p0, Xtr, ttr, epochs=a.epochs)
    np.save(model_path, p)
    pred = forward(p, Xev)
    err = np.abs(pred - tev) * 65536
    print(f"loss first/last epoch {hist[0]:.5f} / {hist[-1]:.6f}; held-out |error| median "
          f"{np.median(err):.0f}, p90 {np.percentile(err, 90):.0f} slope units")
    ev = field_specs(range(3000, 3000 + a.eval_fields), seed_targets=8)
    final, pred, probes, rounds = evaluate(ev, p)
    print(f"held-out fields {len(final)}: codestreams identical with and without the model; "
          f"dependent probe rounds {rounds.mean():.2f} (plain bisection {probes.mean():.2f} probes); "
          f"threshold |error| mean {np.abs(final - pred).mean():.1f}")


if __name__ == "__main__":
    main()
