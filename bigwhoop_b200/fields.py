"""Seeded synthetic test fields with the shapes and statistics of the benchmark workloads.

The reference codec is exercised on simulation fields; no public data set is used, so every
workload is a sum of random Fourier modes (a turbulence-like spectrum) with optional shock
fronts, a constant region and measurement noise.  Arrays are C-ordered with the codec's fastest
axis (x) last: shape (nTS, nZ, nY, nX) or (nZ, nY, nX).

Small fields are evaluated with numpy; large ones can be evaluated with torch on a GPU
(``device="cuda"``).  The mode parameters come from numpy's PCG64 generator in both cases, so a
given seed describes the same field; the two evaluators agree to rounding.
"""
from __future__ import annotations

import math

import numpy as np


def _mode_params(rng, n_modes, ndim, kmin, kmax, slope):
    k = rng.uniform(kmin, kmax, size=(n_modes, ndim))
    phase = rng.uniform(0.0, 2.0 * math.pi, size=n_modes)
    amp = np.linalg.norm(k, axis=1) ** slope
    return k, phase, amp


def spectral_field(shape, seed, *, n_modes=256, slope=-11.0 / 6.0, kmin=1.0, kmax=16.0,
                   noise=1e-6, dtype=np.float64, device=None):
    """Sum of ``n_modes`` cosine modes, amplitude |k|^slope, uniform phase, plus Gaussian noise.

    ``shape`` is (nZ, nY, nX) or (nTS, nZ, nY, nX); wave-vector components are uniform in
    [kmin, kmax] cycles per domain along every spatial axis (the time axis, if present, is
    handled by :func:`advected_field`).  ``noise`` is the noise standard deviation relative to
    the field's standard deviation.
    """
    shape = tuple(int(s) for s in shape)
    rng = np.random.default_rng(seed)
    k, phase, amp = _mode_params(rng, n_modes, len(shape), kmin, kmax, slope)
    noise_seed = int(rng.integers(0, 2**63 - 1))
    if device is not None and str(device).startswith("cuda"):
        f = _eval_torch(shape, k, phase, amp, device)
        if noise:
            import torch
            g = torch.Generator(device=device).manual_seed(noise_seed)
            f += torch.randn(f.shape, generator=g, device=device, dtype=f.dtype) * (noise * f.std())
        return f.to(_torch_dtype(dtype))
    f = _eval_numpy(shape, k, phase, amp)
    if noise:
        nrng = np.random.default_rng(noise_seed)
        f += nrng.standard_normal(f.shape) * (noise * f.std())
    return f.astype(dtype, copy=False)


def _axes_phases(shape, kvec):
    # x is the last array axis; wave-vector component i belongs to array axis -(i+1)
    out = []
    nd = len(shape)
    for ax in range(nd):
        comp = nd - 1 - ax
        n = shape[ax]
        out.append(2.0 * math.pi * kvec[comp] * np.arange(n) / n)
    return out


def _eval_numpy(shape, k, phase, amp):
    f = np.zeros(shape, dtype=np.float64)
    for m in range(k.shape[0]):
        ph = _axes_phases(shape, k[m])
        e = np.exp(1j * ph[0]) * np.exp(1j * phase[m])
        for a in ph[1:]:
            e = np.multiply.outer(e, np.exp(1j * a))
        f += amp[m] * e.real
    return f


def _torch_dtype(dtype):
    import torch
    return torch.float64 if np.dtype(dtype) == np.float64 else torch.float32


def _eval_torch(shape, k, phase, amp, device):
    import torch
    f = torch.zeros(shape, dtype=torch.float64, device=device)
    for m in range(k.shape[0]):
        ph = _axes_phases(shape, k[m])
        e = None
        for ax, a in enumerate(ph):
            v = torch.from_numpy(np.exp(1j * a)).to(device)
            if ax == 0:
                v = v * complex(np.exp(1j * phase[m]))
            view = [1] * len(shape)
            view[ax] = shape[ax]
            v = v.view(view)
            e = v if e is None else e * v
        f += amp[m] * e.real
    return f


def advected_field(shape, seed, *, shift=1.5, n_modes=256, slope=-11.0 / 6.0, kmin=1.0,
                   kmax=16.0, noise=1e-5, dtype=np.float64, device="cuda"):
    """Time series (nTS, nZ, nY, nX) of a 3D spectral field advected along x by `shift` cells
    per step (a phase shift of every mode), each step with fresh Gaussian noise of relative
    standard deviation `noise`.  Evaluated with torch on `device`."""
    import torch
    nt, spatial = int(shape[0]), tuple(int(v) for v in shape[1:])
    rng = np.random.default_rng(seed)
    k, phase, amp = _mode_params(rng, n_modes, 3, kmin, kmax, slope)
    noise_seed = int(rng.integers(0, 2**63 - 1))
    g = torch.Generator(device=device).manual_seed(noise_seed)
    out = torch.empty((nt,) + spatial, dtype=_torch_dtype(dtype), device=device)
    nx = spatial[2]
    for t in range(nt):
        # f(x - shift * t): every mode's phase moves by -2 pi k_x shift t / nx
        ph = phase - 2.0 * math.pi * k[:, 0] * shift * t / nx
        f = _eval_torch(spatial, k, ph, amp, device)
        if noise:
            f += torch.randn(f.shape, generator=g, device=device, dtype=f.dtype) * (noise * f.std())
        out[t] = f.to(out.dtype)
        del f
    return out


def add_shocks(f, seed, n_fronts=8, width=2.0, rel_amp=1.0):
    """Add ``n_fronts`` tanh fronts of the given width (cells) across random planes (numpy)."""
    rng = np.random.default_rng(seed)
    shape = f.shape
    scale = rel_amp * float(np.std(f))
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape], indexing="ij")
    for _ in range(n_fronts):
        nrm = rng.normal(size=len(shape))
        nrm /= np.linalg.norm(nrm)
        centre = np.array([rng.uniform(0, n) for n in shape])
        dist = sum(nrm[i] * (grids[i] - centre[i]) for i in range(len(shape)))
        f += scale * np.tanh(dist / width)
    return f


def constant_quarter(f):
    """Set one quarter of the domain (first half of the two slowest spatial axes) constant."""
    s = [slice(None)] * f.ndim
    s[-3] = slice(0, f.shape[-3] // 2)
    s[-2] = slice(0, f.shape[-2] // 2)
    f[tuple(s)] = float(np.mean(f))
    return f


def shock_field(shape, seed, dtype=np.float64, *, slope=-11.0 / 6.0, noise=1e-6, device=None):
    """Spectral field + 8 tanh fronts (width 2 cells) + a constant quarter.

    With ``device="cuda"`` the spectral part and the fronts are evaluated on the GPU.
    """
    if device is not None and str(device).startswith("cuda"):
        import torch
        f = spectral_field(shape, seed, slope=slope, noise=noise, dtype=np.float64, device=device)
        rng = np.random.default_rng(seed + 7919)
        scale = float(f.std())
        coords = [torch.arange(n, dtype=torch.float64, device=device) for n in shape]
        for _ in range(8):
            nrm = rng.normal(size=len(shape))
            nrm /= np.linalg.norm(nrm)
            centre = [rng.uniform(0, n) for n in shape]
            dist = None
            for ax, c in enumerate(coords):
                view = [1] * len(shape)
                view[ax] = shape[ax]
                term = (float(nrm[ax]) * (c - centre[ax])).view(view)
                dist = term if dist is None else dist + term
            f += scale * torch.tanh(dist / 2.0)
        s = [slice(None)] * f.ndim
        s[-3] = slice(0, shape[-3] // 2)
        s[-2] = slice(0, shape[-2] // 2)
        f[tuple(s)] = f.mean()
        return f.to(_torch_dtype(dtype))
    f = spectral_field(shape, seed, slope=slope, noise=noise, dtype=np.float64)
    add_shocks(f, seed + 7919)
    constant_quarter(f)
    return f.astype(dtype, copy=False)


def uneven_batch(seed=2, n_fields=64, lo=33, hi=300):
    """Descriptors of the uneven batch: per field shape, dtype, rate, decomposition depth, slope."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_fields):
        shape = tuple(int(v) for v in rng.integers(lo, hi + 1, size=3))
        dtype = np.float32 if rng.random() < 0.5 else np.float64
        rate = float(rng.choice([0.25, 0.5, 1.0, 2.0, 4.0]))
        levels = int(rng.integers(2, 5))
        slope = float(rng.uniform(-3.0, -1.0))
        out.append(dict(shape=shape, dtype=dtype, rate=rate, levels=levels, slope=slope,
                        seed=seed * 1000 + i))
    return out
