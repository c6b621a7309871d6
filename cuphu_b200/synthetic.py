"""Seeded synthetic interferograms for the benchmark and test workloads.

No public dataset is involved: these generators define the workloads.  Each
returns ``(igram complex64, corr float32, truth float32 true phase, extra)``.

* ``bumps``    -- Gaussian bumps + linear range ramp, smooth coherence
                  (the 512^2 / 2048^2 / batch scenes; 4096^2 adds a water blob)
* ``fractal``  -- power-law topography converted to phase through the
                  repeat-pass geometry (the 8192^2 TOPO scene)

Noise: circular complex Gaussian added to a unit phasor with per-pixel
standard deviation chosen so the phase error matches the Cramer-Rao bound
sigma^2 = (1 - g^2) / (2 L g^2) for coherence g and L looks.
"""
from __future__ import annotations

import numpy as np


def _smooth_field(rng, shape, sigma):
    """Uniform noise low-passed by a Gaussian of ``sigma`` px (FFT), in [0,1]."""
    from scipy import fft
    nr, nc = shape
    u = rng.random(shape, dtype=np.float32)
    ky = fft.fftfreq(nr).astype(np.float32)[:, None]
    kx = fft.rfftfreq(nc).astype(np.float32)[None, :]
    g = np.exp(-2.0 * (np.pi * sigma) ** 2 * (ky * ky + kx * kx)).astype(np.float32)
    f = fft.irfft2(fft.rfft2(u - u.mean()) * g, s=shape, workers=-1).astype(np.float32)
    lo, hi = float(f.min()), float(f.max())
    return (f - lo) / max(hi - lo, 1e-12)


def _noisy_igram(rng, truth, gamma, nlooks, amp=None):
    g = np.clip(gamma.astype(np.float64), 1e-3, 0.999)
    sig_phase = np.sqrt((1.0 - g * g) / (2.0 * nlooks * g * g))
    s = sig_phase.astype(np.float32)   # per-component std: phase std ~ sig_phase
    noise = (rng.standard_normal(truth.shape, dtype=np.float32)
             + 1j * rng.standard_normal(truth.shape, dtype=np.float32)) * s
    z = np.exp(1j * truth.astype(np.float32)) + noise
    if amp is not None:
        z = z * amp
    return z.astype(np.complex64)


def bumps(n_rows: int, n_cols: int | None = None, seed: int = 0, nbumps: int = 3,
          amp_range=(10.0, 40.0), sigma_range=(30.0, 90.0), ramp: float = 0.05,
          gamma_range=(0.3, 0.95), nlooks: float = 5.0, water_frac: float = 0.0):
    """Gaussian-bump deformation scene (configs: 512^2, 4096^2, batch, 2048^2)."""
    n_cols = n_rows if n_cols is None else n_cols
    rng = np.random.default_rng(seed)
    rr = np.arange(n_rows, dtype=np.float32)[:, None]
    cc = np.arange(n_cols, dtype=np.float32)[None, :]
    truth = (ramp * cc + 0.0 * rr).astype(np.float32)
    for _ in range(nbumps):
        a = rng.uniform(*amp_range) * rng.choice([-1.0, 1.0])
        s = rng.uniform(*sigma_range)
        r0 = rng.uniform(0, n_rows)
        c0 = rng.uniform(0, n_cols)
        truth += (a * np.exp(-((rr - r0) ** 2 + (cc - c0) ** 2) / (2 * s * s))).astype(np.float32)
    gamma = _smooth_field(rng, (n_rows, n_cols), 20.0)
    gamma = (gamma_range[0] + (gamma_range[1] - gamma_range[0]) * gamma).astype(np.float32)
    water = None
    if water_frac > 0:
        blob = _smooth_field(rng, (n_rows, n_cols), max(n_rows, n_cols) / 40.0)
        thr = np.quantile(blob[:: max(1, n_rows // 512), :: max(1, n_cols // 512)],
                          1.0 - water_frac)
        water = blob > thr
        gamma[water] = rng.uniform(0.02, 0.1, size=int(water.sum())).astype(np.float32)
    igram = _noisy_igram(rng, truth, gamma, nlooks)
    return igram, gamma, truth, {"water": water}


def fractal_topo(n: int, seed: int = 0, beta: float = -3.0, hmax: float = 2500.0,
                 wavelength: float = 0.24, bperp: float = 150.0, slant_range: float = 850e3,
                 look_deg: float = 35.0, gamma_range=(0.2, 0.9), nlooks: float = 20.0):
    """Power-law topography scene (the 8192^2 TOPO precision config)."""
    from scipy import fft
    rng = np.random.default_rng(seed)
    ky = fft.fftfreq(n).astype(np.float32)[:, None]
    kx = fft.rfftfreq(n).astype(np.float32)[None, :]
    k2 = ky * ky + kx * kx
    k2[0, 0] = 1.0
    amp = (k2 ** (beta / 4.0)).astype(np.float32)   # |k|^(beta/2)
    amp[0, 0] = 0.0
    w = rng.standard_normal((n, n), dtype=np.float32)
    h = fft.irfft2(fft.rfft2(w) * amp, s=(n, n), workers=-1).astype(np.float32)
    h = (h - h.min()) / max(float(h.max() - h.min()), 1e-12) * hmax
    scale = 4.0 * np.pi * bperp / (wavelength * slant_range * np.sin(np.deg2rad(look_deg)))
    truth = (h * np.float32(scale)).astype(np.float32)
    gamma = _smooth_field(rng, (n, n), 20.0)
    gamma = (gamma_range[0] + (gamma_range[1] - gamma_range[0]) * gamma).astype(np.float32)
    mag = rng.exponential(1.0, size=(n, n)).astype(np.float32)
    igram = _noisy_igram(rng, truth, gamma, nlooks, amp=mag)
    return igram, gamma, truth, {"height": h, "mag": mag}


def config_scene(name: str, seed: int = 0, scale: int | None = None):
    """Scenes of the benchmark configurations by name.

    ``scale`` overrides the edge length (for small parity runs of the same
    generator)."""
    if name == "c0_512_defo":
        n = scale or 512
        ig, g, t, ex = bumps(n, seed=seed, nbumps=3, nlooks=5.0)
        return ig, g, t, dict(ex, cost="defo", nlooks=5.0)
    if name == "c1_4096_smooth":
        n = scale or 4096
        ig, g, t, ex = bumps(n, seed=seed, nbumps=6, amp_range=(10.0, 80.0), nlooks=9.0,
                             water_frac=0.15)
        return ig, g, t, dict(ex, cost="smooth", nlooks=9.0, n_irls=3)
    if name == "c2_8192_topo":
        n = scale or 8192
        ig, g, t, ex = fractal_topo(n, seed=seed)
        return ig, g, t, dict(ex, cost="topo", nlooks=20.0)
    if name == "c4_2048_defo":
        n = scale or 2048
        ig, g, t, ex = bumps(n, seed=seed, nbumps=3, nlooks=5.0)
        return ig, g, t, dict(ex, cost="defo", nlooks=5.0, n_irls=5)
    raise KeyError(name)


def batch_scenes(count: int = 48, seed: int = 0, sides=(512, 1024, 2048, 3072)):
    """The uneven batch: ``count`` bump scenes with sides drawn from ``sides``."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        nr = int(rng.choice(sides))
        nc = int(rng.choice(sides))
        ig, g, t, _ = bumps(nr, nc, seed=seed * 1000 + i + 1, nbumps=3, nlooks=5.0)
        out.append((ig, g, t))
    return out
