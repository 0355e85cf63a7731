"""Shared helpers of the parity tests: small test scenes and the per-pixel
Welch test."""
from __future__ import annotations

import numpy as np

from tinypt_b200 import scenes
from tinypt_b200.scene import RenderConfig


def small_mesh_env_scene(width=96, height=54, subdiv=3, n_spheres=24, env_w=64, env_h=32, seed=7):
    """The 1080p mesh+env workload at test size: same generator, fewer triangles,
    spheres and env texels."""
    return scenes.mesh_env_scene(width, height, subdiv, n_spheres, env_w, env_h, seed)


def cfg(w, h, spp, depth, mode, seed=1, **kw) -> RenderConfig:
    return RenderConfig(width=w, height=h, spp=spp, max_bounces=depth, rr_start=3, seed=seed, mode=mode, **kw)


def welch_z(acc1, sq1, n1, acc2, sq2, n2):
    """Per-pixel, per-channel Welch statistic of two independent-sample
    estimates (sums acc, sums of squares sq, sample counts n)."""
    n1 = np.asarray(n1, dtype=np.float64)[:, None]
    n2 = np.asarray(n2, dtype=np.float64)[:, None]
    m1, m2 = acc1 / n1, acc2 / n2
    v1 = np.maximum(sq1 - n1 * m1 * m1, 0.0) / np.maximum(n1 - 1.0, 1.0)
    v2 = np.maximum(sq2 - n2 * m2 * m2, 0.0) / np.maximum(n2 - 1.0, 1.0)
    se = np.sqrt(v1 / n1 + v2 / n2)
    diff = m1 - m2
    z = np.zeros_like(diff)
    ok = se > 1e-12
    z[ok] = diff[ok] / se[ok]
    z[~ok & (np.abs(diff) > 1e-6)] = np.inf
    return z


def relative_rms(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b ** 2)), 1e-30))


def frac_beyond(z, t=3.0):
    """Fraction of pixel-channels with |z| > t."""
    return float(np.mean(np.abs(z) > t))


def z_tail_bar(null_frac, n_pixels, t=3.0, k=4.0):
    """Upper bar for the |z| > t fraction of a comparison whose statistic
    should behave like the calibration (null) comparison: the larger of the
    nominal two-sided normal tail (0.27% at t = 3) and the null's measured
    fraction, plus k binomial standard deviations counted over pixels (the
    three channels of a pixel are strongly correlated, so channels are not
    independent trials)."""
    from math import erfc, sqrt

    p = max(erfc(t / sqrt(2.0)), null_frac)
    return p + k * sqrt(p * (1.0 - p) / max(n_pixels, 1))


def gpu_film(ds, c, want_sq=True):
    """Renders c into device buffers through tpt_render_device; returns
    ((acc (n,3), acc_w (n,), acc_sq (n,3) or None), stats) on the host."""
    import torch

    n = c.width * c.height
    acc = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    acc_w = torch.zeros(n, dtype=torch.float64, device="cuda")
    acc_sq = torch.zeros(3 * n, dtype=torch.float64, device="cuda") if want_sq else None
    st = ds.render_device(c, acc.data_ptr(), acc_w.data_ptr(), acc_sq.data_ptr() if want_sq else 0)
    torch.cuda.synchronize()
    out = (acc.cpu().numpy().reshape(n, 3), acc_w.cpu().numpy(),
           acc_sq.cpu().numpy().reshape(n, 3) if want_sq else None)
    return out, st


def image_mean_z(acc1, sq1, n1, acc2, sq2, n2):
    """z statistic of the difference of two films' image means (the mean over
    pixels and channels of the pixel means), from the per-pixel sample
    variances; also returns the relative difference."""
    n1 = np.asarray(n1, dtype=np.float64)[:, None]
    n2 = np.asarray(n2, dtype=np.float64)[:, None]
    m1, m2 = acc1 / n1, acc2 / n2
    v1 = np.maximum(sq1 - n1 * m1 * m1, 0.0) / np.maximum(n1 - 1.0, 1.0) / n1
    v2 = np.maximum(sq2 - n2 * m2 * m2, 0.0) / np.maximum(n2 - 1.0, 1.0) / n2
    k = m1.size
    se = np.sqrt(v1.sum() + v2.sum()) / k
    d = m1.mean() - m2.mean()
    return (d / se if se > 0 else (0.0 if d == 0 else np.inf)), abs(d) / max(abs(m2.mean()), 1e-30)


def divergence_rate(exact_frac, spp):
    """Per-sample rate at which a path leaves the reference's stream, from
    the fraction of pixels whose spp samples all match: exact = (1 - p)^spp."""
    return 1.0 - max(exact_frac, 1e-300) ** (1.0 / spp)
