"""Image error against a high-spp FP64 render, and the equal-RMSE speed-up.

The reference has no image-error measure; the B200 forms are compared with a
ground-truth image rendered by the plain f64 kernel (which follows the
reference arithmetic in f64, src/integrator.rs:53-135) at 65536 spp.

Definitions used throughout (img and truth are (n_pixels, 3) linear RGB):

* rmse          = sqrt(mean over pixels and channels of (img - truth)^2)
* rel_rmse      = rmse / mean(truth)
* mean_rel_err  = mean over pixels of |lum(img) - lum(truth)| /
                  max(lum(truth), 0.01 * mean lum(truth))

Monte-Carlo error falls as 1/spp in MSE, so the time one form needs to reach
a given RMSE is proportional to MSE(spp) * spp / throughput.  The equal-RMSE
speed-up of form A over form B, both measured at the same spp, is therefore
(throughput_A / throughput_B) * (MSE_B / MSE_A).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent.parent / "tests" / "golden"
TRUTH_FILE = GOLDEN / "mesh_env_240x135_truth.npz"
TRUTH_WIDTH, TRUTH_HEIGHT = 240, 135
CORNELL_TRUTH_FILE = GOLDEN / "cornell_160x90_truth.npz"
CORNELL_WIDTH, CORNELL_HEIGHT = 160, 90


def luminance(img: np.ndarray) -> np.ndarray:
    img = np.asarray(img, dtype=np.float64).reshape(-1, 3)
    return 0.2126 * img[:, 0] + 0.7152 * img[:, 1] + 0.0722 * img[:, 2]


def image_error(img: np.ndarray, truth: np.ndarray) -> dict:
    img = np.asarray(img, dtype=np.float64).reshape(-1, 3)
    truth = np.asarray(truth, dtype=np.float64).reshape(-1, 3)
    if img.shape != truth.shape:
        raise ValueError(f"image shape {img.shape} != truth shape {truth.shape}")
    d = img - truth
    mse = float(np.mean(d * d))
    mean_t = float(np.mean(truth))
    lt = luminance(truth)
    floor = 0.01 * float(np.mean(lt))
    rel = np.abs(luminance(img) - lt) / np.maximum(lt, floor)
    return {"mse": mse, "rmse": mse ** 0.5, "rel_rmse": mse ** 0.5 / max(mean_t, 1e-300),
            "mean_rel_err": float(np.mean(rel))}


def equal_rmse_speedup(throughput_a: float, mse_a: float, throughput_b: float, mse_b: float) -> float:
    """Speed-up of form A over form B to reach the same RMSE, from each form's
    throughput (paths/s) and its MSE at one common spp."""
    return (throughput_a / throughput_b) * (mse_b / mse_a)


def load_truth(path: Path = TRUTH_FILE):
    """(image (n, 3) float64, metadata dict) of the committed ground truth."""
    with np.load(path, allow_pickle=False) as z:
        img = z["image"].astype(np.float64)
        meta = {k: z[k].item() if z[k].ndim == 0 else z[k].tolist() for k in z.files if k != "image"}
    return img, meta
