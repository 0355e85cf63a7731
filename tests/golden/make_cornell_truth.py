"""Renders the ground-truth image of the Cornell adaptive-sampling scene at 160x90.

The scene is scenes.cornell_scene (Cornell box, 262,144-triangle displaced
GGX mesh, absorbing dielectric sphere, ceiling light; max_depth 32,
rr_depth 3) on a 160x90 film at the 1080p camera and aspect.  The image is
the plain f64 GPU form at 65536 spp without adaptive stopping, summed over
16 renders of 4096 spp with seeds 3000..3015.  Needs a CUDA device; writes a
compressed .npz with the float32 mean image and the settings.

    python tests/golden/make_cornell_truth.py OUT.npz
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

W, H = 160, 90
SPP_PER_RENDER = 4096
SEEDS = list(range(3000, 3016))


def main(out: str) -> None:
    import torch

    from tinypt_b200 import _abi, scenes
    from tinypt_b200.render import DeviceScene
    from tinypt_b200.scene import RenderConfig

    scene = scenes.cornell_scene(W, H)
    n = W * H
    acc = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    acc_w = torch.zeros(n, dtype=torch.float64, device="cuda")
    tot = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    tot_w = torch.zeros(n, dtype=torch.float64, device="cuda")
    t0 = time.perf_counter()
    with DeviceScene(scene) as ds:
        for seed in SEEDS:
            cfg = RenderConfig(width=W, height=H, spp=SPP_PER_RENDER, max_bounces=32, rr_start=3, seed=seed,
                               mode=_abi.TPT_MODE_PLAIN_F64)
            st = ds.render_device(cfg, acc.data_ptr(), acc_w.data_ptr())
            if st.device_flags:
                raise RuntimeError(f"device flags {st.device_flags:#x} at seed {seed}")
            tot += acc
            tot_w += acc_w
            print(f"seed {seed}: {st.render_ms:.0f} ms", flush=True)
    torch.cuda.synchronize()
    img = (tot.view(n, 3) / tot_w.clamp(min=1.0)[:, None]).cpu().numpy()
    spp = int(tot_w.min().item())
    assert spp == SPP_PER_RENDER * len(SEEDS), spp
    np.savez_compressed(out, image=img.astype(np.float32), width=W, height=H, spp=spp,
                        seeds=np.array(SEEDS), max_bounces=32, rr_start=3, mode="plain_f64",
                        scene="cornell_scene(160, 90): Cornell box, 262,144-triangle GGX mesh, absorbing sphere")
    print(f"wrote {out}: {spp} spp, {time.perf_counter() - t0:.1f} s, mean {img.mean():.6g}", flush=True)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(ROOT / "tests" / "golden" / "cornell_160x90_truth.npz"))
