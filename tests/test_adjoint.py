"""Adjoint (path-replay) material gradients.

The reference has no derivative; the bar is the one the adjoint is specified
by: agreement with central finite differences under common random numbers
(same seed, sampling held at the base materials) within 2% per parameter,
and agreement with the f64 reference gradient of the CPU oracle.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from tinypt_b200 import _abi, autodiff, scenes
from tinypt_b200.scene import RenderConfig

# differentiable parameters of scenes.gradcheck_scene(): (material, component)
GC_PARAMS = [(0, 0), (0, 1), (0, 2),            # Lambert ground albedo
             (1, 0), (1, 1), (1, 2), (1, 3),    # GGX albedo + alpha
             (2, 0), (2, 1), (2, 2),            # Metal albedo
             (3, 0), (3, 1), (3, 2),            # Dielectric absorption
             (4, 0), (4, 1), (4, 2),            # Subsurface albedo
             (5, 0), (5, 1), (5, 2),            # Lambert sphere albedo
             (6, 0), (6, 1), (6, 2)]            # area-light emission
NOT_DIFFERENTIATED = [(0, 3), (2, 3), (3, 3), (4, 3), (5, 3), (6, 3)]


def gc_cfg(w=64, h=64, spp=32, seed=7, rr_start=6):
    return RenderConfig(width=w, height=h, spp=spp, max_bounces=6, rr_start=rr_start, seed=seed,
                        mode=_abi.TPT_MODE_WAVEFRONT_FP32)


def adjoint_image(w, h, seed):
    """A fixed dL/dimage with both signs (a linear loss), float32 (h, w, 3)."""
    rng = np.random.default_rng(seed)
    return (0.5 + rng.standard_normal((h, w, 3))).astype(np.float32)


def check_close(name, adj, ref, rel, abs_frac):
    scale = float(np.abs(ref).max())
    err = np.abs(adj - ref)
    bound = rel * np.abs(ref) + abs_frac * scale
    for k, (a, r, e, b) in enumerate(zip(adj, ref, err, bound)):
        print(f"{name} {k:2d}: adjoint {a:+.6e}  reference {r:+.6e}  rel {e / max(abs(r), 1e-300):.2e}"
              f"{'  FAIL' if e > b else ''}")
    assert np.all(err <= bound)


# ---- CPU: host logic and the oracle's detached sampling --------------------------------------
def test_params_roundtrip():
    base = scenes.gradcheck_scene().mats
    p = autodiff.params_of(base)
    assert p.shape == (len(base), 4)
    again = autodiff.params_of(autodiff.materials_with(base, p))
    assert np.array_equal(p, again)
    assert [m.kind for m in autodiff.materials_with(base, p + 0.1)] == [m.kind for m in base]


def test_oracle_detached_sampling(oracle_mod):
    """Sampling materials equal to the evaluation materials change nothing;
    a GGX alpha moved only for evaluation keeps every sample count and moves
    the image a little."""
    scene = scenes.gradcheck_scene(16, 16)
    cfg = gc_cfg(16, 16, spp=4, seed=3)
    with oracle_mod.OracleScene(scene) as os_:
        a0, w0, _, _ = os_.render(cfg)
        os_.set_materials(scene.mats, sampling_materials=scene.mats)
        a1, w1, _, _ = os_.render(cfg)
        assert np.array_equal(a0, a1) and np.array_equal(w0, w1)
        p = autodiff.params_of(scene.mats)
        p[1, 3] += 1e-3
        os_.set_materials(autodiff.materials_with(scene.mats, p), sampling_materials=scene.mats)
        a2, w2, _, _ = os_.render(cfg)
        assert np.array_equal(w0, w2)
        assert 0.0 < np.abs(a2 - a0).max() < 1e-2 * np.abs(a0).max()
        with pytest.raises(RuntimeError):
            bad = list(scene.mats)
            bad[0] = bad[1]
            os_.set_materials(bad)


# ---- GPU ----------------------------------------------------------------------------------------
@pytest.mark.gpu
def test_adjoint_matches_crn_finite_differences(gpu):
    """Every differentiable parameter of the check scene within 2% (plus
    0.1% of the largest gradient, for parameters whose gradient nearly
    cancels) of central differences with h = 1e-3 at the same seed."""
    import torch

    from tinypt_b200.render import DeviceScene

    scene = scenes.gradcheck_scene()
    cfg = gc_cfg()
    d = torch.tensor(adjoint_image(cfg.width, cfg.height, 1), device="cuda")
    with DeviceScene(scene) as ds:
        grad = torch.empty(4 * ds.n_materials, dtype=torch.float64, device="cuda")
        st = ds.render_backward(cfg, d.data_ptr(), grad.data_ptr())
        assert st.device_flags == 0 and st.paths == cfg.width * cfg.height * cfg.spp
        g = grad.cpu().numpy()
        idx = [4 * m + c for m, c in GC_PARAMS]
        fd = autodiff.fd_gradient(ds, scene.mats, cfg, d, idx, h=1e-3)
    check_close("crn-fd", g[idx], fd, 0.02, 1e-3)
    for m, c in NOT_DIFFERENTIATED:
        assert g[4 * m + c] == 0.0


@pytest.mark.gpu
def test_adjoint_with_russian_roulette(gpu):
    """With Russian roulette on, the adjoint holds the survival probability
    constant while finite differences see survival decisions flip, so the
    two agree in expectation only.  Over 16 seeds the mean of (adjoint - FD)
    is within 5 standard errors of zero for every parameter (FD at h = 1e-2
    to keep the flip noise moderate; the standard error itself comes from
    16 samples, hence 5 rather than 4)."""
    import torch

    from tinypt_b200.render import DeviceScene

    scene = scenes.gradcheck_scene(32, 32)
    idx = [4 * m + c for m, c in GC_PARAMS]
    diffs, adjs = [], []
    with DeviceScene(scene) as ds:
        grad = torch.empty(4 * ds.n_materials, dtype=torch.float64, device="cuda")
        for seed in range(16):
            cfg = gc_cfg(32, 32, spp=64, seed=100 + seed, rr_start=2)
            d = torch.tensor(adjoint_image(cfg.width, cfg.height, 2), device="cuda")
            ds.render_backward(cfg, d.data_ptr(), grad.data_ptr())
            g = grad.cpu().numpy()[idx]
            fd = autodiff.fd_gradient(ds, scene.mats, cfg, d, idx, h=1e-2)
            diffs.append(g - fd)
            adjs.append(g)
    diffs, adjs = np.array(diffs), np.array(adjs)
    mean, se = diffs.mean(0), diffs.std(0, ddof=1) / np.sqrt(len(diffs))
    scale = np.abs(adjs.mean(0)).max()
    for k in range(len(idx)):
        print(f"rr {k:2d}: adjoint {adjs[:, k].mean():+.5e}  mean(adj-fd) {mean[k]:+.3e}  se {se[k]:.3e}")
    assert np.all(np.abs(mean) <= 5.0 * se + 1e-3 * scale)


@pytest.mark.gpu
def test_adjoint_matches_f64_oracle_gradient(gpu, oracle_mod, monkeypatch):
    """The f64 reference gradient: central differences of the CPU oracle (f64
    restatement of the reference renderer, same per-pixel RNG streams, one
    task per pixel).  The FP32 adjoint follows the same streams, so the two
    see the same paths except where an FP32 decision flips a branch."""
    import torch

    from tinypt_b200.render import DeviceScene

    scene = scenes.gradcheck_scene(32, 32)
    cfg = gc_cfg(32, 32, spp=16, seed=9)
    monkeypatch.setenv("TPT_TASK_SPP", str(cfg.spp))  # one task per pixel, as the oracle
    dn = adjoint_image(cfg.width, cfg.height, 3)
    d = torch.tensor(dn, device="cuda")
    with DeviceScene(scene) as ds:
        grad = torch.empty(4 * ds.n_materials, dtype=torch.float64, device="cuda")
        ds.render_backward(cfg, d.data_ptr(), grad.data_ptr())
    idx = [4 * m + c for m, c in GC_PARAMS]
    with oracle_mod.OracleScene(scene) as os_:
        ref = autodiff.oracle_fd_gradient(os_, scene.mats, cfg, dn, idx, h=1e-3)
    check_close("f64-oracle", grad.cpu().numpy()[idx], ref, 0.05, 5e-3)


@pytest.mark.gpu
def test_autograd_wrapper_and_descent(gpu):
    """torch.autograd through RenderMaterials gives the adjoint's gradient of
    an L2 loss, and a few gradient steps on a small inverse-rendering scene
    lower the loss towards the seeded ground truth."""
    import torch

    from tinypt_b200.render import DeviceScene

    truth = scenes.inverse_params()
    start = np.clip(truth + np.random.default_rng(4).normal(0.0, 0.12, truth.shape), 0.05, 0.95)
    scene = scenes.inverse_scene(64, 64, nx=64, nz=128)
    base = scene.mats
    fwd = RenderConfig(width=64, height=64, spp=32, max_bounces=6, rr_start=3, seed=21,
                       mode=_abi.TPT_MODE_WAVEFRONT_FP32)
    adj = RenderConfig(width=64, height=64, spp=32, max_bounces=6, rr_start=3, seed=22,
                       mode=_abi.TPT_MODE_WAVEFRONT_FP32)
    tgt_cfg = RenderConfig(width=64, height=64, spp=256, max_bounces=6, rr_start=3, seed=23,
                           mode=_abi.TPT_MODE_WAVEFRONT_FP32)
    with DeviceScene(scene) as ds:
        target = torch.empty((64, 64, 3), dtype=torch.float32, device="cuda")
        ds.render_forward(tgt_cfg, target.data_ptr())
        params = torch.tensor(start, dtype=torch.float64, requires_grad=True)
        img = autodiff.RenderMaterials.apply(params, ds, base, fwd, adj)
        loss = ((img - target) ** 2).mean()
        loss.backward()
        direct = torch.empty(4 * len(base), dtype=torch.float64, device="cuda")
        dimg = (2.0 * (img.detach() - target) / img.numel()).contiguous()
        ds.render_backward(adj, dimg.data_ptr(), direct.data_ptr())
        # the two calls differ only in the order of the f32/f64 gradient sums
        dg = direct.cpu().numpy()
        assert np.allclose(params.grad.numpy().ravel(), dg, rtol=1e-5, atol=1e-9 * np.abs(dg).max())

        opt = torch.optim.Adam([params], lr=0.04)
        losses = []
        for it in range(16):
            opt.zero_grad()
            img = autodiff.RenderMaterials.apply(params, ds, base, dataclasses.replace(fwd, seed=100 + it),
                                                 dataclasses.replace(adj, seed=200 + it))
            loss = ((img - target) ** 2).mean()
            loss.backward()
            opt.step()
            with torch.no_grad():
                params.clamp_(0.02, 0.98)
            losses.append(loss.item())
        print("losses", [f"{v:.3e}" for v in losses])
        assert np.mean(losses[-3:]) < 0.9 * np.mean(losses[:3])
        err0 = np.abs(start - truth).mean()
        err1 = np.abs(params.detach().numpy() - truth).mean()
        print(f"parameter error {err0:.4f} -> {err1:.4f}")
        assert err1 < err0


@pytest.mark.gpu
@pytest.mark.parametrize("rr_start", [6, 2])
def test_wavefront_adjoint_follows_forward_paths(gpu, monkeypatch, rr_start):
    """The wavefront adjoint (one pass per sample, vertex lists) traces the
    forward form's paths: its linearised loss sum_k delta . c_k equals
    sum_p delta_p . I_p of the forward render at the same seed (f32 sums:
    2e-5).  The two-pass replay megakernel (TPT_ADJOINT=megakernel), a
    separately compiled kernel whose FP32 contractions differ, flips a few
    path decisions: its gradient agrees to 1% (plus 0.1% of the largest)
    and its path count exactly."""
    import torch

    from tinypt_b200.render import DeviceScene

    scene = scenes.gradcheck_scene(48, 48)
    cfg = gc_cfg(48, 48, spp=32, seed=11, rr_start=rr_start)
    dn = adjoint_image(cfg.width, cfg.height, 5)
    d = torch.tensor(dn, device="cuda")
    out = {}
    with DeviceScene(scene) as ds:
        img = torch.empty((cfg.height, cfg.width, 3), dtype=torch.float32, device="cuda")
        ds.render_forward(cfg, img.data_ptr())
        lin_fwd = float((img.double() * d.double()).sum())
        for form in ("wavefront", "megakernel"):
            if form == "megakernel":
                monkeypatch.setenv("TPT_ADJOINT", "megakernel")
            else:
                monkeypatch.delenv("TPT_ADJOINT", raising=False)
            grad = torch.empty(4 * ds.n_materials, dtype=torch.float64, device="cuda")
            st = ds.render_backward(cfg, d.data_ptr(), grad.data_ptr())
            assert st.device_flags == 0
            out[form] = (grad.cpu().numpy(), st.paths, st.adjoint_linear)
    gw, pw, lw = out["wavefront"]
    gm, pm, lm = out["megakernel"]
    print(f"linearised loss: forward {lin_fwd:.9e}  wavefront {lw:.9e}  megakernel {lm:.9e}")
    assert pw == pm == cfg.width * cfg.height * cfg.spp
    assert abs(lw - lin_fwd) <= 2e-5 * abs(lin_fwd)
    check_close(f"wf-vs-mk rr{rr_start}", gw, gm, 1e-2, 1e-3)


@pytest.mark.gpu
def test_adjoint_culling_changes_no_gradient(gpu, monkeypatch):
    """The backward replay culls pixels whose every camera ray leaves the
    scene, and a coherent kernel adds only their linearised-loss terms.
    Those pixels have no surface vertex, so their material gradient is
    exactly zero. The test renders the inverse-rendering scene (a
    heightfield under a sky with the horizon in view) at 96x96, 16 spp. With
    culling on and off:
    * the gradients agree to f32 summation order (1e-5 relative + 1e-7 of
      the largest);
    * the linearised loss agrees to 1e-6;
    * the path counts agree.
    Part of the samples is culled."""
    import torch

    from tinypt_b200.render import DeviceScene

    scene = scenes.inverse_scene(96, 96, nx=32, nz=64, env_w=64, env_h=32)
    cfg = RenderConfig(width=96, height=96, spp=16, max_bounces=8, rr_start=3, seed=5,
                       mode=_abi.TPT_MODE_WAVEFRONT_FP32)
    d = torch.tensor(adjoint_image(cfg.width, cfg.height, 3), device="cuda")
    out = {}
    with DeviceScene(scene) as ds:
        for cull in ("0", "1"):
            monkeypatch.setenv("TPT_SKY_CULL", cull)
            grad = torch.empty(4 * ds.n_materials, dtype=torch.float64, device="cuda")
            st = ds.render_backward(cfg, d.data_ptr(), grad.data_ptr())
            assert st.device_flags == 0
            out[cull] = (grad.cpu().numpy(), st.paths, st.adjoint_linear, st.sky_samples)
    g0, p0, l0, s0 = out["0"]
    g1, p1, l1, s1 = out["1"]
    print(f"adjoint culling: culled {s1 / p1:.3f} of {p1} samples, linearised loss {l0:.9e} vs {l1:.9e}")
    assert p0 == p1 == cfg.width * cfg.height * cfg.spp
    assert s0 == 0 and 0 < s1 < p1
    assert abs(l1 - l0) <= 1e-6 * abs(l0)
    scale = float(np.abs(g0).max())
    assert np.all(np.abs(g1 - g0) <= 1e-5 * np.abs(g0) + 1e-7 * scale)
