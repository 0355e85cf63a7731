"""Material-parameter gradients: torch.autograd wrapper and finite differences.

The reference renders only.  ``render_backward`` (C ABI
``tpt_render_backward_device``) is a path-replay adjoint of the FP32 form;
this module exposes it as a ``torch.autograd.Function`` for the
gradient-check harness and for inverse rendering, and provides the
central-difference estimate it is checked against.

Parameters are an (n_materials, 4) float64 array: rgb (albedo, Dielectric
absorption, DiffuseLight emission) and param (GGX alpha; the gradient of a
Dielectric ior or Subsurface scatter_dist is 0).
"""
from __future__ import annotations

from typing import Iterable, Sequence

import numpy as np

from .render import DeviceScene
from .scene import Material, RenderConfig


def params_of(materials: Sequence[Material]) -> np.ndarray:
    return np.array([[*m.rgb, m.param] for m in materials], dtype=np.float64)


def materials_with(base: Sequence[Material], params) -> list:
    p = np.asarray(params, dtype=np.float64).reshape(len(base), 4)
    return [Material(m.kind, (float(r[0]), float(r[1]), float(r[2])), float(r[3])) for m, r in zip(base, p)]


def _torch():
    import torch

    return torch


class RenderMaterials:
    """``image = RenderMaterials.apply(params, ds, base, cfg_forward, cfg_adjoint)``:
    the FP32 forward render of the scene with its materials set from
    ``params`` (float64 (n, 4), any device); the backward pass runs the
    adjoint render with ``cfg_adjoint`` (a seed other than the forward's gives
    an estimate independent of the forward image)."""

    _fn = None

    @classmethod
    def apply(cls, params, ds: DeviceScene, base: Sequence[Material], cfg_forward: RenderConfig,
              cfg_adjoint: RenderConfig):
        if cls._fn is None:
            cls._fn = _make_function()
        return cls._fn.apply(params, ds, list(base), cfg_forward, cfg_adjoint)


def _make_function():
    torch = _torch()

    class _Render(torch.autograd.Function):
        @staticmethod
        def forward(ctx, params, ds, base, cfg_forward, cfg_adjoint):
            ds.set_materials(materials_with(base, params.detach().cpu().numpy()))
            img = torch.empty((cfg_forward.height, cfg_forward.width, 3), dtype=torch.float32, device="cuda")
            ds.render_forward(cfg_forward, img.data_ptr())
            ctx.ds, ctx.cfg_adjoint = ds, cfg_adjoint
            ctx.n, ctx.p_device, ctx.p_dtype = len(base), params.device, params.dtype
            return img

        @staticmethod
        def backward(ctx, grad_img):
            torch_ = _torch()
            g_img = grad_img.detach().to(device="cuda", dtype=torch_.float32).contiguous()
            grad = torch_.empty(4 * ctx.n, dtype=torch_.float64, device="cuda")
            ctx.ds.render_backward(ctx.cfg_adjoint, g_img.data_ptr(), grad.data_ptr())
            return grad.view(ctx.n, 4).to(device=ctx.p_device, dtype=ctx.p_dtype), None, None, None, None

    return _Render


def fd_gradient(ds: DeviceScene, base: Sequence[Material], cfg: RenderConfig, dimage, indices: Iterable,
                h: float = 1e-3) -> np.ndarray:
    """Central differences of sum(dimage * image) with common random numbers:
    for each flat parameter index k (material k // 4, component k % 4), two
    forward renders at the same seed with parameter k at +-h and sampling
    held at the base materials (detached sampling, tpt_scene_set_materials).
    dimage: CUDA float32 (height, width, 3).  Returns one value per index.
    The scene's materials are restored to ``base`` afterwards."""
    torch = _torch()
    p0 = params_of(base)
    n = cfg.width * cfg.height
    acc = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    acc_w = torch.empty(n, dtype=torch.float64, device="cuda")
    d64 = dimage.to(torch.float64).reshape(n, 3)

    def image(params):
        ds.set_materials(materials_with(base, params), sampling_materials=base)
        ds.render_device(cfg, acc.data_ptr(), acc_w.data_ptr())
        return acc.view(n, 3) / acc_w.clamp(min=1.0)[:, None]

    out = []
    try:
        for k in indices:
            pp, pm = p0.copy(), p0.copy()
            pp.flat[k] += h
            pm.flat[k] -= h
            diff = image(pp) - image(pm)
            out.append(float((d64 * diff).sum().item()) / (2.0 * h))
    finally:
        ds.set_materials(list(base))
    return np.array(out)


def fd_gradient_adjoint_paths(ds: DeviceScene, base: Sequence[Material], cfg: RenderConfig, dimage,
                              indices: Iterable, h: float = 1e-3) -> np.ndarray:
    """Central differences of the linearised loss that the adjoint render
    reports for its own paths (RenderStats.adjoint_linear), at +-h with
    sampling held at ``base``: common random numbers path for path with the
    adjoint itself."""
    torch = _torch()
    p0 = params_of(base)
    grad = torch.empty(4 * len(base), dtype=torch.float64, device="cuda")
    d = dimage.to(device="cuda", dtype=torch.float32).contiguous()

    def lin(params):
        ds.set_materials(materials_with(base, params), sampling_materials=base)
        return ds.render_backward(cfg, d.data_ptr(), grad.data_ptr()).adjoint_linear

    out = []
    try:
        for k in indices:
            pp, pm = p0.copy(), p0.copy()
            pp.flat[k] += h
            pm.flat[k] -= h
            out.append((lin(pp) - lin(pm)) / (2.0 * h))
    finally:
        ds.set_materials(list(base))
    return np.array(out)


def oracle_fd_gradient(oscene, base: Sequence[Material], cfg: RenderConfig, dimage: np.ndarray, indices: Iterable,
                       h: float = 1e-3, threads: int = 0) -> np.ndarray:
    """The same central differences computed by the f64 CPU oracle (an
    ``oracle.oracle.OracleScene``): the f64 reference gradient."""
    p0 = params_of(base)
    d = np.asarray(dimage, dtype=np.float64).reshape(-1, 3)

    def image(params):
        oscene.set_materials(materials_with(base, params), sampling_materials=base)
        acc, acc_w, _, _ = oscene.render(cfg, threads=threads)
        return acc / np.maximum(acc_w, 1.0)[:, None]

    out = []
    try:
        for k in indices:
            pp, pm = p0.copy(), p0.copy()
            pp.flat[k] += h
            pm.flat[k] -= h
            out.append(float(np.sum(d * (image(pp) - image(pm)))) / (2.0 * h))
    finally:
        oscene.set_materials(list(base))
    return np.array(out)
