"""Differentiable rendering of the loaded scene (scene 0 of the current
context) through the path-replay adjoint entry points
noor_adjoint_forward / noor_adjoint_backward, as a torch.autograd.Function:

    image = render(albedo, roughness, env, width, height, spp)

albedo (M, 3) is the Lambert reflectance or the conductor tint of each
material, roughness (M,) the microfacet roughness (alpha = max(r^2, 1e-3)),
env (H, W, 3) the environment texels; all float32 CUDA tensors.  The image
is (height, width, 3), the mean over `spp` samples of the clamped radiance.

The estimator is differentiated with its sampling detached: directions,
light picks, MIS weights and pdfs come from the scene as loaded, so the
parameters the scene was loaded with are the point the sampling is good
for (reload the scene with new parameters to move it).  Russian roulette
must be off (spec.rr >= bounces).  Albedo channels must stay non-zero: the
replay recovers the radiance after a vertex by division by that vertex's
BSDF value.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi


def _ptr(t: torch.Tensor):
    return C.cast(C.c_void_p(t.data_ptr()), _capi.pf)


def _check(name: str, t: torch.Tensor, shape) -> None:
    if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
        raise ValueError(f"{name} must be a contiguous float32 CUDA tensor")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")


def _desc(cfg, albedo, roughness, env) -> _capi.AdjointDesc:
    width, height, spp, first_frame, bounces = cfg
    d = _capi.AdjointDesc()
    d.width, d.height, d.spp, d.first_frame, d.bounces = width, height, spp, first_frame, bounces
    d.d_albedo, d.d_roughness = _ptr(albedo), _ptr(roughness)
    d.d_env = _ptr(env) if env is not None and env.numel() else _capi.pf()
    return d


class AdjointRender(torch.autograd.Function):
    """forward: noor_adjoint_forward; backward: noor_adjoint_backward.
    The library runs on its own stream and returns after its work is done;
    torch's current stream is synchronised before each call so that the
    inputs are complete."""

    @staticmethod
    def forward(ctx, albedo, roughness, env, width: int, height: int, spp: int, first_frame: int = 1,
                bounces: int = 0):
        M = albedo.shape[0]
        _check("albedo", albedo, (M, 3))
        _check("roughness", roughness, (M,))
        if env is not None and env.numel():
            _check("env", env, (env.shape[0], env.shape[1], 3))
        cfg = (int(width), int(height), int(spp), int(first_frame), int(bounces))
        img = torch.empty((height, width, 3), device=albedo.device, dtype=torch.float32)
        torch.cuda.current_stream(albedo.device).synchronize()
        d = _desc(cfg, albedo, roughness, env)
        _capi.call("noor_adjoint_forward", C.byref(d), C.c_void_p(img.data_ptr()))
        ctx.save_for_backward(albedo, roughness, env)
        ctx.cfg = cfg
        # autograd may run backward on a worker thread: remember the render
        # context (contexts are per host thread) to borrow it there
        ctx.noor_context = _capi.lib().noor_context_current()
        return img

    @staticmethod
    def backward(ctx, grad_img):
        albedo, roughness, env = ctx.saved_tensors
        g = grad_img.contiguous().to(torch.float32)
        ga = torch.zeros_like(albedo)
        gr = torch.zeros_like(roughness)
        ge = torch.zeros_like(env) if env is not None and env.numel() else None
        torch.cuda.current_stream(albedo.device).synchronize()
        d = _desc(ctx.cfg, albedo, roughness, env)
        prev = _capi.lib().noor_context_current()
        _capi.call("noor_context_bind", ctx.noor_context)
        try:
            _capi.call("noor_adjoint_backward", C.byref(d), C.c_void_p(g.data_ptr()), C.c_void_p(ga.data_ptr()),
                       C.c_void_p(gr.data_ptr()), C.c_void_p(ge.data_ptr()) if ge is not None else None)
        finally:
            _capi.call("noor_context_bind", prev)
        return ga, gr, ge, None, None, None, None, None


def render(albedo: torch.Tensor, roughness: torch.Tensor, env: torch.Tensor, width: int, height: int, spp: int,
           first_frame: int = 1, bounces: int = 0) -> torch.Tensor:
    """Differentiable render of the current context's scene 0."""
    return AdjointRender.apply(albedo, roughness, env, width, height, spp, first_frame, bounces)


def scene_parameters(scene, device: str = "cuda"):
    """(albedo (M,3), roughness (M,), env (H,W,3)) float32 tensors holding the
    values a SceneData was built with: the diffuse colour of Lambert
    materials, the specular tint of the others, roughness[0], env rgb."""
    alb = np.zeros((len(scene.materials), 3), np.float32)
    rough = np.zeros(len(scene.materials), np.float32)
    for i, m in enumerate(scene.materials):
        alb[i] = m["diffuse"] if m["type"] == _capi.NOOR_DIFFUSE else m["specular"]
        rough[i] = m["roughness"][0]
    env = np.zeros((0, 0, 3), np.float32) if scene.env is None else np.ascontiguousarray(scene.env[..., :3])
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(device)
    return t(alb), t(rough), t(env)
