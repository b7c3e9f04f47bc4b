"""Helpers shared by the GPU tests: device buffers through torch (plumbing
only) and the oracle over the same payload."""
import ctypes as C
import os

import numpy as np
import torch

from noor_b200 import _capi, scenes

THREADS = max(1, min(16, os.cpu_count() or 1))


def dev(a: np.ndarray) -> torch.Tensor:
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    torch.cuda.synchronize()
    return t


def dev_empty(nbytes: int) -> torch.Tensor:
    return torch.zeros(nbytes, dtype=torch.uint8, device="cuda")


def host(t: torch.Tensor, dtype, shape) -> np.ndarray:
    torch.cuda.synchronize()
    return t.cpu().numpy().view(dtype).reshape(shape)


def rays_to_np(rays) -> np.ndarray:
    return np.ascontiguousarray(rays, np.float32)


def camera_rays(r: scenes.Renderer, frame: int) -> np.ndarray:
    n = r.w * r.h
    buf = dev_empty(n * 32)
    _capi.call("noor_camera_rays", frame, C.c_void_p(buf.data_ptr()))
    return host(buf, np.float32, (n, 8))


def trace_closest(rays: np.ndarray) -> np.ndarray:
    d_r = dev(rays)
    d_h = dev_empty(rays.shape[0] * 32)
    _capi.call("noor_trace_closest", C.c_void_p(d_r.data_ptr()), C.c_void_p(d_h.data_ptr()), rays.shape[0])
    return host(d_h, np.uint32, (rays.shape[0], 8))


def trace_any(rays: np.ndarray) -> np.ndarray:
    d_r = dev(rays)
    d_o = dev_empty(rays.shape[0] * 4)
    _capi.call("noor_trace_any", C.c_void_p(d_r.data_ptr()), C.c_void_p(d_o.data_ptr()), rays.shape[0])
    return host(d_o, np.uint32, (rays.shape[0],))


def random_rays(rng, n, lo, hi, tmax=np.inf):
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, :3] = o
    r[:, 3] = tmax
    r[:, 4:7] = d
    return r
