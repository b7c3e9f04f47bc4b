"""ORACLE -- test infrastructure, not product code.

ctypes wrapper of oracle/_ref/libnoor_refdev.so: the reference's own device
routines (noor/cuda/*.cuh) compiled unmodified by nvcc for sm_100a with
-fmad=false behind the harness in oracle/refdev/refdev.cu.  It needs a GPU to
run.  Only tests/ and tests/golden/make_refdev_golden.py use it, as the
checker: fixtures frozen from it pin the CPU restatement
(oracle/noor_oracle.cpp) and the product's CUDA routines.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .oracle import REFDEV_SO

_lib = None


def available() -> bool:
    return REFDEV_SO.exists()


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not REFDEV_SO.exists():
            raise FileNotFoundError(f"{REFDEV_SO} not built (make -C oracle refdev, needs the reference tree)")
        L = C.CDLL(str(REFDEV_SO))
        vp, sz = C.c_void_p, C.c_size_t
        L.refdev_last_error.restype = C.c_char_p
        L.refdev_load.argtypes = [vp, vp, vp, vp, vp]
        L.refdev_render.argtypes = [C.c_uint32, C.c_uint32, vp]
        L.refdev_trace.argtypes = [C.c_int, vp, vp, sz]
        L.refdev_camera_rays.argtypes = [C.c_uint32, vp]
        L.refdev_bsdf.argtypes = [C.c_int, vp, vp, sz]
        L.refdev_microfacet.argtypes = [C.c_int, vp, vp, sz]
        L.refdev_fresnel.argtypes = [vp, vp, sz]
        L.refdev_warps.argtypes = [vp, vp, sz]
        L.refdev_sky.argtypes = [C.c_int, vp, vp, vp, sz]
        L.refdev_env_sample.argtypes = [vp, vp, sz]
        L.refdev_env_distribution.argtypes = [vp, vp, vp, vp]
        L.refdev_rng.argtypes = [vp, sz, C.c_int, vp, vp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"{what}: {lib().refdev_last_error().decode()}")


def _batch(fn: str, arr: np.ndarray, out_cols: int, *lead):
    a = np.ascontiguousarray(arr, np.float32)
    out = np.zeros((a.shape[0], out_cols), np.float32)
    _check(getattr(lib(), fn)(*lead, _p(a), _p(out), a.shape[0]), fn)
    return out


def rng(seeds: np.ndarray, draws: int):
    """CudaRNG(id, frame) for (n, 2) uint32 seeds: the TEA<16> seed words and
    `draws` LCG floats each"""
    s = np.ascontiguousarray(seeds, np.uint32)
    n = s.shape[0]
    seed = np.zeros(n, np.uint32)
    out = np.zeros((n, draws), np.float32)
    _check(lib().refdev_rng(_p(s), n, draws, _p(seed), _p(out)), "refdev_rng")
    return seed, out


def microfacet(beckmann: bool, rec: np.ndarray) -> np.ndarray:
    """rec (n, 12): roughness[2], wo[3], wh[3], u[2]; returns (n, 12):
    D(wh), G(wo, wh), Pdf(wo, wh), Sample_wh(wo, u)[3], 0, alpha_x"""
    return _batch("refdev_microfacet", rec, 12, int(beckmann))


def fresnel(rec: np.ndarray) -> np.ndarray:
    """rec (n, 9): cos, etaI, etaT, eta[3], k[3]; returns (n, 4): dielectric
    F and conductor F[3] (etaI 1)"""
    return _batch("refdev_fresnel", rec, 4)


def warps(rec: np.ndarray) -> np.ndarray:
    """rec (n, 3): u[2], x; returns (n, 16): concentric disk[2], cosine
    hemisphere[3], uniform hemisphere[3] (both local z up), spherical
    direction[3] + sinTheta, power heuristic(u.x, u.y), Erf(x), ErfInv(x), -"""
    return _batch("refdev_warps", rec, 16)


def sky_query(hosek, dirs: np.ndarray) -> np.ndarray:
    """querySkyModel of a noor_hosek_sky for unit directions (n, 3)"""
    d = np.ascontiguousarray(dirs, np.float32)
    out = np.zeros((d.shape[0], 3), np.float32)
    _check(lib().refdev_sky(0, C.addressof(hosek), _p(d), _p(out), d.shape[0]), "refdev_sky")
    return out


class RefDevice:
    """One scene loaded into the reference's managers (the harness keeps one
    at a time).  Renders run with MIS off: the reference's MIS path reads an
    unset light index."""

    def __init__(self, payload, hosek, camera, spec):
        self._keep = (payload, hosek, camera, spec)
        slice_ = C.c_uint32()
        _check(lib().refdev_load(C.addressof(payload), C.addressof(hosek), C.addressof(camera), C.addressof(spec),
                                 C.addressof(slice_)), "refdev_load")
        self.stack_slice = slice_.value
        self.w, self.h = int(camera.w), int(camera.h)

    def close(self):
        lib().refdev_free()

    def render(self, first_frame: int, n_frames: int) -> np.ndarray:
        film = np.zeros((self.h, self.w, 4), np.float32)
        _check(lib().refdev_render(first_frame, n_frames, _p(film)), "refdev_render")
        return film

    def trace_closest(self, rays: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(rays, np.float32)
        out = np.zeros((r.shape[0], 8), np.uint32)
        _check(lib().refdev_trace(0, _p(r), _p(out), r.shape[0]), "refdev_trace")
        return out

    def trace_any(self, rays: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(rays, np.float32)
        out = np.zeros(r.shape[0], np.uint32)
        _check(lib().refdev_trace(1, _p(r), _p(out), r.shape[0]), "refdev_trace")
        return out

    def camera_rays(self, frame: int) -> np.ndarray:
        out = np.zeros((self.w * self.h, 8), np.float32)
        _check(lib().refdev_camera_rays(frame, _p(out)), "refdev_camera_rays")
        return out

    def bsdf(self, kind: int, rec: np.ndarray) -> np.ndarray:
        """rec (n, 16): wo_local[3], wi_local[3], probe origin[3], probe
        dir[3], seed id, seed frame; returns (n, 12): f[3], pdf,
        wi_local[3], sampled type, the two uniforms Sample_f drew, hit,
        material index"""
        return _batch("refdev_bsdf", rec, 12, kind)

    def sky(self, dirs: np.ndarray) -> np.ndarray:
        """the sky dome's evaluate(dir) (Hosek for the physical sky, the
        texture unit's bilinear for an HDR map)"""
        d = np.ascontiguousarray(dirs, np.float32)
        out = np.zeros((d.shape[0], 3), np.float32)
        _check(lib().refdev_sky(1, None, _p(d), _p(out), d.shape[0]), "refdev_sky")
        return out

    def env_sample(self, u: np.ndarray) -> np.ndarray:
        """u (n, 2) -> (n, 4): x, y, pdf of the sample, Pdf(x, y)"""
        return _batch("refdev_env_sample", u, 4)

    def env_distribution(self):
        """the sky dome's CudaDistribution2D arrays: w, h and func, cdf as
        (h + 1, w + 1) tables (row r: w values then the row integral; row h:
        the marginal's h values then its integral, padded)"""
        w, h = C.c_int(), C.c_int()
        _check(lib().refdev_env_distribution(C.addressof(w), C.addressof(h), None, None), "refdev_env_distribution")
        W, H = w.value, h.value
        n = H * (W + 2) + 1
        func = np.zeros(n, np.float32)
        cdf = np.zeros(n, np.float32)
        _check(lib().refdev_env_distribution(None, None, _p(func), _p(cdf)), "refdev_env_distribution")
        return W, H, func, cdf
