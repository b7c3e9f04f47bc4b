"""ORACLE -- test infrastructure, not product code.

ctypes loader for the CPU restatement (oracle/_build/liboracle.so, built from
noor_oracle.cpp) and for the reference's own host routines compiled from the
reference tree (oracle/_ref/libnoor_ref.so).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import importlib
import math
import subprocess
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libnoor_ref.so"
REFDEV_SO = HERE / "_ref" / "libnoor_refdev.so"


def reference_tree() -> Path:
    """the reference tree the recipe reads ($NOOR_REFERENCE, else the
    recipe's default)"""
    out = subprocess.run(["make", "-s", "-C", str(HERE), "ref-path"], check=True, capture_output=True, text=True)
    return Path(out.stdout.strip())


def build(ref: bool = True) -> None:
    """make the oracle and, when the reference tree is present, oracle/_ref
    (the reference's host routines and its device routines)"""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    if ref and (reference_tree() / "noor").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", "refdev"], check=True)


_orc = None
_ref = None


def lib() -> C.CDLL:
    global _orc
    if _orc is None:
        if not ORACLE_SO.exists():
            build(ref=False)
        L = C.CDLL(str(ORACLE_SO))
        vp, sz = C.c_void_p, C.c_size_t
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [vp, vp, vp]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_trace_closest.argtypes = [vp, vp, vp, sz, C.c_int, C.c_int]
        L.oracle_trace_any.argtypes = [vp, vp, vp, sz, C.c_int]
        L.oracle_camera_rays.argtypes = [vp, C.c_uint32, vp]
        L.oracle_render.argtypes = [vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, vp, C.c_int, C.c_int,
                                    C.c_int, vp, vp]
        L.oracle_eval_bsdf.argtypes = [vp, C.c_int, vp, vp, sz, C.c_int]
        L.oracle_eval_sky.argtypes = [vp, vp, vp, sz, C.c_int]
        L.oracle_env_distribution.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
        L.oracle_env_sample.argtypes = [vp, vp, vp, sz]
        L.oracle_adjoint.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, vp, vp, vp, C.c_int, C.c_int,
                                     vp, vp, vp, vp]
        L.oracle_env_footprint.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, vp, vp, C.c_int, C.c_int,
                                           vp]
        L.oracle_routines.argtypes = [C.c_int, vp, vp, sz, C.c_int]
        L.oracle_rng.argtypes = [vp, sz, C.c_int, vp, vp]
        L.oracle_ref_dist_sample.argtypes = [vp, vp, C.c_int, C.c_int, vp, vp, sz]
        L.oracle_tea16.restype = C.c_uint32
        L.oracle_tea16.argtypes = [C.c_uint32, C.c_uint32]
        _orc = L
    return _orc


def ref_available() -> bool:
    return REF_SO.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (needs the reference tree)")
        L = C.CDLL(str(REF_SO))
        vp = C.c_void_p
        L.ref_build_bvh.restype = C.c_int
        L.ref_build_bvh.argtypes = [vp, vp, C.c_size_t, vp, vp, vp, vp]
        L.ref_wald.argtypes = [vp, vp]
        L.ref_hosek_state.argtypes = [C.c_float, C.c_float, C.c_float, vp]
        L.ref_hosek_dataset.argtypes = [vp]
        L.ref_build_payload.restype = vp
        L.ref_build_payload.argtypes = [vp]
        L.ref_payload_view.argtypes = [vp, vp]
        L.ref_payload_spec.argtypes = [vp, C.c_uint32, C.c_uint32, vp]
        L.ref_free_payload.argtypes = [vp]
        _ref = L
    return _ref


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def host_modules():
    """noor_b200/_capi.py (the C-ABI's struct layouts) and noor_b200/scenes.py
    (the seeded scene generators) as modules of a bare package: the
    package's __init__, which loads the product library, does not run.  The
    bench's reference arm builds its workload through these and the
    reference builder alone."""
    name = "_noor_b200_host"
    if name not in sys.modules:
        pkg = types.ModuleType(name)
        pkg.__path__ = [str(HERE.parent / "noor_b200")]
        sys.modules[name] = pkg
    return importlib.import_module(name + "._capi"), importlib.import_module(name + ".scenes")


class RefPayload:
    """A scene's payload from the reference's own BVH builder and Wald
    records (oracle/_ref/libnoor_ref.so, ref_build_payload), with the spec
    Scene::load derives.  `capi` and `scenes` are the modules of
    host_modules() or of the product package (only their struct layouts and
    scene description are used)."""

    def __init__(self, scene, capi, scenes):
        self.capi = capi
        self.desc, self._keep = scenes.scene_desc(scene)
        self.h = ref().ref_build_payload(C.addressof(self.desc))
        self.payload = capi.Payload()
        ref().ref_payload_view(self.h, C.addressof(self.payload))

    def default_spec(self, bounces: int, rr: int):
        sp = self.capi.Spec()
        ref().ref_payload_spec(self.h, bounces, rr, C.addressof(sp))
        return sp

    def free(self):
        if self.h:
            ref().ref_free_payload(self.h)
            self.h = None


def camera_lookat(capi, cam: dict):
    """A pinhole camera as Camera's constructor and CudaCamera::update build
    it (noor/header/camera.h:99-153,255-334; noor/cuda/camera.cuh:66-94),
    evaluated in FP64 and rounded once: cameraToWorld = translate(lookAt) *
    [right, up, forward] * translate(0, 0, |eye - lookAt|); rasterToCamera
    maps the raster onto the screen window (+-aspect x +-1, or +-1 x
    +-1/aspect) on the plane z = -1 scaled by 1/cot(fov/2).  Perspective
    cameras only."""
    if cam.get("type", "persp") != "persp" or cam.get("lens_radius", 0.0):
        raise ValueError("camera_lookat: pinhole perspective cameras only")
    f32 = lambda x: float(np.float32(x))
    eye = [f32(x) for x in cam["eye"]]
    at = [f32(x) for x in cam["look_at"]]
    up = [f32(x) for x in cam["up"]]
    fov = f32(math.radians(cam["fov_deg"]))
    w, h = int(cam["w"]), int(cam["h"])
    fwd = [eye[k] - at[k] for k in range(3)]
    scale = math.sqrt(sum(x * x for x in fwd))
    fwd = [x / scale for x in fwd]
    right = [up[1] * fwd[2] - up[2] * fwd[1], up[2] * fwd[0] - up[0] * fwd[2], up[0] * fwd[1] - up[1] * fwd[0]]
    rl = math.sqrt(sum(x * x for x in right))
    right = [x / rl for x in right]
    out = capi.Camera()
    for r in range(3):
        out.camera_to_world[r][:] = [right[r], up[r], fwd[r], at[r] + fwd[r] * scale]
    aspect = w / h
    smin, smax = ((-aspect, -1.0), (aspect, 1.0)) if aspect > 1.0 else ((-1.0, -1.0 / aspect), (1.0, 1.0 / aspect))
    cot = 1.0 / math.tan(fov / 2.0)
    sx, sy = (smax[0] - smin[0]) / w / cot, (smax[1] - smin[1]) / h / cot
    out.raster_to_camera[0][:] = [sx, 0.0, 0.0, smin[0] / cot]
    out.raster_to_camera[1][:] = [0.0, sy, 0.0, smin[1] / cot]
    out.raster_to_camera[2][:] = [0.0, 0.0, 0.0, -1.0]
    out.dx_camera[:] = [sx, 0.0, 0.0]
    out.dy_camera[:] = [0.0, sy, 0.0]
    out.image_area = abs((smax[0] - smin[0]) / cot * (smax[1] - smin[1]) / cot)
    out.lens_radius = 0.0
    out.focal_length = scale
    out.w, out.h = w, h
    out.center = w * (h >> 1) + (w >> 1)
    out.type = capi.NOOR_CAMERA_PERSP
    return out


class Oracle:
    """CPU restatement over the same payload/spec/sky structs the library uses."""

    def __init__(self, payload, spec, hosek):
        self._refs = (payload, spec, hosek)
        self.h = lib().oracle_create(C.addressof(payload), C.addressof(spec), C.addressof(hosek))

    def close(self):
        if self.h:
            lib().oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def trace_closest(self, rays: np.ndarray, isect: int, threads: int = 8) -> np.ndarray:
        hits = np.zeros(rays.shape[0] * 8, np.uint32)
        lib().oracle_trace_closest(self.h, _p(rays), _p(hits), rays.shape[0], isect, threads)
        return hits.reshape(-1, 8)

    def trace_any(self, rays: np.ndarray, isect: int) -> np.ndarray:
        occ = np.zeros(rays.shape[0], np.uint32)
        lib().oracle_trace_any(self.h, _p(rays), _p(occ), rays.shape[0], isect)
        return occ

    def render(self, camera, frame0: int, nframes: int, p0: int = 0, p1: int = None, fp64: bool = False,
               isect: int = 0, threads: int = 8, counters: bool = False):
        if p1 is None:
            p1 = camera.w * camera.h
        out = np.zeros((p1 - p0) * 3, np.float32)
        ctr = np.zeros(8, np.uint64)  # ext, shadow, nodes, tris, in range (all rays); the last three of shadow rays
        lib().oracle_render(self.h, frame0, nframes, p0, p1, C.addressof(camera), int(fp64), isect, threads,
                            _p(out), _p(ctr) if counters else None)
        out = out.reshape(-1, 3)
        return (out, ctr) if counters else out

    def eval_bsdf(self, kind: int, recs: np.ndarray, fp64: bool = False) -> np.ndarray:
        out = np.zeros(recs.shape[0] * 8, np.float32)
        lib().oracle_eval_bsdf(self.h, kind, _p(recs), _p(out), recs.shape[0], int(fp64))
        return out.reshape(-1, 8)

    def eval_sky(self, dirs: np.ndarray, fp64: bool = False) -> np.ndarray:
        out = np.zeros(dirs.shape[0] * 3, np.float32)
        lib().oracle_eval_sky(self.h, _p(dirs), _p(out), dirs.shape[0], int(fp64))
        return out.reshape(-1, 3)

    def env_distribution(self):
        w, h = C.c_int(), C.c_int()
        lib().oracle_env_distribution(self.h, C.addressof(w), C.addressof(h), None, None, None, None, None)
        W, H = w.value, h.value
        func = np.zeros(W * H)
        cdf = np.zeros(H * (W + 1))
        row = np.zeros(H)
        mcdf = np.zeros(H + 1)
        mi = C.c_double()
        lib().oracle_env_distribution(self.h, None, None, _p(func), _p(cdf), _p(row), _p(mcdf), C.addressof(mi))
        return dict(w=W, h=H, func=func.reshape(H, W), cdf=cdf.reshape(H, W + 1), row_int=row, marg_cdf=mcdf,
                    marg_int=mi.value)

    def adjoint(self, camera, frame0: int, spp: int, bounces: int, albedo: np.ndarray, roughness: np.ndarray,
                env: np.ndarray, grad_img: np.ndarray = None, isect: int = 0, threads: int = 8):
        """FP64 detached-sampling estimator: image (h*w, 3) and, when grad_img
        is given, the gradients of sum(grad_img * image) w.r.t. albedo (M,3),
        roughness (M,) and env texels (H,W,3)."""
        alb = np.ascontiguousarray(albedo, np.float32)
        rough = np.ascontiguousarray(roughness, np.float32)
        env3 = np.ascontiguousarray(env, np.float32)
        npix = camera.w * camera.h
        img = np.zeros((npix, 3))
        ga = np.zeros(alb.shape)
        gr = np.zeros(rough.shape)
        ge = np.zeros(env3.shape)
        gi = None if grad_img is None else np.ascontiguousarray(grad_img, np.float32)
        lib().oracle_adjoint(self.h, C.addressof(camera), frame0, spp, bounces, _p(alb), _p(rough), _p(env3),
                             None if gi is None else _p(gi), isect, threads, _p(img), _p(ga), _p(gr), _p(ge))
        return (img, ga, gr, ge) if gi is not None else img

    def env_footprint(self, camera, frame0: int, spp: int, bounces: int, albedo: np.ndarray,
                      roughness: np.ndarray, env: np.ndarray, isect: int = 0, threads: int = 8) -> np.ndarray:
        """(H, W) counts of the forward paths' radiance lookups per env
        texel (oracle_env_footprint): the texels the image depends on"""
        env3 = np.ascontiguousarray(env, np.float32)
        out = np.zeros(env3.shape[:2], np.uint32)
        lib().oracle_env_footprint(self.h, C.addressof(camera), frame0, spp, bounces,
                                   _p(np.ascontiguousarray(albedo, np.float32)),
                                   _p(np.ascontiguousarray(roughness, np.float32)), _p(env3), isect, threads, _p(out))
        return out

    def env_sample(self, u: np.ndarray) -> np.ndarray:
        out = np.zeros(u.shape[0] * 4)
        lib().oracle_env_sample(self.h, _p(np.ascontiguousarray(u, np.float32)), _p(out), u.shape[0])
        return out.reshape(-1, 4)


def rng(pairs: np.ndarray, draws: int):
    """CudaRNG(id, frame) of (n, 2) uint32 pairs: seed words and `draws`
    floats each"""
    p = np.ascontiguousarray(pairs, np.uint32)
    seed = np.zeros(p.shape[0], np.uint32)
    out = np.zeros((p.shape[0], draws), np.float32)
    lib().oracle_rng(_p(p), p.shape[0], draws, _p(seed), _p(out))
    return seed, out


def ref_dist_sample(func: np.ndarray, cdf: np.ndarray, w: int, h: int, u: np.ndarray) -> np.ndarray:
    """the reference's CudaDistribution2D sampling on its tables (h*(w+2)+1
    floats each, plus padding): u (n, 2) -> (n, 4) x, y, pdf, Pdf(x, y)"""
    pad = lambda a: np.concatenate([np.ascontiguousarray(a, np.float32), np.zeros(2, np.float32)])
    f, c = pad(func), pad(cdf)
    uu = np.ascontiguousarray(u, np.float32)
    out = np.zeros((uu.shape[0], 4), np.float32)
    lib().oracle_ref_dist_sample(_p(f), _p(c), int(w), int(h), _p(uu), _p(out), uu.shape[0])
    return out


def routines(kind: int, rec: np.ndarray, fp64: bool = False) -> np.ndarray:
    """the stand-alone shading routines in noor_eval_routines' record
    layouts: 0 / 1 Trowbridge-Reitz / Beckmann, 2 Fresnel, 3 warps"""
    r = np.ascontiguousarray(rec, np.float32)
    out = np.zeros((r.shape[0], 12 if kind <= 1 else (4 if kind == 2 else 16)), np.float32)
    lib().oracle_routines(kind, _p(r), _p(out), r.shape[0], int(fp64))
    return out


def ref_build_bvh(desc, num_triangles: int):
    """nodes (n,8) u32, root, triangle order, height from the reference builder"""
    L = ref()
    n = C.c_uint32()
    root = C.c_uint32()
    height = C.c_uint32()
    order = np.zeros(num_triangles, np.uint32)
    rc = L.ref_build_bvh(C.addressof(desc), None, 0, C.addressof(n), C.addressof(root), _p(order),
                         C.addressof(height))
    nodes = np.zeros(n.value * 8, np.uint32)
    rc = L.ref_build_bvh(C.addressof(desc), _p(nodes), n.value, C.addressof(n), C.addressof(root), _p(order),
                         C.addressof(height))
    assert rc == 0
    return nodes.reshape(-1, 8), root.value, order, height.value


def ref_wald(v9: np.ndarray) -> np.ndarray:
    out = np.zeros(12, np.uint32)
    ref().ref_wald(_p(np.ascontiguousarray(v9, np.float32)), _p(out))
    return out


def ref_hosek_state(turbidity: float, albedo: float, elevation: float) -> np.ndarray:
    out = np.zeros(30, np.float32)
    ref().ref_hosek_state(turbidity, albedo, elevation, _p(out))
    return out


def ref_hosek_dataset() -> np.ndarray:
    out = np.zeros(3 * 1080 + 3 * 120, np.float32)
    ref().ref_hosek_dataset(_p(out))
    return out


# ------------------------------------------------- display (noor/shader/cuda.fs)
def tonemap(film: np.ndarray, op: int, exposure: float = 1.0) -> np.ndarray:
    """The display shader's transforms (noor/shader/cuda.fs:36-78) in FP32
    numpy: op 0 gammaCorrect (c^(1/2.2)), 1 tonemapReinhard, 2 tonemapFilmic
    (Hejl-Burgess-Dawson, gamma included), 3 tonemapUncharted2 (Hable's
    curve, exposure bias 4, white 11.2); then an 8-bit unorm store (clamp to
    [0, 1], round to nearest).  film: (..., 4) float; returns (..., 4) uint8
    with alpha 255."""
    f32 = np.float32
    c = f32(exposure) * np.asarray(film, f32)[..., :3]
    g = f32(1.0) / f32(2.2)
    with np.errstate(invalid="ignore", divide="ignore"):
        if op == 1:
            out = np.power(c / (c + f32(1)), g)
        elif op == 2:
            x = np.maximum(f32(0), c - f32(0.004))
            out = (x * (f32(6.2) * x + f32(0.5))) / (x * (f32(6.2) * x + f32(1.7)) + f32(0.06))
        elif op == 3:
            A, B, Cc, D, E, F = (f32(v) for v in (0.15, 0.50, 0.10, 0.20, 0.02, 0.30))

            def hable(x):
                return ((x * (A * x + Cc * B) + D * E) / (x * (A * x + B) + D * F)) - E / F
            ws = f32(1) / hable(f32(11.2))
            out = np.power(hable(f32(4) * c) * ws, g)
        else:
            out = np.power(c, g)
    out = np.nan_to_num(out.astype(f32), nan=0.0)
    q = np.rint(np.clip(out, 0, 1) * f32(255)).astype(np.uint8)
    alpha = np.full(q.shape[:-1] + (1,), 255, np.uint8)
    return np.concatenate([q, alpha], axis=-1)
