"""Freezes outputs of the reference's own device routines as fixtures.

Runs on a machine with a GPU and oracle/_ref/libnoor_refdev.so built (the
reference's noor/cuda/*.cuh compiled unmodified by nvcc, oracle/refdev/):

    python tests/golden/make_refdev_golden.py [out_dir]

writes refdev_*.npz (default: next to this script).  The tests hold the CPU
restatement (oracle/noor_oracle.cpp) and the product's CUDA routines to these
files, so neither needs the reference tree or this library to run.

Fixtures:
  refdev_rng.npz        CudaRNG seeds and 16 draws for (id, frame) pairs
  refdev_micro.npz      Trowbridge-Reitz and Beckmann D, G, Pdf, Sample_wh
  refdev_fresnel.npz    dielectric and conductor Fresnel
  refdev_warps.npz      disk / hemisphere / sphere warps, power heuristic, Erf
  refdev_sky.npz        querySkyModel for the C2 sky's fitted state
  refdev_bsdf.npz       CudaBSDF Eval / Pdf / Sample_f on the probe scene
  refdev_trace.npz      closest and any hit on the room and a sphere field
  refdev_render.npz     MIS-off renders (path_tracer_kernel + pathtracer) of
                        the room, a sky-lit and an HDR-lit sphere field
  refdev_envdist.npz    the sky dome's CudaDistribution2D for an HDR map and
                        for the physical sky (sampled rows), with samples
  refdev_textures.npz   the textured room: camera-ray hits (alpha cuts) and
                        an 8-frame film (image maps, bump, differentials)
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from noor_b200 import _capi, scenes  # noqa: E402
from oracle import reference_device as rd  # noqa: E402

import refdev_probe as probe  # noqa: E402


def struct_bytes(s) -> np.ndarray:
    return np.frombuffer(bytes(s), np.uint8).copy()


def built_structs(scene, built=None):
    """payload, spec, camera and sky for a scene, as the product builds them"""
    built = built or scenes.BuiltPayload(scene)
    r = scene.render
    spec = built.default_spec(r.get("bounces", 5), r.get("rr", 1))
    spec.mis = 0
    spec.intersector = _capi.NOOR_ISECT_REF_WALD
    spec.film_mode = _capi.NOOR_FILM_REF_LERP
    cam = scenes.make_camera(scene.camera)
    hosek = scenes.make_hosek(scene.hosek)
    return built, spec, cam, hosek


def routines(out: Path):
    rng = np.random.default_rng(20261203)
    # RNG: edge ids and frames plus random pairs
    seeds = np.stack([rng.integers(0, 2 ** 32, 4096, dtype=np.uint64),
                      rng.integers(0, 2 ** 32, 4096, dtype=np.uint64)], 1).astype(np.uint32)
    seeds[:6] = [(0, 0), (0, 1), (1, 1), (2 ** 32 - 1, 1), (1920 * 1080 - 1, 64), (123456, 2 ** 32 - 1)]
    seed, draws = rd.rng(seeds, 16)
    np.savez_compressed(out / "refdev_rng.npz", seeds=seeds, seed=seed, draws=draws)

    mrec = probe.microfacet_records(rng, 8192)
    np.savez_compressed(out / "refdev_micro.npz", rec=mrec, ggx=rd.microfacet(False, mrec),
                        beckmann=rd.microfacet(True, mrec))
    frec = probe.fresnel_records(rng, 8192)
    np.savez_compressed(out / "refdev_fresnel.npz", rec=frec, out=rd.fresnel(frec))
    wrec = probe.warp_records(rng, 8192)
    np.savez_compressed(out / "refdev_warps.npz", rec=wrec, out=rd.warps(wrec))

    # the C2 sky as the product fits it (FP64 on the GPU, pinned to the
    # reference's own fit by tests/golden/hosek_states.npz)
    hosek = scenes.make_hosek(probe.HOSEK)
    d = rng.normal(size=(60000, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    sun = np.array(hosek.solar_dir[:], np.float32)
    near = sun + 0.05 * rng.normal(size=(4000, 3)).astype(np.float32)
    near /= np.linalg.norm(near, axis=1, keepdims=True)
    d = np.concatenate([d, near]).astype(np.float32)
    np.savez_compressed(out / "refdev_sky.npz", hosek=struct_bytes(hosek), dirs=d, rgb=rd.sky_query(hosek, d))


def bsdf(out: Path):
    scene = probe.probe_scene()
    built, spec, cam, hosek = built_structs(scene)
    dev = rd.RefDevice(built.payload, hosek, cam, spec)
    rng = np.random.default_rng(7)
    res = {}
    for kind in (0, 1, 2):
        rec = probe.bsdf_records(rng, 1024)
        res[f"rec{kind}"] = rec
        res[f"out{kind}"] = dev.bsdf(kind, rec)
    dev.close()
    np.savez_compressed(out / "refdev_bsdf.npz", **res)


def trace(out: Path):
    res = {}
    rng = np.random.default_rng(11)
    for name, scene in probe.trace_scenes().items():
        built, spec, cam, hosek = built_structs(scene)
        dev = rd.RefDevice(built.payload, hosek, cam, spec)
        cam_rays = np.concatenate([dev.camera_rays(1), dev.camera_rays(5)])
        lo, hi = (np.array([-0.95, 0.05, -0.95]), np.array([0.95, 1.95, 0.95])) if name == "room" else \
            (np.array([-10.0, -10.0, -10.0]), np.array([10.0, 10.0, 10.0]))
        o = rng.uniform(lo, hi, (20000, 3))
        dd = rng.normal(size=(20000, 3))
        dd /= np.linalg.norm(dd, axis=1, keepdims=True)
        rnd = np.zeros((20000, 8), np.float32)
        rnd[:, :3], rnd[:, 3], rnd[:, 4:7] = o, np.inf, dd
        rnd[10000:, 3] = rng.uniform(0.1, 5.0, 10000)
        rays = np.concatenate([cam_rays, rnd]).astype(np.float32)
        res[f"{name}_rays"] = rays
        res[f"{name}_hits"] = dev.trace_closest(rays)
        res[f"{name}_any"] = dev.trace_any(rays)
        res[f"{name}_slice"] = np.array([dev.stack_slice])
        dev.close()
    np.savez_compressed(out / "refdev_trace.npz", **res)


def render(out: Path):
    res = {}
    for name, scene in list(probe.trace_scenes().items()) + [("envfield", probe.env_field())]:
        built, spec, cam, hosek = built_structs(scene)
        dev = rd.RefDevice(built.payload, hosek, cam, spec)
        res[f"{name}_film"] = dev.render(1, 8)
        dev.close()
    np.savez_compressed(out / "refdev_render.npz", **res)


def envdist(out: Path):
    s = probe.envdist_scene()
    env = s.env
    built, spec, cam, hosek = built_structs(s)
    dev = rd.RefDevice(built.payload, hosek, cam, spec)
    W, H, func, cdf = dev.env_distribution()
    u = np.random.default_rng(5).random((20000, 2)).astype(np.float32)
    d = np.random.default_rng(6).normal(size=(20000, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    res = dict(env=env.astype(np.float32), w=W, h=H, func=func, cdf=cdf, u=u, samples=dev.env_sample(u), dirs=d,
               radiance=dev.sky(d))
    dev.close()
    # the physical sky's tables (1024 x 1024 cells): the rows probe.ENV_ROWS
    # and the marginal, and samples drawn from the whole tables
    built, spec, cam, hosek = built_structs(probe.trace_scenes()["field16"])
    dev = rd.RefDevice(built.payload, hosek, cam, spec)
    W, H, func, cdf = dev.env_distribution()
    rows = np.concatenate([(r * (W + 1) + np.arange(W + 1)) for r in probe.ENV_ROWS] +
                          [H * (W + 1) + np.arange(H + 1)])
    res.update(sky_w=W, sky_h=H, sky_func=func[rows], sky_cdf=cdf[rows], sky_samples=dev.env_sample(u))
    dev.close()
    np.savez_compressed(out / "refdev_envdist.npz", **res)


def textures(out: Path):
    """the textured room (image maps, a roughness map, a bump map with ray
    differentials, an alpha-cut panel): camera-ray hits and an 8-frame film"""
    scene = scenes.textured_room_scene()
    built, spec, cam, hosek = built_structs(scene)
    dev = rd.RefDevice(built.payload, hosek, cam, spec)
    rays = np.concatenate([dev.camera_rays(1), dev.camera_rays(3)])
    res = dict(rays=rays, hits=dev.trace_closest(rays), any=dev.trace_any(rays), film=dev.render(1, 8))
    dev.close()
    np.savez_compressed(out / "refdev_textures.npz", **res)


STEPS = (routines, bsdf, trace, render, envdist, textures)


def main():
    """python make_refdev_golden.py [out_dir] [step ...] (all steps by default)"""
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent
    out.mkdir(parents=True, exist_ok=True)
    names = sys.argv[2:]
    for step in STEPS:
        if names and step.__name__ not in names:
            continue
        step(out)
        print(f"{step.__name__}: ok", flush=True)


if __name__ == "__main__":
    main()
