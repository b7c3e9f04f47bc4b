"""The product's CUDA routines against the reference's own device routines.

Fixture tests hold the library to tests/golden/refdev_*.npz (frozen from
noor/cuda/*.cuh compiled unmodified, oracle/refdev/, by
tests/golden/make_refdev_golden.py); they need no reference tree.  Where the
reference library itself (oracle/_ref/libnoor_refdev.so) is present, the
closest-hit parity is also checked live at the sky-lit configuration's full
size (2,621,440 triangles, 1920x1080 camera rays plus a million secondary
rays), against the reference's traversal and against the CPU oracle.
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from noor_b200 import _capi, scenes
from oracle import reference_device as rd
from oracle.oracle import Oracle

import refdev_probe as probe
from gpu_util import THREADS, camera_rays, dev, dev_empty, host, trace_any, trace_closest

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def load(name):
    return np.load(GOLD / f"refdev_{name}.npz")


def routine(kind, rec):
    no = 12 if kind <= 1 else (4 if kind == 2 else 16)
    d_in = dev(np.ascontiguousarray(rec, np.float32))
    d_out = dev_empty(rec.shape[0] * no * 4)
    _capi.call("noor_eval_routines", kind, C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), rec.shape[0])
    return host(d_out, np.float32, (rec.shape[0], no))


@pytest.mark.parametrize("kind,key", [(0, "ggx"), (1, "beckmann")])
def test_microfacet(kind, key):
    z = load("micro")
    probe.check_microfacet(z[key], routine(kind, z["rec"]), exact=False)


def test_fresnel():
    z = load("fresnel")
    probe.check_fresnel(z["out"], routine(2, z["rec"]))


def test_warps():
    z = load("warps")
    probe.check_warps(z["out"], routine(3, z["rec"]), tol=1e-5)


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_bsdf(kind):
    z = load("bsdf")
    rec, ref = z[f"rec{kind}"], z[f"out{kind}"]
    r = scenes.Renderer(probe.probe_scene())
    try:
        pr = probe.product_records(rec, ref if kind == 2 else None)
        d_in = dev(pr)
        d_out = dev_empty(pr.shape[0] * 32)
        _capi.call("noor_eval_bsdf", kind, C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), pr.shape[0])
        got = host(d_out, np.float32, (pr.shape[0], 8))
    finally:
        r.close()
    probe.check_bsdf(kind, rec, ref, got)


def test_sky():
    """Hosek radiance within 1e-5 relative at the 99.9th percentile, 5e-5 at
    most (sun-disc edge and sRGB knee)"""
    z = load("sky")
    hosek = _capi.HosekSky.from_buffer_copy(z["hosek"].tobytes())
    r = scenes.Renderer(probe.trace_scenes()["field16"], hosek=hosek)
    try:
        d = dev(z["dirs"])
        o = dev_empty(z["dirs"].shape[0] * 12)
        _capi.call("noor_eval_sky", C.c_void_p(d.data_ptr()), C.c_void_p(o.data_ptr()), z["dirs"].shape[0])
        got = host(o, np.float32, (-1, 3))
    finally:
        r.close()
    e = probe.rel_err(got, z["rgb"]).max(1)
    assert np.quantile(e, 0.999) < 1e-5 and e.max() < 5e-5, (np.quantile(e, 0.999), e.max())


@pytest.mark.parametrize("name", ["room", "field16"])
def test_closest_any_hit_and_camera(name):
    z = load("trace")
    r = scenes.Renderer(probe.trace_scenes()[name], intersector=_capi.NOOR_ISECT_REF_WALD)
    try:
        rays = z[f"{name}_rays"]
        probe.check_trace(z[f"{name}_hits"], z[f"{name}_any"], trace_closest(rays), trace_any(rays))
        n = r.w * r.h
        probe.check_camera_rays(rays[:n], camera_rays(r, 1), tol=1e-6)
    finally:
        r.close()


def test_room_render_megakernel_and_wavefront():
    """C1 room with a sphere light node, MIS off, 8 frames: the megakernel
    with the reference's running-mean film, and the wavefront integrator,
    against path_tracer_kernel's film"""
    z = load("render")
    s = probe.trace_scenes()["room"]
    r = scenes.Renderer(s, intersector=_capi.NOOR_ISECT_REF_WALD, film_mode=_capi.NOOR_FILM_REF_LERP)
    try:
        r.render(8)
        probe.check_film(z["room_film"], r.framebuffer())
        import torch
        film = torch.zeros(r.w * r.h * 4, dtype=torch.float32, device="cuda")
        f = scenes.wf_frame(0, s.camera, 8, bounces=s.render["bounces"], first_frame=1, d_film=film.data_ptr())
        _capi.call("noor_wavefront_render", C.byref(f), 1, C.byref(scenes.wf_params(block=128, capacity=1 << 16)))
        torch.cuda.synchronize()
        probe.check_film(z["room_film"], film.cpu().numpy().reshape(r.h, r.w, 4))
    finally:
        r.close()


# ------------------------------------------------ textures, alpha, bump
def test_textured_room_against_the_reference():
    """the textured room (floor checker, roughness map, a bump map read with
    ray differentials, an alpha-cut panel): closest and any hits of the
    camera rays bit for bit (the alpha cuts included), and the 8-frame film
    of the megakernel and of the wavefront against path_tracer_kernel's --
    the texture unit does the same fetches for both.  Per pixel the films
    agree to the untextured bars at the median; in the tails, pixels whose
    paths read the bump map move: its slopes come from ray differentials,
    and a last-bit difference in them (FMA contraction here, none in the
    reference built for the harness) moves the map's 8-bit filter weights,
    hence bars of 1e-3 / 1e-2 at the 99th / 99.9th percentile."""
    z = load("textures")
    s = scenes.textured_room_scene()
    r = scenes.Renderer(s, intersector=_capi.NOOR_ISECT_REF_WALD, film_mode=_capi.NOOR_FILM_REF_LERP)
    try:
        rays = z["rays"]
        hits = trace_closest(rays)
        probe.check_trace(z["hits"], z["any"], hits, trace_any(rays))
        r.render(8)
        img = r.framebuffer()
        # where the error lives: by the material the camera ray of frame 1 hits
        e = probe.rel_err(img[..., :3], z["film"][..., :3], 1e-3).max(-1).ravel()
        n = r.w * r.h
        mats = np.array([r.built.payload.attribute_indices[4 * int(t) + 3] for t in hits[:n, 1]])
        mats[hits[:n, 6] == 0] = -1
        for m in np.unique(mats):
            print("material", int(m), "pixels", int((mats == m).sum()), "q99", float(np.quantile(e[mats == m], 0.99)))
        probe.check_film(z["film"], img, q99=1e-3, q999=1e-2)
        import torch
        film = torch.zeros(r.w * r.h * 4, dtype=torch.float32, device="cuda")
        f = scenes.wf_frame(0, s.camera, 8, bounces=s.render["bounces"], first_frame=1, d_film=film.data_ptr())
        _capi.call("noor_wavefront_render", C.byref(f), 1, C.byref(scenes.wf_params(block=128, capacity=1 << 16)))
        torch.cuda.synchronize()
        probe.check_film(z["film"], film.cpu().numpy().reshape(r.h, r.w, 4), q99=1e-3, q999=1e-2)
        assert r.status(reset=True) == 0
    finally:
        r.close()


# ------------------------------------------------ NOOR_ENV_REFERENCE mode
def _ref_mode(scene, **kw):
    r = scenes.Renderer(scene, **kw)
    r.update_spec(env_sampling=_capi.NOOR_ENV_REFERENCE)
    return r


def _ref_tables():
    w, h = C.c_int(), C.c_int()
    _capi.call("noor_get_reference_distribution", C.byref(w), C.byref(h), None, None)
    n = h.value * (w.value + 2) + 1
    func = np.zeros(n, np.float32)
    cdf = np.zeros(n, np.float32)
    pf = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    _capi.call("noor_get_reference_distribution", None, None, pf(func), pf(cdf))
    return w.value, h.value, func, cdf


def _env_samples(u):
    d_u = dev(np.ascontiguousarray(u, np.float32))
    d_o = dev_empty(u.shape[0] * 16)
    _capi.call("noor_eval_env_sample", C.c_void_p(d_u.data_ptr()), C.c_void_p(d_o.data_ptr()), u.shape[0])
    return host(d_o, np.float32, (u.shape[0], 4))


def test_reference_env_mode_hdr_bit_exact():
    """a 256 x 128 HDR map: the reference's tables (3x3 texture-filtered
    luminance, FP32 Blelloch sums), its samples and its texture-unit lookups,
    all to the bit"""
    z = load("envdist")
    r = _ref_mode(probe.envdist_scene())
    try:
        w, h, func, cdf = _ref_tables()
        assert (w, h) == (int(z["w"]), int(z["h"]))
        assert np.array_equal(func, z["func"]) and np.array_equal(cdf, z["cdf"])
        assert np.array_equal(_env_samples(z["u"]), z["samples"])
        d = dev(z["dirs"])
        o = dev_empty(z["dirs"].shape[0] * 12)
        _capi.call("noor_eval_sky", C.c_void_p(d.data_ptr()), C.c_void_p(o.data_ptr()), z["dirs"].shape[0])
        assert np.array_equal(host(o, np.float32, (-1, 3)), z["radiance"])
    finally:
        r.close()


def test_reference_env_mode_sky():
    """the physical sky baked into 2048 x 2048 and its 1024 x 1024 tables;
    the Hosek radiance itself agrees to ~1e-5, so the tables to 1e-4 and the
    samples to 1e-4 of the unit square"""
    z = load("envdist")
    r = _ref_mode(probe.trace_scenes()["field16"])
    try:
        w, h, func, cdf = _ref_tables()
        assert (w, h) == (int(z["sky_w"]), int(z["sky_h"]))
        rows = np.concatenate([(k * (w + 1) + np.arange(w + 1)) for k in probe.ENV_ROWS] +
                              [h * (w + 1) + np.arange(h + 1)])
        assert probe.rel_err(func[rows], z["sky_func"], 1e-6).max() < 1e-4
        assert np.abs(cdf[rows] - z["sky_cdf"]).max() < 1e-5
        s = _env_samples(z["u"])
        assert np.quantile(np.abs(s[:, :2] - z["sky_samples"][:, :2]).max(1), 0.999) < 1e-4
    finally:
        r.close()


@pytest.mark.parametrize("name", ["field16", "envfield"])
def test_render_reference_env_mode(name):
    """sphere fields lit by the physical sky or an HDR map, MIS off, 8
    frames: with the reference's environment sampling the megakernel draws
    the reference's light samples, and its film follows path_tracer_kernel's"""
    z = load("render")
    s = probe.env_field() if name == "envfield" else probe.trace_scenes()[name]
    r = _ref_mode(s, intersector=_capi.NOOR_ISECT_REF_WALD, film_mode=_capi.NOOR_FILM_REF_LERP)
    try:
        r.render(8)
        img = r.framebuffer()
    finally:
        r.close()
    # a few paths in a thousand part ways on rounding (the product's BSDF
    # sampling contracts multiply-adds, the reference's build does not) and
    # take another branch at a glass or a lobe of the map
    probe.check_film(z[f"{name}_film"], img, q999=1e-3)


# ------------------------------------------------------------ live, C2 size
live = pytest.mark.skipif(not rd.available(), reason="reference device library not built here")


@pytest.fixture(scope="module")
def c2():
    s = scenes.sky_scene()
    built = scenes.BuiltPayload(s, gpu=True)
    yield s, built
    built.free()


def _secondary_rays(prim: np.ndarray, hits: np.ndarray, n: int, seed: int) -> np.ndarray:
    """rays from the surface points the camera rays hit (nudged back along
    the camera ray) in uniformly random directions, half of them bounded"""
    rng = np.random.default_rng(seed)
    h = np.where(hits[:, 6] == 1)[0]
    pick = rng.choice(h, n)
    t = hits[pick, 0].view(np.float32)
    o = prim[pick, 0:3] + prim[pick, 4:7] * (t * np.float32(0.999))[:, None]
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    out = np.zeros((n, 8), np.float32)
    out[:, 0:3], out[:, 3], out[:, 4:7] = o, np.inf, d
    out[n // 2:, 3] = rng.uniform(0.5, 20.0, n - n // 2)
    return out


@live
def test_c2_closest_hit_bit_exact_against_the_reference(c2):
    """the sky-lit configuration's 2,621,440-triangle two-level BVH: every
    camera ray of a 1920x1080 frame plus 1M secondary rays; Wald mode gives
    the reference's triangle, instance, t and barycentric bits for every ray
    and its any-hit answers; the watertight test names the same triangle for
    at least 99.9 % of the hits"""
    s, built = c2
    spec = built.default_spec(8, 1)
    spec.intersector = _capi.NOOR_ISECT_REF_WALD
    cam = scenes.make_camera(s.camera)
    hosek = scenes.make_hosek(s.hosek)
    ref = rd.RefDevice(built.payload, hosek, cam, spec)
    try:
        prim = ref.camera_rays(1)
        ph = ref.trace_closest(prim)
        rays = np.concatenate([prim, _secondary_rays(prim, ph, 1_000_000, 3)])
        ref_hits, ref_any = ref.trace_closest(rays), ref.trace_any(rays)
    finally:
        ref.close()
    r = scenes.Renderer(s, built=built, intersector=_capi.NOOR_ISECT_REF_WALD)
    try:
        probe.check_trace(ref_hits, ref_any, trace_closest(rays), trace_any(rays))
        probe.check_camera_rays(prim, camera_rays(r, 1), tol=1e-6)
        r.update_spec(intersector=_capi.NOOR_ISECT_WATERTIGHT)
        wt = trace_closest(rays)
        hit = ref_hits[:, 6] == 1
        same = (wt[:, 6] == ref_hits[:, 6]) & (~hit | ((wt[:, 1] == ref_hits[:, 1]) & (wt[:, 2] == ref_hits[:, 2])))
        assert same.mean() >= 0.999, same.mean()
    finally:
        r.close()
    # the CPU oracle on a 200k subset of the same rays
    orc = Oracle(built.payload, spec, hosek)
    sub = np.random.default_rng(4).choice(rays.shape[0], 200_000, replace=False)
    probe.check_trace(ref_hits[sub], ref_any[sub], orc.trace_closest(rays[sub], 1, THREADS),
                      orc.trace_any(rays[sub], 1))
    orc.close()
