"""The CPU restatement (oracle/noor_oracle.cpp, FP32) against the
reference's own device routines.

The fixtures tests/golden/refdev_*.npz were frozen on a B200 by
tests/golden/make_refdev_golden.py from noor/cuda/*.cuh compiled unmodified
by nvcc (oracle/refdev/, no FMA contraction): CudaRNG, the microfacet
distributions, Fresnel, the sampling warps, querySkyModel, the CudaBSDF on a
probe scene, the BVH traversal with the Wald test, generateRay and
path_tracer_kernel's bounce loop.  This pins the restatement to the
reference's code rather than to a reading of it.
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from noor_b200 import _capi, scenes
from oracle import oracle as O
from oracle.oracle import Oracle

import refdev_probe as probe

GOLD = Path(__file__).resolve().parent / "golden"


def load(name):
    return np.load(GOLD / f"refdev_{name}.npz")


def test_rng_bit_exact():
    z = load("rng")
    seed, draws = O.rng(z["seeds"], z["draws"].shape[1])
    assert np.array_equal(seed, z["seed"])
    assert np.array_equal(draws, z["draws"])


@pytest.mark.parametrize("kind,key", [(0, "ggx"), (1, "beckmann")])
def test_microfacet(kind, key):
    z = load("micro")
    # the Trowbridge-Reitz D, G and Pdf are the same operations in the same
    # order: bit-identical; Beckmann's D goes through expf (libm vs CUDA)
    probe.check_microfacet(z[key], O.routines(kind, z["rec"]), exact=(kind == 0))


def test_fresnel_bit_exact():
    z = load("fresnel")
    assert np.array_equal(O.routines(2, z["rec"]), z["out"])


def test_warps():
    z = load("warps")
    probe.check_warps(z["out"], O.routines(3, z["rec"]))


@pytest.fixture(scope="module")
def probe_oracle():
    s = probe.probe_scene()
    b = scenes.BuiltPayload(s)
    spec = b.default_spec(2, 1)
    orc = Oracle(b.payload, spec, scenes.make_hosek(None))
    yield orc
    orc.close()
    b.free()


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_bsdf(probe_oracle, kind):
    z = load("bsdf")
    rec, ref = z[f"rec{kind}"], z[f"out{kind}"]
    got = probe_oracle.eval_bsdf(kind, probe.product_records(rec, ref if kind == 2 else None))
    probe.check_bsdf(kind, rec, ref, got)


def test_sky():
    z = load("sky")
    hosek = _capi.HosekSky.from_buffer_copy(z["hosek"].tobytes())
    s = probe.trace_scenes()["field16"]
    b = scenes.BuiltPayload(s)
    orc = Oracle(b.payload, b.default_spec(2, 1), hosek)
    got = orc.eval_sky(z["dirs"])
    orc.close()
    e = probe.rel_err(got, z["rgb"]).max(1)
    assert e.max() < 1e-5, e.max()


@pytest.mark.parametrize("name", ["room", "field16"])
def test_closest_and_any_hit(name):
    z = load("trace")
    s = probe.trace_scenes()[name]
    b = scenes.BuiltPayload(s)
    spec = b.default_spec(5, 1)
    spec.intersector = _capi.NOOR_ISECT_REF_WALD
    orc = Oracle(b.payload, spec, scenes.make_hosek(None))
    rays = z[f"{name}_rays"]
    probe.check_trace(z[f"{name}_hits"], z[f"{name}_any"], orc.trace_closest(rays, 1), orc.trace_any(rays, 1))
    orc.close()


@pytest.mark.parametrize("name", ["room", "field16"])
def test_camera_rays(name):
    z = load("trace")
    s = probe.trace_scenes()[name]
    cam = scenes.make_camera(s.camera)
    n = cam.w * cam.h
    got = np.zeros((n, 8), np.float32)
    O.lib().oracle_camera_rays(C.addressof(cam), 1, got.ctypes.data_as(C.c_void_p))
    probe.check_camera_rays(z[f"{name}_rays"][:n], got)


def test_room_render():
    """the C1 room with a sphere light node, 8 frames, MIS off: the
    reference's running-mean film against the oracle's mean"""
    z = load("render")
    s = probe.trace_scenes()["room"]
    b = scenes.BuiltPayload(s)
    spec = b.default_spec(5, 1)
    spec.intersector = _capi.NOOR_ISECT_REF_WALD
    orc = Oracle(b.payload, spec, scenes.make_hosek(None))
    cam = scenes.make_camera(s.camera)
    img = orc.render(cam, 1, 8, isect=_capi.NOOR_ISECT_REF_WALD).reshape(cam.h, cam.w, 3)
    orc.close()
    probe.check_film(z["room_film"], img)


def test_reference_distribution_sampling_bit_exact():
    """the restatement of CudaDistribution2D's sampling (its n + 1 searches
    included) on the reference's own tables for a 256 x 128 map"""
    z = load("envdist")
    got = O.ref_dist_sample(z["func"], z["cdf"], int(z["w"]), int(z["h"]), z["u"])
    assert np.array_equal(got, z["samples"])


def test_textured_room_against_the_reference():
    """the oracle on the textured room: camera-ray hits bit for bit (alpha
    cuts included); the film through the oracle's emulation of the texture
    unit (its fetches match the unit's on about 99 %, the rest within
    1/256 of a texel difference), to looser bars than the untextured room"""
    z = load("textures")
    s = scenes.textured_room_scene()
    b = scenes.BuiltPayload(s)
    spec = b.default_spec(s.render["bounces"], s.render.get("rr", 1))
    spec.intersector = _capi.NOOR_ISECT_REF_WALD
    orc = Oracle(b.payload, spec, scenes.make_hosek(None))
    rays = z["rays"]
    probe.check_trace(z["hits"], z["any"], orc.trace_closest(rays, 1), orc.trace_any(rays, 1))
    cam = scenes.make_camera(s.camera)
    img = orc.render(cam, 1, 8, isect=_capi.NOOR_ISECT_REF_WALD).reshape(cam.h, cam.w, 3)
    orc.close()
    probe.check_film(z["film"], img, q99=1e-3, q999=3e-2)
