"""Plain megakernel images against the oracle: the FP32 transcription on the
same seeds (per-pixel agreement where the paths coincide), and RMSE against
an FP64 high-spp render."""
import ctypes

import numpy as np
import pytest
import torch

from noor_b200 import _capi, scenes
from oracle.oracle import Oracle

from gpu_util import THREADS

pytestmark = pytest.mark.gpu


def rmse(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)))


@pytest.fixture(scope="module")
def room_ref():
    s = scenes.room_scene(width=96, height=96, spp=16)
    r = scenes.Renderer(s)
    orc = Oracle(r.built.payload, r.spec, r.hosek)
    ref64 = orc.render(r.camera, 1, 256, fp64=True, threads=THREADS).reshape(96, 96, 3)
    yield s, r, orc, ref64
    orc.close()
    r.close()


@pytest.mark.parametrize("mis", [0, 1])
@pytest.mark.parametrize("isect,film", [(_capi.NOOR_ISECT_WATERTIGHT, _capi.NOOR_FILM_KAHAN),
                                        (_capi.NOOR_ISECT_REF_WALD, _capi.NOOR_FILM_REF_LERP)])
def test_room_matches_oracle(room_ref, mis, isect, film):
    s, r, orc, ref64 = room_ref
    r.update_spec(mis=mis, intersector=isect, film_mode=film)
    orc_spec = r.spec  # the oracle reads the same struct
    r.render(16)
    img = r.framebuffer()[..., :3]
    o32 = orc.render(r.camera, 1, 16, fp64=False, isect=isect, threads=THREADS).reshape(96, 96, 3)
    diff = np.abs(img - o32)
    rel = diff / np.maximum(np.abs(o32), 1e-2)
    # identical random streams: most pixels agree to float noise
    assert np.median(rel) < 1e-5
    assert (rel > 1e-3).mean() < 0.05
    # equal error against the FP64 oracle
    e_gpu, e_orc = rmse(img, ref64), rmse(o32, ref64)
    assert abs(e_gpu - e_orc) <= 0.05 * e_orc + 1e-4
    assert np.isfinite(img).all() and img.max() > 0.05
    assert r.status(reset=True) == 0


def test_cuda_path_tracer_frame_by_frame_equals_batched(room_ref):
    """cuda_path_tracer (1 spp per call, frame number advanced) folds the same
    samples as one batched launch"""
    s, r, orc, _ = room_ref
    r.update_spec(mis=0, intersector=_capi.NOOR_ISECT_WATERTIGHT, film_mode=_capi.NOOR_FILM_KAHAN)
    for _ in range(4):
        r.path_tracer()
    a = r.framebuffer()
    assert r.frame.value == 5
    r.frame.value = 1
    r.render(4)
    b = r.framebuffer()
    assert np.abs(a - b).max() < 1e-5


def test_lookat_and_counters(room_ref):
    import ctypes as C
    s, r, orc, _ = room_ref
    r.counters(reset=True)
    r.frame.value = 1
    r.render(2)
    ext, shadow, paths = r.counters()
    assert paths == 2 * 96 * 96
    assert ext >= paths and shadow > 0
    la = (C.c_float * 4)()
    _capi.call("get_lookAt", la)
    assert la[3] == 1.0 and 0.0 <= la[1] <= 2.0


def _small_sphere_scene(kind: str):
    g, (c, rad) = scenes.sphere_field(2, 32, 3)
    cam = dict(scenes.frame_spheres(c, rad, 2), w=128, h=72)
    if kind == "sky":
        return scenes.SceneData(**g, skydome_type=_capi.NOOR_SKY_PHYSICAL, camera=cam,
                                render=dict(spp=8, bounces=8, rr=1, mis=0),
                                hosek=dict(turbidity=3.0, albedo=0.3, sun_lat=float(np.radians(60.0)),
                                           sun_lon=float(np.pi / 4), solar_scale=250.0, solar_radius_scale=2.0),
                                name="sky-small")
    return scenes.SceneData(**g, skydome_type=_capi.NOOR_SKY_HDR, env=scenes.env_map(3, 512, 256), camera=cam,
                            render=dict(spp=8, bounces=8, rr=1, mis=1), name="env-small")


@pytest.mark.parametrize("kind", ["sky", "env"])
def test_sphere_field_matches_oracle(kind):
    """Lambert, GGX gold and glass under the Hosek sky (NEE) and under an
    importance-sampled environment map with MIS"""
    s = _small_sphere_scene(kind)
    r = scenes.Renderer(s)
    orc = Oracle(r.built.payload, r.spec, r.hosek)
    try:
        r.render(8)
        img = r.framebuffer()[..., :3].reshape(-1, 3)
        o32 = orc.render(r.camera, 1, 8, threads=THREADS)
        ref64 = orc.render(r.camera, 1, 128, fp64=True, threads=THREADS)
        rel = np.abs(img - o32) / np.maximum(np.abs(o32), 1e-2)
        e_gpu, e_orc = rmse(img, ref64), rmse(o32, ref64)
        diag = dict(median_rel=float(np.median(rel)), frac_off=float((rel > 1e-3).mean()), rmse_gpu=e_gpu,
                    rmse_oracle=e_orc, mean_gpu=img.mean(0).tolist(), mean_oracle=o32.mean(0).tolist())
        # paths start identical; rounding differences (FMA, rsqrt, libm)
        # make a fraction of glass/metal paths take another branch, so the
        # criterion is equal error against the FP64 render
        assert np.median(rel) < 1e-5, diag
        assert (rel > 1e-3).mean() < 0.3, diag
        assert abs(e_gpu - e_orc) <= 0.1 * e_orc + 1e-4, diag
        assert np.isfinite(img).all() and img.mean() > 0.01
        assert r.status() == 0
    finally:
        orc.close()
        r.close()


@pytest.mark.parametrize("pair", [("glossy", "roughglass"), ("substrate", "mirror"), ("translucent", "glossy"),
                                  ("clearcoat", "shadowcatcher")])
def test_room_with_other_materials_matches_oracle(pair):
    """the lobes no configuration uses, on the two boxes: GPU megakernel and
    wavefront against the oracle on the same seeds"""
    kw = {"glossy": dict(albedo=(0.6, 0.4, 0.3), roughness=0.25, ior=1.5),
          "roughglass": dict(roughness=0.3, ior=1.5),
          "substrate": dict(albedo=(0.3, 0.5, 0.7), specular=(0.05, 0.05, 0.05), roughness=0.3),
          "mirror": dict(albedo=(0.9, 0.9, 0.9)),
          "translucent": dict(albedo=(0.6, 0.6, 0.5)),
          "clearcoat": dict(albedo=(0.9, 0.9, 0.9), specular=(0.8, 0.6, 0.5), roughness=0.3, coat_weight=0.5,
                            coat_sigma=0.4, coat_thickness=0.5),
          "shadowcatcher": dict()}
    boxes = [scenes.material(k, **kw[k]) for k in pair]
    s = scenes.room_scene(width=64, height=64, spp=16, box_materials=boxes)
    r = scenes.Renderer(s)
    try:
        for mis in (0, 1):
            r.update_spec(mis=mis)
            r.render(16)
            img = r.framebuffer()[..., :3]
            # the wavefront on the same samples
            film = torch.zeros((64, 64, 4), dtype=torch.float32, device="cuda")
            fr = (_capi.WfFrame * 1)(scenes.wf_frame(0, s.camera, 16, 5, d_film=film.data_ptr()))
            _capi.call("noor_wavefront_render", fr, 1, ctypes.byref(scenes.wf_params(64, 1 << 16, 1, 1)))
            wf = film.cpu().numpy()[..., :3]
            relw = np.abs(wf - img) / np.maximum(np.abs(img), 1e-2)
            assert np.median(relw) < 1e-5 and (relw > 1e-3).mean() < 0.05, (pair, mis)
            orc = Oracle(r.built.payload, r.spec, r.hosek)
            o32 = orc.render(r.camera, 1, 16, fp64=False, threads=THREADS).reshape(64, 64, 3)
            o64 = orc.render(r.camera, 1, 256, fp64=True, threads=THREADS).reshape(64, 64, 3)
            orc.close()
            rel = np.abs(img - o32) / np.maximum(np.abs(o32), 1e-2)
            assert np.isfinite(img).all() and img.mean() > 0.01
            assert np.median(rel) < 1e-5, (pair, mis, float(np.median(rel)))
            # paths that enter a translucent box bounce between its inner
            # faces, where the last bit of a float (the GPU fuses multiply-
            # adds, the oracle does not) can send a path elsewhere: ~6 % of
            # pixels then differ by more than 1e-3, with the same error
            # against the FP64 oracle
            frac = 0.10 if "translucent" in pair else 0.05
            assert (rel > 1e-3).mean() < frac, (pair, mis, float((rel > 1e-3).mean()))
            e_gpu, e_orc = rmse(img, o64), rmse(o32, o64)
            assert abs(e_gpu - e_orc) <= 0.01 * e_orc, (pair, mis, e_gpu, e_orc)
        assert r.status(reset=True) == 0
    finally:
        r.close()


@pytest.mark.parametrize("light", ["sphere", "disk", "point", "spot", "distant"])
def test_room_lit_by_each_light_type_matches_oracle(light):
    """sphere and disk area lights (light nodes in the BVH), point, spot and
    distant lights: GPU megakernel and wavefront against the oracle on the
    same seeds, with and without MIS"""
    s = scenes.room_scene(width=64, height=64, spp=16, light=light)
    r = scenes.Renderer(s)
    try:
        for mis in (0, 1):
            r.update_spec(mis=mis)
            r.render(16)
            img = r.framebuffer()[..., :3]
            film = torch.zeros((64, 64, 4), dtype=torch.float32, device="cuda")
            fr = (_capi.WfFrame * 1)(scenes.wf_frame(0, s.camera, 16, 5, d_film=film.data_ptr()))
            _capi.call("noor_wavefront_render", fr, 1, ctypes.byref(scenes.wf_params(64, 1 << 16, 1, 1)))
            wf = film.cpu().numpy()[..., :3]
            relw = np.abs(wf - img) / np.maximum(np.abs(img), 1e-2)
            assert np.median(relw) < 1e-5 and (relw > 1e-3).mean() < 0.05, (light, mis)
            orc = Oracle(r.built.payload, r.spec, r.hosek)
            o32 = orc.render(r.camera, 1, 16, fp64=False, threads=THREADS).reshape(64, 64, 3)
            o64 = orc.render(r.camera, 1, 256, fp64=True, threads=THREADS).reshape(64, 64, 3)
            orc.close()
            rel = np.abs(img - o32) / np.maximum(np.abs(o32), 1e-2)
            assert np.isfinite(img).all() and img.mean() > 0.005, (light, mis, float(img.mean()))
            assert np.median(rel) < 1e-5, (light, mis, float(np.median(rel)))
            assert (rel > 1e-3).mean() < 0.05, (light, mis, float((rel > 1e-3).mean()))
            e_gpu, e_orc = rmse(img, o64), rmse(o32, o64)
            assert abs(e_gpu - e_orc) <= 0.02 * e_orc + 1e-5, (light, mis, e_gpu, e_orc)
        assert r.status(reset=True) == 0
    finally:
        r.close()


@pytest.mark.parametrize("camera", [dict(type="ortho", ortho_scale=2.2), dict(type="env"),
                                    dict(lens_radius=0.08, focal_length=3.0)])
def test_other_cameras_match_oracle(camera):
    """orthographic, environment and thin-lens cameras: the megakernel
    (its camera build), the wavefront and the oracle on the same seeds"""
    s = scenes.room_scene(width=64, height=48, spp=8)
    # a view slightly off the axes: the reference's ray setup counts a zero
    # direction component as negative with an infinite inverse
    # (ray.cuh:200-206), so an exactly axis-aligned orthographic ray misses
    # every box, here as there
    s.camera = dict(s.camera, eye=(0.07, 1.05, 3.75), **camera)
    if camera.get("type") == "env":
        s.camera = dict(s.camera, eye=(0.0, 1.0, 0.2))      # inside the room
    r = scenes.Renderer(s)
    try:
        r.render(8)
        img = r.framebuffer()[..., :3]
        film = torch.zeros((48, 64, 4), dtype=torch.float32, device="cuda")
        fr = (_capi.WfFrame * 1)(scenes.wf_frame(0, s.camera, 8, 5, d_film=film.data_ptr()))
        _capi.call("noor_wavefront_render", fr, 1, ctypes.byref(scenes.wf_params(64, 1 << 16, 1, 1)))
        wf = film.cpu().numpy()[..., :3]
        relw = np.abs(wf - img) / np.maximum(np.abs(img), 1e-2)
        assert np.median(relw) < 1e-5 and (relw > 1e-3).mean() < 0.05, camera
        orc = Oracle(r.built.payload, r.spec, r.hosek)
        o32 = orc.render(r.camera, 1, 8, fp64=False, threads=THREADS).reshape(48, 64, 3)
        orc.close()
        rel = np.abs(img - o32) / np.maximum(np.abs(o32), 1e-2)
        assert np.isfinite(img).all() and img.mean() > 0.01, camera
        assert np.median(rel) < 1e-5 and (rel > 1e-3).mean() < 0.05, (camera, float((rel > 1e-3).mean()))
        assert r.status(reset=True) == 0
    finally:
        r.close()
