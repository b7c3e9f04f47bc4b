"""Persistent wavefront integrator against the plain megakernel on the same
samples (identical random streams), single frames and uneven batches, in the
CUDA-graph (device while loop) and host-loop forms."""
import ctypes as C

import numpy as np
import pytest
import torch

from noor_b200 import _capi, scenes
from oracle.oracle import Oracle

from gpu_util import THREADS

pytestmark = pytest.mark.gpu


def film(w, h):
    return torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")


def run_wf(frames, params):
    arr = (_capi.WfFrame * len(frames))(*frames)
    ms = C.c_float()
    _capi.call("noor_wavefront_render_timed", arr, len(frames), C.byref(params), C.byref(ms))
    return ms.value


def run_mk(frames):
    arr = (_capi.WfFrame * len(frames))(*frames)
    ms = C.c_float()
    _capi.call("noor_megakernel_batch", arr, len(frames), C.byref(ms))
    return ms.value


def compare(a, b, frac=0.05):
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-2)
    assert np.median(rel) < 1e-5, float(np.median(rel))
    assert (rel > 1e-3).mean() < frac, float((rel > 1e-3).mean())


@pytest.fixture
def room():
    s = scenes.room_scene(width=96, height=96, spp=16)
    r = scenes.Renderer(s)
    yield s, r
    r.close()


@pytest.mark.parametrize("graph", [1, 0])
@pytest.mark.parametrize("sort", [3, 2, 1, 0])
def test_room_wavefront_equals_megakernel(room, graph, sort):
    s, r = room
    a, b = film(96, 96), film(96, 96)
    fw = scenes.wf_frame(0, s.camera, 16, bounces=5, d_film=a.data_ptr())
    fm = scenes.wf_frame(0, s.camera, 16, bounces=5, d_film=b.data_ptr())
    run_wf([fw], scenes.wf_params(128, 1 << 14, sort, graph))
    run_mk([fm])
    torch.cuda.synchronize()
    compare(a.cpu().numpy()[..., :3], b.cpu().numpy()[..., :3])
    ctr = (C.c_uint64 * 3)()
    _capi.call("noor_wavefront_counters", ctr, 1)
    assert ctr[2] == 96 * 96 * 16
    assert r.status(reset=True) == 0


def test_room_wavefront_matches_fp64_oracle(room):
    s, r = room
    a = film(96, 96)
    run_wf([scenes.wf_frame(0, s.camera, 16, bounces=5, d_film=a.data_ptr())], scenes.wf_params())
    orc = Oracle(r.built.payload, r.spec, r.hosek)
    ref = orc.render(r.camera, 1, 256, fp64=True, threads=THREADS).reshape(96, 96, 3)
    o32 = orc.render(r.camera, 1, 16, threads=THREADS).reshape(96, 96, 3)
    orc.close()
    img = a.cpu().numpy()[..., :3]
    e_wf = float(np.sqrt(np.mean((img - ref) ** 2)))
    e_o = float(np.sqrt(np.mean((o32 - ref) ** 2)))
    assert abs(e_wf - e_o) <= 0.05 * e_o + 1e-4


def test_uneven_batch_across_scenes(room):
    """frames of different scenes, resolutions, spp and depths in one launch"""
    s, r = room
    g, (c, rad) = scenes.sphere_field(2, 32, 3)
    sky = scenes.SceneData(**g, skydome_type=_capi.NOOR_SKY_PHYSICAL, render=dict(spp=4, bounces=6, rr=1, mis=0),
                           hosek=dict(turbidity=3.0, albedo=0.3, sun_lat=float(np.radians(60.0)),
                                      sun_lon=float(np.pi / 4), solar_scale=250.0, solar_radius_scale=2.0))
    env = scenes.SceneData(**g, skydome_type=_capi.NOOR_SKY_HDR, env=scenes.env_map(5, 256, 128),
                           render=dict(spp=4, bounces=6, rr=1, mis=1))
    sid1, keep1 = scenes.upload_scene(sky)
    sid2, keep2 = scenes.upload_scene(env)
    cam = scenes.frame_spheres(c, rad, 2)
    specs = [(0, dict(s.camera, w=64, h=48), 8, 5), (sid1, dict(cam, w=80, h=45), 4, 6),
             (sid2, dict(cam, w=40, h=40), 12, 6), (sid1, dict(cam, w=128, h=72), 5, 6)]
    fa = [film(c_["w"], c_["h"]) for _, c_, _, _ in specs]
    fb = [film(c_["w"], c_["h"]) for _, c_, _, _ in specs]
    frw = [scenes.wf_frame(i, c_, spp, b, d_film=t.data_ptr()) for (i, c_, spp, b), t in zip(specs, fa)]
    frm = [scenes.wf_frame(i, c_, spp, b, d_film=t.data_ptr()) for (i, c_, spp, b), t in zip(specs, fb)]
    run_wf(frw, scenes.wf_params(128, 1 << 15, 1, 1))
    run_mk(frm)
    torch.cuda.synchronize()
    for x, y in zip(fa, fb):
        compare(x.cpu().numpy()[..., :3], y.cpu().numpy()[..., :3], frac=0.3)
    assert r.status(reset=True) == 0


def test_autotune_picks_a_candidate(room):
    s, r = room
    a = film(96, 96)
    best = scenes.wf_params(graph=1)
    ms = C.c_float()
    fr = (_capi.WfFrame * 1)(scenes.wf_frame(0, s.camera, 4, bounces=5, d_film=a.data_ptr()))
    _capi.call("noor_wavefront_autotune", fr, 1, C.byref(best), C.byref(ms))
    assert best.block_size in (64, 128) and best.queue_capacity >= 1 << 18 and ms.value > 0


@pytest.mark.parametrize("which", ["room", "sky"])
def test_wavefront_trees_trace_the_same_paths(which):
    """the extension and shadow stages on the binary tree and on the
    four-wide tree: the same hits, so the same rays traced (counted) and the
    same image up to the film's atomic summation order"""
    if which == "room":
        s = scenes.room_scene(width=96, height=96, spp=16)
    else:
        s = scenes.sky_scene(width=96, height=64, count=8, level=4)
    r = scenes.Renderer(s)
    try:
        w, h = s.camera["w"], s.camera["h"]
        out, rays = [], []
        for tree in (_capi.NOOR_TRAVERSAL_BINARY, _capi.NOOR_TRAVERSAL_WIDE, _capi.NOOR_TRAVERSAL_WIDE_SHADOW):
            f = film(w, h)
            fr = scenes.wf_frame(0, s.camera, 16, bounces=5, d_film=f.data_ptr())
            c = (C.c_uint64 * 3)()
            _capi.call("noor_wavefront_counters", c, 1)
            run_wf([fr], scenes.wf_params(128, 1 << 16, 1, 1, traversal=tree))
            _capi.call("noor_wavefront_counters", c, 1)
            torch.cuda.synchronize()
            out.append(f.cpu().numpy()[..., :3])
            rays.append(tuple(int(x) for x in c))
        assert rays[0] == rays[1] == rays[2] and rays[0][0] > 0, rays
        for k in (1, 2):
            rel = np.abs(out[0] - out[k]) / np.maximum(np.abs(out[k]), 1e-2)
            assert rel.max() < 1e-5, (k, float(rel.max()))
        assert r.status(reset=True) == 0
    finally:
        r.close()


def test_shade_register_budgets_give_the_same_image(room):
    """the single-scene shading stage built for 80 and for 128 registers:
    the same code, so the same rays and the same image (up to the film's
    atomic summation order); a budget it is not built for is refused"""
    s, r = room
    out, rays = [], []
    for regs in (80, 128):
        f = film(96, 96)
        fr = scenes.wf_frame(0, s.camera, 16, bounces=5, d_film=f.data_ptr())
        c = (C.c_uint64 * 3)()
        _capi.call("noor_wavefront_counters", c, 1)
        run_wf([fr], scenes.wf_params(128, 1 << 14, 1, 1, shade_regs=regs))
        _capi.call("noor_wavefront_counters", c, 1)
        torch.cuda.synchronize()
        out.append(f.cpu().numpy()[..., :3])
        rays.append(tuple(int(x) for x in c))
    assert rays[0] == rays[1] and rays[0][0] > 0
    rel = np.abs(out[0] - out[1]) / np.maximum(np.abs(out[1]), 1e-2)
    assert rel.max() < 1e-5, float(rel.max())
    fr = scenes.wf_frame(0, s.camera, 16, bounces=5, d_film=film(96, 96).data_ptr())
    with pytest.raises(_capi.NoorError):
        run_wf([fr], scenes.wf_params(128, 1 << 14, 1, 1, shade_regs=64))
