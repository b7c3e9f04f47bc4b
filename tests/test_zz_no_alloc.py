"""noor_megakernel_frame_noalloc (scratch in a fixed device array, no device
allocation) against noor_megakernel_batch (scratch from cudaMalloc) on the
same frames, two calls in a row, through the C-ABI.  The module creates its
own render context, so it passes alone in a fresh process and after the
other GPU tests."""
import ctypes as C

import numpy as np
import pytest
import torch

from noor_b200 import _capi, scenes

pytestmark = pytest.mark.gpu

MAX_PIXELS = (32 << 20) // 16


def _film(w, h):
    return torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")


def _compare(a, b):
    # the tolerance the wavefront/megakernel comparisons use
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-2)
    assert np.median(rel) < 1e-5, float(np.median(rel))
    assert (rel > 1e-3).mean() < 0.05, float((rel > 1e-3).mean())


@pytest.fixture(scope="module")
def sky():
    g, (c, rad) = scenes.sphere_field(2, 32, 3)
    cam = dict(scenes.frame_spheres(c, rad, 2), w=96, h=64)
    s = scenes.SceneData(**g, skydome_type=_capi.NOOR_SKY_PHYSICAL, camera=cam,
                         render=dict(spp=8, bounces=6, rr=1, mis=1),
                         hosek=dict(turbidity=3.0, albedo=0.3, sun_lat=float(np.radians(60.0)),
                                    sun_lon=float(np.pi / 4), solar_scale=250.0, solar_radius_scale=2.0))
    r = scenes.Renderer(s)
    yield s, r
    r.close()


def test_noalloc_frames_match_batch_megakernel(sky):
    s, r = sky
    cam = s.camera
    frames = [(cam, 8, 1, 6), (dict(cam, w=160, h=90), 5, 3, 4)]   # two calls in a row, different sizes
    for c_, spp, first, bounces in frames:
        a, b = _film(c_["w"], c_["h"]), _film(c_["w"], c_["h"])
        fa = scenes.wf_frame(0, c_, spp, bounces, first_frame=first, d_film=a.data_ptr())
        fb = scenes.wf_frame(0, c_, spp, bounces, first_frame=first, d_film=b.data_ptr())
        torch.cuda.synchronize()
        _capi.call("noor_megakernel_frame_noalloc", C.byref(fa))
        ms = C.c_float()
        arr = (_capi.WfFrame * 1)(fb)
        _capi.call("noor_megakernel_batch", arr, 1, C.byref(ms))
        torch.cuda.synchronize()
        A, B = a.cpu().numpy()[..., :3], b.cpu().numpy()[..., :3]
        assert A.mean() > 0.01
        _compare(A, B)


def test_noalloc_single_chunk_1080p_allocates_nothing(sky):
    """a 1920 x 1080 frame (2,073,600 of the array's 2,097,152 pixels)
    takes the single-chunk path; two calls in a row match the batch
    megakernel, and the device's free memory is the same before and after
    the second call (the first one may still size the kernel's local memory)"""
    s, r = sky
    c_ = dict(s.camera, w=1920, h=1080)
    a = _film(1920, 1080)
    b = _film(1920, 1080)
    for first in (1, 7):
        fa = scenes.wf_frame(0, c_, 2, 4, first_frame=first, d_film=a.data_ptr())
        fb = scenes.wf_frame(0, c_, 2, 4, first_frame=first, d_film=b.data_ptr())
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        _capi.call("noor_megakernel_frame_noalloc", C.byref(fa))
        torch.cuda.synchronize()
        if first == 7:
            assert torch.cuda.mem_get_info()[0] == free_before
        arr = (_capi.WfFrame * 1)(fb)
        ms = C.c_float()
        _capi.call("noor_megakernel_batch", arr, 1, C.byref(ms))
        torch.cuda.synchronize()
        A, B = a.cpu().numpy()[..., :3], b.cpu().numpy()[..., :3]
        assert A.mean() > 0.01
        _compare(A, B)


def test_noalloc_rejects_frames_beyond_the_scratch_array(sky):
    s, r = sky
    w = 4096
    h = MAX_PIXELS // w + 1
    dummy = _film(1, 1)
    f = scenes.wf_frame(0, dict(s.camera, w=w, h=h), 1, 1, d_film=dummy.data_ptr())
    with pytest.raises(_capi.NoorError, match="exceed the scratch array"):
        _capi.call("noor_megakernel_frame_noalloc", C.byref(f))
