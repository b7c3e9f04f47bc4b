"""Headless display path: the display shader's transforms (oracle) on known
values, and the library's tonemap kernel and image files against them on the
GPU."""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from noor_b200 import _capi, scenes
from oracle.oracle import tonemap


def test_oracle_tonemap_known_values():
    film = np.array([[0.0, 1.0, 4.0, 1.0], [0.25, 100.0, -1.0, 1.0]], np.float32)
    g = tonemap(film, 0)
    assert list(g[0, :3]) == [0, 255, 255] and list(g[1, 1:3]) == [255, 0]
    assert g[1, 0] == round(255 * 0.25 ** (1 / 2.2))
    r = tonemap(film, 1)
    assert r[0, 1] == round(255 * 0.5 ** (1 / 2.2))            # 1 / (1 + 1)
    assert r[1, 1] == round(255 * (100 / 101) ** (1 / 2.2))
    f = tonemap(film, 2)
    assert f[0, 0] == 0 and f[1, 1] == 255                       # the curve tends to 1
    u = tonemap(np.array([[11.2 / 4, 0.0, 1.0, 1.0]], np.float32), 3)
    assert u[0, 0] == 255 and u[0, 1] == 0                       # white point maps to 1
    assert (tonemap(film, 0, exposure=0.0)[..., :3] == 0).all()
    assert (g[..., 3] == 255).all()
    # every operator is monotone in the input
    ramp = np.zeros((256, 4), np.float32)
    ramp[:, :3] = np.linspace(0, 20, 256)[:, None]
    for op in range(4):
        v = tonemap(ramp, op)[:, 0].astype(int)
        assert (np.diff(v) >= 0).all(), op


@pytest.mark.gpu
def test_tonemap_kernel_and_image_files_match_oracle():
    import torch
    rng = np.random.default_rng(5)
    film = np.zeros((64, 48, 4), np.float32)
    film[..., :3] = rng.lognormal(-1.0, 1.5, (64, 48, 3)).astype(np.float32)
    film[..., 3] = 1
    s = scenes.room_scene(width=24, height=16, spp=4)
    r = scenes.Renderer(s)
    try:
        d_film = torch.from_numpy(film).cuda()
        d_out = torch.zeros((64, 48, 4), dtype=torch.uint8, device="cuda")
        for op in range(4):
            for exposure in (1.0, 0.5):
                _capi.call("noor_tonemap_device", d_film.data_ptr(), 64 * 48, op, exposure, d_out.data_ptr())
                got = d_out.cpu().numpy().astype(int)
                want = tonemap(film, op, exposure).astype(int)
                d = np.abs(got - want)
                # powf and numpy's pow may round a value across a .5 step
                assert d.max() <= 1 and (d == 0).mean() > 0.999, (op, exposure, d.max(), (d == 0).mean())
        with pytest.raises(_capi.NoorError):
            _capi.call("noor_tonemap_device", d_film.data_ptr(), 64 * 48, 7, 1.0, d_out.data_ptr())
        # image files of the context's film
        r.render(4)
        fb = r.framebuffer()
        with tempfile.TemporaryDirectory() as d:
            pfm, ppm = os.path.join(d, "a.pfm"), os.path.join(d, "a.ppm")
            _capi.call("noor_save_image", pfm.encode(), _capi.NOOR_TONEMAP_NONE, 1.0)
            _capi.call("noor_save_image", ppm.encode(), _capi.NOOR_TONEMAP_REINHARD, 1.5)
            raw = open(pfm, "rb").read()
            head = b"PF\n24 16\n-1.0\n"
            assert raw.startswith(head)
            lin = np.frombuffer(raw[len(head):], np.float32).reshape(16, 24, 3)
            assert np.array_equal(lin, fb[..., :3])               # bottom row first = film row 0
            raw = open(ppm, "rb").read()
            head = b"P6\n24 16\n255\n"
            assert raw.startswith(head)
            img = np.frombuffer(raw[len(head):], np.uint8).reshape(16, 24, 3)[::-1].astype(int)
            want = tonemap(fb, 1, 1.5)[..., :3].astype(int)
            assert np.abs(img - want).max() <= 1
    finally:
        r.close()
