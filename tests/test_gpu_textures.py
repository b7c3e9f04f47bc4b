"""Image textures, alpha cuts and bump maps through the library's own modes
(watertight test, compensated film) against the oracle on the same samples:
the textured room, with and without a textured ceiling light (an emitter's
map is read at the hit's barycentrics), by the megakernel and the wavefront.
The texture unit's 8-bit filter weights are emulated by the oracle (its
fetches match about 99 %), so the bars are those of the untextured scenes
except in the tails."""
import numpy as np
import pytest
import torch

from noor_b200 import _capi, scenes
from oracle.oracle import Oracle

from gpu_util import THREADS
from test_gpu_wavefront import film, run_mk, run_wf

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("textured_light", [False, True])
def test_textured_room_matches_the_oracle(textured_light):
    s = scenes.textured_room_scene(textured_light=textured_light)
    r = scenes.Renderer(s)
    try:
        w, h, spp = s.camera["w"], s.camera["h"], 16
        a, b = film(w, h), film(w, h)
        run_wf([scenes.wf_frame(0, s.camera, spp, 5, d_film=a.data_ptr())], scenes.wf_params(128, 1 << 16, 2, 1))
        run_mk([scenes.wf_frame(0, s.camera, spp, 5, d_film=b.data_ptr())])
        torch.cuda.synchronize()
        wf, mk = a.cpu().numpy()[..., :3], b.cpu().numpy()[..., :3]
        orc = Oracle(r.built.payload, r.spec, r.hosek)
        o32 = orc.render(r.camera, 1, spp, threads=THREADS).reshape(h, w, 3)
        o64 = orc.render(r.camera, 1, spp, fp64=True, threads=THREADS).reshape(h, w, 3)
        orc.close()
        rel = lambda x, y: np.abs(x - y) / np.maximum(np.abs(y), 1e-2)
        assert (rel(wf, mk) > 1e-5).mean() < 1e-3
        e = rel(mk, o32)
        assert np.median(e) < 1e-5 and (e > 1e-3).mean() < 0.01, (float(np.median(e)), float((e > 1e-3).mean()))
        # the render's distance from FP64 is the FP32 oracle's
        e_mk = float(np.sqrt(np.mean((mk - o64) ** 2)))
        e_o = float(np.sqrt(np.mean((o32 - o64) ** 2)))
        assert e_mk <= 1.5 * e_o + 1e-6, (e_mk, e_o)
        assert mk.mean() > 0.05
        assert r.status(reset=True) == 0
    finally:
        r.close()


def test_alpha_cut_lets_rays_through_the_holes():
    """rays through a hole of the panel pass it; rays on the panel stop"""
    s = scenes.textured_room_scene()
    r = scenes.Renderer(s)
    try:
        from gpu_util import trace_closest
        # the panel spans (0.55..0.95, 0..1.5, -0.75..-0.2); aim rays at it
        # from the camera side along its normal
        n = np.array([-0.8, 0.0, 0.6]); n /= np.linalg.norm(n)
        rng = np.random.default_rng(3)
        t = rng.random((4000, 2))
        p = np.array([0.55, 0.0, -0.75]) + t[:, :1] * np.array([0.4, 0.0, 0.55]) + t[:, 1:] * np.array([0.0, 1.5, 0.0])
        rays = np.zeros((4000, 8), np.float32)
        # (tilted off the y = 0 plane: the reference's slab test misses boxes
        # along a zero direction component)
        dirs = -n + np.array([0.0, 0.013, 0.0])
        dirs /= np.linalg.norm(dirs)
        rays[:, :3] = p + 0.5 * n
        rays[:, 3] = np.inf
        rays[:, 4:7] = dirs
        hits = trace_closest(rays)
        b = scenes.BuiltPayload(s)
        spec = b.default_spec(5, 1)
        orc = Oracle(b.payload, spec, scenes.make_hosek(None))
        ref = orc.trace_closest(rays, 0, THREADS)
        orc.close()
        mats = np.array([b.payload.attribute_indices[4 * int(k) + 3] for k in hits[:, 1]])
        on_panel = (hits[:, 6] == 1) & (mats == 8)
        assert 0.2 < on_panel.mean() < 0.9, on_panel.mean()   # some rays pass through holes
        assert np.array_equal(hits[:, [1, 6]], ref[:, [1, 6]])
    finally:
        r.close()
