"""Image error against the FP64 oracle for the room (C1), the sky-lit
2.6M-triangle scene (C2) and the env-map MIS scene (C3), for the plain
megakernel and the wavefront integrator, at the configurations' sizes.

Two errors per integrator, on oracle-rendered pixels (all of C1; four full
rows of C2, two of C3):
  * precision: RMSE against the FP64 oracle on the same seeds (what FP32
    arithmetic and compensated accumulation cost);
  * estimator: RMSE against the FP64 oracle at 16x the samples.
The two integrators draw the same samples, so their errors must agree
(equal RMSE within 1 %); the precision error must be far below the
estimator's."""
import json

import numpy as np
import pytest
import torch

from noor_b200 import _capi, scenes
from oracle.oracle import Oracle

from gpu_util import THREADS

pytestmark = pytest.mark.gpu


def _wavefront(s, spp, bounces):
    import ctypes as C
    film = torch.zeros((s.camera["h"], s.camera["w"], 4), dtype=torch.float32, device="cuda")
    fr = (_capi.WfFrame * 1)(scenes.wf_frame(0, s.camera, spp, bounces, d_film=film.data_ptr()))
    p = scenes.wf_params(128, 1 << 21, 1, 1)
    _capi.call("noor_wavefront_render", fr, 1, C.byref(p))
    torch.cuda.synchronize()
    return film.cpu().numpy()[..., :3]


def _rows(h, n):
    return [int(h * (k + 1) / (n + 1)) for k in range(n)]


@pytest.mark.parametrize("config", ["C1", "C2", "C3"])
def test_rmse_against_fp64_oracle(config):
    if config == "C1":
        s = scenes.room_scene()
        rows, mult = list(range(s.camera["h"])), 16
    elif config == "C2":
        s = scenes.sky_scene()
        rows, mult = _rows(s.camera["h"], 4), 16
    else:
        s = scenes.env_scene()
        rows, mult = _rows(s.camera["h"], 2), 16
    spp, bounces = s.render["spp"], s.render["bounces"]
    r = scenes.Renderer(s)
    try:
        r.render(spp)
        mk = r.framebuffer()[..., :3]
        wf = _wavefront(s, spp, bounces)
        W = s.camera["w"]
        orc = Oracle(r.built.payload, r.spec, r.hosek)
        same, high = [], []
        for y in rows:
            same.append(orc.render(r.camera, 1, spp, p0=y * W, p1=(y + 1) * W, fp64=True, threads=THREADS))
            high.append(orc.render(r.camera, 1, spp * mult, p0=y * W, p1=(y + 1) * W, fp64=True, threads=THREADS))
        orc.close()
        same, high = np.concatenate(same), np.concatenate(high)
        sel = lambda img: np.concatenate([img[y] for y in rows])
        rm = lambda a, b: float(np.sqrt(np.mean((a - b) ** 2)))
        res = {"config": config, "pixels": len(rows) * W, "spp": spp, "reference_spp": spp * mult,
               "precision_rmse": {"megakernel": rm(sel(mk), same), "wavefront": rm(sel(wf), same)},
               "estimator_rmse": {"megakernel": rm(sel(mk), high), "wavefront": rm(sel(wf), high)},
               "mean": float(high.mean())}
        print("RMSE", json.dumps(res))
        e = res["estimator_rmse"]
        assert abs(e["wavefront"] - e["megakernel"]) <= 0.01 * e["megakernel"]
        p = res["precision_rmse"]
        assert max(p.values()) < 0.1 * e["megakernel"], res
        assert r.status() == 0
    finally:
        r.close()
