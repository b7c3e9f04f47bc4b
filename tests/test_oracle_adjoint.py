"""The oracle's FP64 reference gradient of the detached-sampling estimator
against central differences of its own FP64 forward (CPU only).  The
sampling is detached, so the estimator is a smooth function of the
parameters and the two must agree to FP64 rounding (albedo and env enter
linearly) or to the difference step's truncation error (roughness)."""
import numpy as np
import pytest

from noor_b200 import _capi, scenes
from noor_b200.adjoint import scene_parameters
from oracle.oracle import Oracle


@pytest.fixture(scope="module")
def small():
    s = scenes.adjoint_scene(width=16, height=16, spp=2, count=4, level=2, n_materials=8, env_w=32, env_h=16)
    b = scenes.BuiltPayload(s)
    spec = b.default_spec(4, 4)
    spec.mis = 1
    hk = scenes.make_hosek(None)
    cam = scenes.make_camera(s.camera)
    o = Oracle(b.payload, spec, hk)
    alb, rough, env = (t.numpy() for t in scene_parameters(s, device="cpu"))
    gi = np.random.default_rng(0).normal(size=(16 * 16, 3)).astype(np.float32)
    yield o, cam, alb, rough, env, gi
    o.close()


def test_scene_parameters_follow_materials(small):
    _, _, alb, rough, env, _ = small
    assert alb.shape == (8, 3) and rough.shape == (8,) and env.shape == (16, 32, 3)
    assert (alb > 0.1 - 1e-6).all() and (alb < 0.9 + 1e-6).all()


def test_oracle_gradient_matches_fp64_differences(small):
    o, cam, alb, rough, env, gi = small
    img, ga, gr, ge = o.adjoint(cam, 1, 2, 4, alb, rough, env, gi)
    assert np.isfinite(img).all() and img.mean() > 0

    def loss(a, r, e):
        return float((o.adjoint(cam, 1, 2, 4, a, r, e) * gi).sum())

    scale = max(np.abs(ga).max(), np.abs(gr).max())
    for i in range(alb.shape[0]):
        for c in range(3):
            a1, a2 = alb.copy(), alb.copy()
            a1[i, c] += 1e-3
            a2[i, c] -= 1e-3
            fd = (loss(a1, rough, env) - loss(a2, rough, env)) / (float(a1[i, c]) - float(a2[i, c]))
            assert abs(fd - ga[i, c]) <= 1e-7 * scale + 1e-7 * abs(fd), (i, c, ga[i, c], fd)
        r1, r2 = rough.copy(), rough.copy()
        r1[i] += 1e-4
        r2[i] -= 1e-4
        fd = (loss(alb, r1, env) - loss(alb, r2, env)) / (float(r1[i]) - float(r2[i]))
        assert abs(fd - gr[i]) <= 1e-5 * scale + 1e-4 * abs(fd), (i, gr[i], fd)
    assert np.count_nonzero(gr) >= 2 and np.count_nonzero(ga) >= 6
    nz = np.argwhere(ge != 0)
    assert len(nz) > 100
    escale = np.abs(ge).max()
    for (y, x, c) in nz[:: max(1, len(nz) // 16)]:
        e1, e2 = env.copy(), env.copy()
        e1[y, x, c] += 1e-2
        e2[y, x, c] -= 1e-2
        fd = (loss(alb, rough, e1) - loss(alb, rough, e2)) / (float(e1[y, x, c]) - float(e2[y, x, c]))
        assert abs(fd - ge[y, x, c]) <= 1e-8 * escale + 1e-7 * abs(fd), (y, x, c, ge[y, x, c], fd)


def test_env_footprint_bounds_the_gradient(small):
    """the forward footprint (oracle_env_footprint) holds every texel with a
    non-zero gradient, and a texel outside it leaves the image unchanged"""
    o, cam, alb, rough, env, gi = small
    foot = o.env_footprint(cam, 1, 2, 4, alb, rough, env)
    assert foot.shape == env.shape[:2] and foot.sum() > 0
    _, _, _, ge = o.adjoint(cam, 1, 2, 4, alb, rough, env, gi)
    assert not ((ge != 0).any(axis=2) & (foot == 0)).any()
    img = o.adjoint(cam, 1, 2, 4, alb, rough, env)
    outside = np.argwhere(foot == 0)
    assert len(outside) > 0
    for (y, x) in outside[:: max(1, len(outside) // 8)]:
        e = env.copy()
        e[y, x] += 1.0
        assert np.array_equal(o.adjoint(cam, 1, 2, 4, alb, rough, e), img)
    inside = np.argwhere(foot > 0)
    changed = 0
    for (y, x) in inside[:: max(1, len(inside) // 8)]:
        e = env.copy()
        e[y, x] += 1.0
        changed += int(not np.array_equal(o.adjoint(cam, 1, 2, 4, alb, rough, e), img))
    assert changed == len(inside[:: max(1, len(inside) // 8)])
