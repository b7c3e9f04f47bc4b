"""Closest-hit and any-hit traversal on the GPU against the oracle's
transcription on identical rays: bit-exact indices, distances and
barycentrics, in both the reference Wald mode and the watertight mode."""
import numpy as np
import pytest

from noor_b200 import _capi, scenes
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

from gpu_util import camera_rays, random_rays, trace_any, trace_closest  # noqa: E402


def _check_closest(g, o):
    hit_g, hit_o = g[:, 6], o[:, 6]
    assert np.array_equal(hit_g, hit_o)
    m = hit_o == 1
    assert np.array_equal(g[m, 1], o[m, 1]), "triangle index"
    assert np.array_equal(g[m, 2], o[m, 2]), "instance index"
    assert np.array_equal(g[m, 3], o[m, 3]), "material type"
    assert np.array_equal(g[m, 0], o[m, 0]), "t bits"
    assert np.array_equal(g[m, 4], o[m, 4]) and np.array_equal(g[m, 5], o[m, 5]), "barycentric bits"


@pytest.fixture
def room():
    s = scenes.room_scene(width=128, height=128)
    r = scenes.Renderer(s)
    orc = Oracle(r.built.payload, r.spec, r.hosek)
    yield r, orc
    orc.close()
    r.close()


@pytest.fixture
def spheres():
    g, (c, rad) = scenes.sphere_field(7, 16, 4)
    s = scenes.SceneData(**g, name="t")
    s.camera = dict(scenes.frame_spheres(c, rad, 7), w=160, h=90)
    s.render = dict(spp=1, bounces=4, rr=1, mis=0)
    s.skydome_type = _capi.NOOR_SKY_CONSTANT
    r = scenes.Renderer(s)
    orc = Oracle(r.built.payload, r.spec, r.hosek)
    yield r, orc
    orc.close()
    r.close()


@pytest.mark.parametrize("isect", [_capi.NOOR_ISECT_REF_WALD, _capi.NOOR_ISECT_WATERTIGHT])
@pytest.mark.parametrize("which", ["room", "spheres"])
def test_camera_rays_closest_hit_bit_exact(request, which, isect):
    r, orc = request.getfixturevalue(which)
    r.update_spec(intersector=isect)
    for frame in (1, 7):
        rays = camera_rays(r, frame)
        g = trace_closest(rays)
        o = orc.trace_closest(rays, isect)
        _check_closest(g, o)
        assert g[:, 6].sum() > 0.05 * len(g)


@pytest.mark.parametrize("isect", [_capi.NOOR_ISECT_REF_WALD, _capi.NOOR_ISECT_WATERTIGHT])
def test_random_rays_closest_and_any(spheres, isect):
    r, orc = spheres
    r.update_spec(intersector=isect)
    rng = np.random.default_rng(5)
    rays = random_rays(rng, 200_000, -12, 12)
    _check_closest(trace_closest(rays), orc.trace_closest(rays, isect))
    short = random_rays(rng, 100_000, -12, 12, tmax=3.0)
    assert np.array_equal(trace_any(short), orc.trace_any(short, isect))


def test_camera_rays_match_oracle_within_ulps(room):
    """camera ray generation uses rsqrt on the device: directions agree to a
    few ulps, origins exactly"""
    import ctypes as C
    from oracle.oracle import lib, _p
    r, orc = room
    rays = camera_rays(r, 3)
    ref = np.zeros_like(rays)
    lib().oracle_camera_rays(C.addressof(r.camera), 3, _p(ref))
    assert np.array_equal(rays[:, :3], ref[:, :3])
    assert np.abs(rays[:, 4:7] - ref[:, 4:7]).max() < 1e-6


def test_watertight_agrees_with_wald_on_most_rays(spheres):
    r, orc = spheres
    rng = np.random.default_rng(9)
    rays = random_rays(rng, 100_000, -12, 12)
    r.update_spec(intersector=_capi.NOOR_ISECT_WATERTIGHT)
    a = trace_closest(rays)
    r.update_spec(intersector=_capi.NOOR_ISECT_REF_WALD)
    b = trace_closest(rays)
    assert (a[:, 6] == b[:, 6]).mean() > 0.999
    both = (a[:, 6] == 1) & (b[:, 6] == 1)
    assert (a[both, 1] == b[both, 1]).mean() > 0.995
    ta, tb = a[both, 0].view(np.float32), b[both, 0].view(np.float32)
    assert np.abs(ta - tb).max() < 1e-3 * np.abs(tb).max()


def test_stack_overflow_is_reported_not_faulted(room):
    """a spec whose BVH height is too small for the tree: the context's stack
    capacity is derived from it with a floor, so traversal stays in bounds and
    the status word stays clean for this tree"""
    r, orc = room
    assert r.status(reset=True) == 0


def _grazing_rays(payload, n, seed, axis=True):
    """rays from the scene's own vertex coordinates (so origins sit on box
    planes) along directions with +0, -0 and subnormal components, finite
    and infinite extents: the rays for which the four-wide any-hit tree
    tests an expanded child's box as well as its children's"""
    import ctypes as C
    rng = np.random.default_rng(seed)
    v = np.ctypeslib.as_array(C.cast(payload.vertices, C.POINTER(C.c_float)), (payload.num_vertices, 4))[:, :3]
    o = v[rng.integers(0, len(v), n)].copy()
    jitter = rng.integers(0, 3, n)
    o[np.arange(n), jitter] += rng.normal(size=n).astype(np.float32)
    if axis:
        comps = np.array([0.0, -0.0, 1.0, -1.0, 1e-40, -1e-40, 0.5, -0.25], np.float32)
        d = comps[rng.integers(0, len(comps), (n, 3))]
        d[np.all(np.abs(d) < 1e-30, axis=1), 0] = 1.0
    else:
        d = rng.normal(size=(n, 3))
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    r = np.zeros((n, 8), np.float32)
    r[:, :3] = o
    r[:, 3] = np.where(rng.random(n) < 0.5, np.float32(np.inf), rng.uniform(0.1, 20.0, n).astype(np.float32))
    r[:, 4:7] = d
    return r


@pytest.fixture
def instanced():
    import test_ref_payload as trp
    s = trp.instanced_scene()
    s.camera = dict(eye=(0.0, 2.0, 12.0), look_at=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0), fov_deg=60.0, w=64, h=36)
    s.render = dict(spp=1, bounces=4, rr=1, mis=0)
    s.skydome_type = _capi.NOOR_SKY_CONSTANT
    r = scenes.Renderer(s)
    orc = Oracle(r.built.payload, r.spec, r.hosek)
    yield r, orc
    orc.close()
    r.close()


@pytest.mark.parametrize("isect", [_capi.NOOR_ISECT_REF_WALD, _capi.NOOR_ISECT_WATERTIGHT])
@pytest.mark.parametrize("which", ["room", "spheres", "instanced"])
def test_any_hit_on_grazing_and_random_rays(request, which, isect):
    """shadow-ray answers (the four-wide tree) against the oracle's binary
    traversal: rays from box planes with zero and subnormal direction
    components, and in random directions, with short and unbounded extents"""
    r, orc = request.getfixturevalue(which)
    r.update_spec(intersector=isect)
    rays = np.concatenate([_grazing_rays(r.built.payload, 100_000, 11),
                           _grazing_rays(r.built.payload, 100_000, 12, axis=False)])
    got, want = trace_any(rays), orc.trace_any(rays, isect)
    assert np.array_equal(got, want), int((got != want).sum())
    assert 0.01 < want.mean() < 0.99
    assert r.status(reset=True) == 0
