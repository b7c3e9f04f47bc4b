"""The oracle's point, spot, distant, sphere and disk lights against closed
forms (CPU only).  A diffuse floor under one light, one bounce: the pixel
value is albedo / pi times the irradiance the light gives the hit point.
Delta lights are sampled without noise, so each pixel must equal the
formula to rounding; area lights are Monte Carlo estimates whose mean over
many samples must approach the on-axis value: for a sphere the irradiance
pi Le (r/d)^2 (its cone sampling is exact); for quads and disks the
expectation of the reference's own estimator, whose sampling pdf carries
one power of the distance too few (see reference_area_estimate)."""
import ctypes as C

import numpy as np
import pytest

from noor_b200 import _capi, scenes
from oracle.oracle import Oracle, lib, _p

ALBEDO = 0.6
W = H = 16


def floor_scene(**lights) -> scenes.SceneData:
    """a 40 x 40 diffuse floor at y = 0 seen from straight above, from
    below the lights"""
    V = np.array([[-20, 0, -20, 1], [20, 0, -20, 1], [20, 0, 20, 1], [-20, 0, 20, 1]], np.float32)
    N = np.array([[0, 1, 0, 0]], np.float32)
    vi = np.array([[0, 2, 1], [0, 3, 2]], np.uint32)
    s = scenes.SceneData(vertices=V, normals=N, uvs=np.zeros((1, 2), np.float32), vindices=vi,
                         nindices=np.zeros((2, 3), np.uint32), uvindices=np.zeros((2, 3), np.uint32),
                         material_indices=np.zeros(2, np.uint32),
                         meshes=[dict(tri_start=0, tri_count=2, to_global=scenes.IDENTITY, instance=-1,
                                      light_idx=-1)],
                         materials=[scenes.material("diffuse", albedo=(ALBEDO,) * 3)],
                         camera=dict(eye=(0.0, 1.0, 0.0), look_at=(0.0, 0.0, 0.0), up=(0.0, 0.0, -1.0),
                                     fov_deg=30.0, w=W, h=H), name="floor", **lights)
    if s.area_lights:
        s.meshes.append(dict(tri_start=0, tri_count=0, to_global=scenes.IDENTITY, instance=-1, light_idx=0))
    return s


def render(s, spp, fp64=True, mis=0):
    b = scenes.BuiltPayload(s)
    spec = b.default_spec(1, 8)
    spec.mis = mis
    cam = scenes.make_camera(s.camera)
    o = Oracle(b.payload, spec, scenes.make_hosek(None))
    img = o.render(cam, 1, spp, fp64=fp64, threads=8).reshape(H, W, 3)   # mean over the samples
    rays = np.zeros((W * H, 8), np.float32)
    lib().oracle_camera_rays(C.addressof(cam), 1, _p(rays))
    o.close()
    return img, rays, b


def floor_points(rays):
    o, d = rays[:, 0:3].astype(np.float64), rays[:, 4:7].astype(np.float64)
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    t = -o[:, 1] / d[:, 1]
    return o + t[:, None] * d


@pytest.mark.parametrize("fp64", [True, False])
def test_point_light_is_inverse_square(fp64):
    P, ke = np.array([0.3, 1.5, -0.2]), np.array([3.0, 2.0, 1.0])
    img, rays, _ = render(floor_scene(point_lights=[dict(position=tuple(P), ke=tuple(ke))]), 1, fp64)
    x = floor_points(rays)
    v = P - x
    d2 = (v ** 2).sum(1)
    cos = v[:, 1] / np.sqrt(d2)
    want = (ALBEDO / np.pi) * ke[None] * (cos / d2)[:, None]
    np.testing.assert_allclose(img.reshape(-1, 3), want, rtol=1e-5 if fp64 else 1e-4)


def test_spot_light_falloff():
    P, ke = np.array([0.0, 2.0, 0.0]), np.array([4.0, 4.0, 4.0])
    ci, co = np.cos(np.radians(3.0)), np.cos(np.radians(8.0))
    img, rays, _ = render(floor_scene(spot_lights=[dict(position=tuple(P), direction=(0.0, 1.0, 0.0), ke=tuple(ke),
                                                        cos_inner=float(ci), cos_outer=float(co))]), 1)
    x = floor_points(rays)
    v = P - x
    d2 = (v ** 2).sum(1)
    w = v / np.sqrt(d2)[:, None]
    c = np.float64(np.float32(1.0)) * w[:, 1]          # dot(direction, point-to-light)
    fo = np.where(c < np.float32(co), 0.0, np.where(c >= np.float32(ci), 1.0,
                                                     ((c - np.float32(co)) / (np.float32(ci) - np.float32(co))) ** 4))
    want = (ALBEDO / np.pi) * ke[None] * (fo * w[:, 1] / d2)[:, None]
    # the falloff's kink at cos_outer / cos_inner can flip one rounding
    # step away; everywhere else the pixel is the formula
    ok = np.isclose(img.reshape(-1, 3), want, rtol=1e-5, atol=1e-7).all(1)
    assert ok.mean() > 0.98
    assert (fo > 0).any() and (fo == 0).any() and ((fo > 0) & (fo < 1)).any()


def test_distant_light_is_cosine():
    dirn = np.array([0.3, 1.0, 0.2])
    ke = np.array([2.0, 1.5, 1.0])
    img, _, b = render(floor_scene(distant_lights=[dict(direction=tuple(dirn), ke=tuple(ke))]), 1)
    u = dirn / np.linalg.norm(dirn)
    stored = np.ctypeslib.as_array(b.payload.distant_lights, (1,))[0]
    assert np.allclose(np.array(stored["direction"]), u, atol=1e-6)    # normalised by the builder
    want = (ALBEDO / np.pi) * ke * u[1]
    np.testing.assert_allclose(img.reshape(-1, 3), np.broadcast_to(want, (W * H, 3)), rtol=1e-5)


def centre_mean(img):
    return img[H // 2 - 1:H // 2 + 1, W // 2 - 1:W // 2 + 1].mean(axis=(0, 1))


def test_sphere_light_matches_solid_angle():
    r, h = 0.25, 1.5
    Le = np.array([2.0, 2.0, 2.0])
    sph = dict(type="sphere", center=(-r, h, -r), u=(2 * r, 0.0, 0.0), v=(0.0, 0.0, 2 * r), ke=tuple(Le))
    img, _, b = render(floor_scene(area_lights=[sph]), 4096)
    sh = b.payload.area_lights[0].shape
    assert sh.type == _capi.NOOR_SHAPE_SPHERE and abs(sh.center[1] - h) < 1e-6 and abs(sh.radius - r) < 1e-6
    # the centre pixels see floor points within ~0.03 of the axis
    want = ALBEDO * Le * (r / h) ** 2
    np.testing.assert_allclose(centre_mean(img), want, rtol=0.01)


def reference_area_estimate(Le, h, inside, half):
    """mean of the reference's quad / disk light estimator at the floor
    point below the light's centre: its sampling pdf divides by |n . w|
    with w = P - p unnormalised (noor/cuda/geometry.cuh:37-38, 98-100), so
    each sample is Le f cos_x cos_l A / d instead of / d^2; the mean is
    (albedo / pi) Le times the integral of cos_x cos_l / d over the light
    (midpoint rule on a 2000^2 grid)"""
    n = 2000
    xs = (np.arange(n) + 0.5) / n * 2 * half - half
    X, Z = np.meshgrid(xs, xs)
    d2 = X ** 2 + Z ** 2 + h * h
    g = (h * h / d2) / np.sqrt(d2)
    return (ALBEDO / np.pi) * Le * np.sum(g[inside(X, Z)]) * (2 * half / n) ** 2


@pytest.mark.parametrize("kind", ["quad", "disk"])
def test_quad_and_disk_lights_follow_the_reference_estimator(kind):
    r, h = 0.5, 1.2
    Le = np.array([3.0, 3.0, 3.0])
    # u x v = (0, -1, 0): the light faces the floor
    light = dict(type=kind, center=(-r, h, -r), u=(2 * r, 0.0, 0.0), v=(0.0, 0.0, 2 * r), ke=tuple(Le))
    img, _, _ = render(floor_scene(area_lights=[light]), 4096)
    inside = (lambda X, Z: X ** 2 + Z ** 2 <= r * r) if kind == "disk" else (lambda X, Z: np.ones_like(X, bool))
    want = reference_area_estimate(Le, h, inside, r)
    if kind == "disk":   # closed form of the same integral on the axis
        assert np.allclose(want, 2 * ALBEDO * Le * h * (1 - h / np.sqrt(h * h + r * r)), rtol=1e-4)
    np.testing.assert_allclose(centre_mean(img), want, rtol=0.01)


def test_one_sided_disk_facing_away_is_dark():
    r, h = 0.5, 1.2
    disk = dict(type="disk", center=(-r, h, -r), u=(0.0, 0.0, 2 * r), v=(2 * r, 0.0, 0.0), ke=(3.0, 3.0, 3.0))
    img, _, _ = render(floor_scene(area_lights=[disk]), 64)
    assert img.max() == 0.0


def test_shadow_catcher_is_a_shadow_matte():
    """a shadow-catcher floor under a point light, one bounce: where the
    light is unblocked the pixel is the sky seen along the camera ray
    (direct.cuh:51, bxdf.cuh:213-218), under the blocker it is 0"""
    s = floor_scene(point_lights=[dict(position=(0.6, 1.5, 0.0), ke=(3.0, 3.0, 3.0))])
    s.materials = [scenes.material("shadowcatcher"), scenes.material("diffuse")]
    # a small blocker between the light and part of the floor (material 1)
    q = np.array([[-0.05, 0.5, -0.05, 1], [0.15, 0.5, -0.05, 1], [0.15, 0.5, 0.15, 1], [-0.05, 0.5, 0.15, 1]],
                 np.float32)
    s.vertices = np.concatenate([s.vertices, q])
    s.vindices = np.concatenate([s.vindices, np.array([[4, 5, 6], [4, 6, 7]], np.uint32)])
    s.nindices = np.zeros((4, 3), np.uint32)
    s.uvindices = np.zeros((4, 3), np.uint32)
    s.material_indices = np.array([0, 0, 1, 1], np.uint32)
    s.meshes = [dict(tri_start=0, tri_count=4, to_global=scenes.IDENTITY, instance=-1, light_idx=-1)]
    img, rays, b = render(s, 1)
    env = b.payload.textures[b.payload.num_textures - 1]
    sky = np.array(env.rgba[0:3])
    assert env.width == 1 and env.height == 1 and sky.max() > 0
    # floor pixels in the blocker's shadow (the light is off to the side, so
    # part of the shadow is not hidden behind the blocker)
    x = floor_points(rays)
    P = np.array([0.6, 1.5, 0.0])
    t = (0.5 - x[:, 1]) / (P[1] - x[:, 1])
    hit = x + t[:, None] * (P - x)
    shadow = (hit[:, 0] > -0.05) & (hit[:, 0] < 0.15) & (hit[:, 2] > -0.05) & (hit[:, 2] < 0.15)
    # pixels whose camera ray meets the blocker first show the blocker
    o, d = rays[:, 0:3].astype(np.float64), rays[:, 4:7].astype(np.float64)
    tb = (0.5 - o[:, 1]) / d[:, 1]
    pb = o + tb[:, None] * d
    on_blocker = (pb[:, 0] > -0.05) & (pb[:, 0] < 0.15) & (pb[:, 2] > -0.05) & (pb[:, 2] < 0.15)
    pix = img.reshape(-1, 3)
    lit = ~shadow & ~on_blocker
    assert lit.sum() > 50 and (shadow & ~on_blocker).sum() > 3
    np.testing.assert_allclose(pix[lit], np.broadcast_to(sky, (lit.sum(), 3)), rtol=1e-5)
    # pixels whose shadow ray passes within the blocker's edge may go
    # either way (the shadow ray starts off the floor by the bias)
    dark = pix[shadow & ~on_blocker].max(1) == 0
    assert dark.mean() > 0.8, dark.mean()


def _camera_rays(cam_dict, frame=1):
    cam = scenes.make_camera(cam_dict)
    rays = np.zeros((cam.w * cam.h, 8), np.float32)
    lib().oracle_camera_rays(C.addressof(cam), frame, _p(rays))
    return cam, rays[:, 0:3].astype(np.float64), rays[:, 4:7].astype(np.float64)


def test_orthographic_camera_rays_are_parallel():
    """CudaOrthoCamera: every ray along the camera's -z, origins spread over
    the window"""
    base = dict(eye=(0.0, 1.0, 3.0), look_at=(0.0, 1.0, 0.0), up=(0.0, 1.0, 0.0), fov_deg=40.0, w=16, h=12)
    _, o, d = _camera_rays(dict(base, type="ortho", ortho_scale=2.0))
    assert np.allclose(d, [0.0, 0.0, -1.0], atol=1e-6)
    assert np.allclose(o[:, 2], 3.0, atol=1e-5)
    assert o[:, 0].min() < -0.8 and o[:, 0].max() > 0.8 and o[:, 1].min() < 0.4 and o[:, 1].max() > 1.6


def test_environment_camera_covers_the_sphere():
    """CudaEnvCamera: the centre pixel looks along the camera's -z, the
    image spans all longitudes and latitudes"""
    base = dict(eye=(0.0, 0.0, 0.0), look_at=(0.0, 0.0, -1.0), up=(0.0, 1.0, 0.0), fov_deg=40.0, w=64, h=32)
    cam, o, d = _camera_rays(dict(base, type="env"))
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-6) and np.allclose(o, 0.0)
    c = d.reshape(32, 64, 3)[16, 32]
    assert c[2] < -0.99
    assert d[:, 1].min() < -0.95 and d[:, 1].max() > 0.95            # both poles
    assert (d[:, 0] > 0.9).any() and (d[:, 0] < -0.9).any() and (d[:, 2] > 0.9).any()


def test_thin_lens_rays_meet_on_the_plane_of_focus():
    """thin lens: rays of one pixel from different lens points cross the
    plane of focus at one point (the pinhole ray's)"""
    base = dict(eye=(0.0, 1.0, 4.0), look_at=(0.0, 1.0, 0.0), up=(0.0, 1.0, 0.0), fov_deg=40.0, w=8, h=8)
    f = 3.0
    pts = []
    for frame in (1, 2, 3):
        _, o, d = _camera_rays(dict(base, lens_radius=0.2, focal_length=f), frame)
        _, o0, d0 = _camera_rays(base, frame)
        assert np.abs(o - o0).max() > 1e-3                              # origins on the lens
        t = (4.0 - f - o[:, 2]) / d[:, 2]                                 # plane z = 4 - f
        t0 = (4.0 - f - o0[:, 2]) / d0[:, 2]
        assert np.allclose(o + t[:, None] * d, o0 + t0[:, None] * d0, atol=2e-4)
