"""Scenes and records shared by the reference-device fixtures
(tests/golden/make_refdev_golden.py) and the tests that check against them.

The BSDF probe scene puts material k on its own triangle (2k, 0, 0),
(2k + 1, 0, 0), (2k, 1, 0) in the z = 0 plane, vertex normals +z, with uvs
chosen so that the reference's v flip (noor/cuda/mesh.cuh:145-148) leaves
du along +x and dv along +y: the shading frame of a hit is then exactly the
world axes, and local directions are world directions.  A probe ray
straight down at (2k + 0.25, 0.25) hits material k.
"""
from __future__ import annotations

import numpy as np

from noor_b200 import _capi, scenes

MATS = [scenes.material("diffuse", albedo=(0.2, 0.5, 0.8)),
        scenes.material("metal", roughness=float(np.sqrt(0.05))),
        scenes.material("metal", roughness=float(np.sqrt(0.5))),
        scenes.material("glass", ior=1.5),
        scenes.material("mirror", albedo=(0.9, 0.8, 0.7)),
        scenes.material("substrate", albedo=(0.3, 0.5, 0.7), specular=(0.04, 0.05, 0.06), roughness=0.3),
        scenes.material("translucent", albedo=(0.6, 0.5, 0.4)),
        scenes.material("glossy", albedo=(0.5, 0.3, 0.2), roughness=0.2, ior=1.5),
        scenes.material("roughglass", roughness=0.3, ior=1.5),
        scenes.material("clearcoat", albedo=(0.9, 0.9, 0.9), specular=(0.8, 0.6, 0.5), roughness=0.3, ior=1.5,
                        coat_weight=0.5, coat_sigma=0.4, coat_thickness=0.5),
        scenes.material("shadowcatcher")]

HOSEK = dict(turbidity=3.0, albedo=0.3, sun_lat=float(np.radians(60)), sun_lon=float(np.pi / 4), solar_scale=250.0,
             solar_radius_scale=2.0)


def probe_scene(mats=MATS) -> scenes.SceneData:
    M = len(mats)
    V = np.zeros((3 * M, 4), np.float32)
    for k in range(M):
        V[3 * k:3 * k + 3, :3] = [(2 * k, 0, 0), (2 * k + 1, 0, 0), (2 * k, 1, 0)]
    V[:, 3] = 1.0
    N = np.zeros((1, 4), np.float32)
    N[0, 2] = 1.0
    U = np.array([(0.0, 1.0), (1.0, 1.0), (0.0, 0.0)], np.float32)
    vi = np.arange(3 * M, dtype=np.uint32).reshape(M, 3)
    ni = np.zeros((M, 3), np.uint32)
    ui = np.tile(np.arange(3, dtype=np.uint32), (M, 1))
    meshes = [dict(tri_start=0, tri_count=M, to_global=scenes.IDENTITY, instance=-1, light_idx=-1)]
    s = scenes.SceneData(vertices=V, normals=N, uvs=U, vindices=vi, nindices=ni, uvindices=ui,
                         material_indices=np.arange(M, dtype=np.uint32), meshes=meshes, materials=list(mats),
                         skydome_type=_capi.NOOR_SKY_CONSTANT, name="probe")
    s.camera = dict(eye=(M, 0.5, 6.0), look_at=(M, 0.5, 0.0), up=(0.0, 1.0, 0.0), fov_deg=40.0, w=16, h=16)
    s.render = dict(spp=1, bounces=2, rr=1, mis=0)
    return s


PROBE_DIR = (np.array([1e-3, 2e-3, -1.0]) / np.linalg.norm([1e-3, 2e-3, -1.0])).astype(np.float32)


def unit_dirs(rng, n, zmin=0.05):
    out = []
    while sum(len(x) for x in out) < n:
        d = rng.normal(size=(2 * n, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        out.append(d[np.abs(d[:, 2]) > zmin])
    return np.concatenate(out)[:n]


def bsdf_records(rng, per_material, n_mats=len(MATS)) -> np.ndarray:
    """(n_mats * per_material, 16) probe records: wo, wi (local), probe
    origin and direction, seed (id, frame); grouped by material in runs of
    whole warps (per_material is rounded up to a multiple of 32), because
    the reference's texture reads need one texture object per warp"""
    per = -(-per_material // 32) * 32
    n = per * n_mats
    rec = np.zeros((n, 16), np.float32)
    rec[:, 0:3] = unit_dirs(rng, n)
    rec[:, 3:6] = unit_dirs(rng, n)
    k = np.repeat(np.arange(n_mats), per)
    rec[:, 6] = 2 * k + 0.25
    rec[:, 7] = 0.25
    rec[:, 8] = 1.0
    # slightly tilted: the reference's slab test misses every box for a ray
    # with an exactly zero direction component (noor/cuda/ray.cuh:200-206)
    rec[:, 9:12] = PROBE_DIR
    rec[:, 12] = np.arange(n)
    rec[:, 13] = 1 + rng.integers(0, 1000, n)
    return rec


def product_records(rec: np.ndarray, ref_out: np.ndarray = None) -> np.ndarray:
    """the same samples in noor_eval_bsdf's record layout: wo, wi, u (the
    uniforms the reference's Sample_f drew, when given), material index"""
    out = np.zeros((rec.shape[0], 16), np.float32)
    out[:, 0:6] = rec[:, 0:6]
    if ref_out is not None:
        out[:, 6:8] = ref_out[:, 8:10]
    out[:, 8] = np.floor(rec[:, 6] / 2.0)
    return out


def microfacet_records(rng, n) -> np.ndarray:
    rec = np.zeros((n, 12), np.float32)
    rec[:, 0] = rng.uniform(0.05, 1.0, n)
    rec[:, 1] = np.where(rng.random(n) < 0.5, rec[:, 0], rng.uniform(0.05, 1.0, n))
    rec[:, 2:5] = unit_dirs(rng, n)
    # half vectors: wo + wi for a random wi, in FP32
    wh = rec[:, 2:5] + unit_dirs(rng, n).astype(np.float32)
    rec[:, 5:8] = wh / np.linalg.norm(wh, axis=1, keepdims=True)
    rec[:, 8:10] = rng.random((n, 2))
    return rec


def fresnel_records(rng, n) -> np.ndarray:
    rec = np.zeros((n, 9), np.float32)
    rec[:, 0] = rng.uniform(-1, 1, n)
    rec[:, 1] = np.where(rng.random(n) < 0.5, 1.0, rng.uniform(1.0, 2.5, n))
    rec[:, 2] = np.where(rng.random(n) < 0.5, 1.5, rng.uniform(1.0, 2.5, n))
    rec[:, 3:6] = rng.uniform(0.1, 2.0, (n, 3))
    rec[:, 6:9] = rng.uniform(0.0, 5.0, (n, 3))
    rec[: n // 4, 3:6] = scenes.GOLD_ETA
    rec[: n // 4, 6:9] = scenes.GOLD_K
    return rec


def warp_records(rng, n) -> np.ndarray:
    rec = np.zeros((n, 3), np.float32)
    rec[:, :2] = rng.random((n, 2))
    rec[:, 2] = rng.uniform(-1.0, 1.0, n)
    rec[:8, :2] = [(0, 0), (0.5, 0.5), (1 - 2 ** -24, 0), (0, 1 - 2 ** -24), (0.25, 0.75), (0.5, 0), (0, 0.5), (1e-7, 1e-7)]
    return rec


def env_field(seed: int = 9, env_w: int = 256, env_h: int = 128) -> scenes.SceneData:
    """a 16-sphere field at subdivision 4 lit only by a log-normal + lobes
    HDR map (the env-lit configuration's map at reduced size)"""
    g, (c, r) = scenes.sphere_field(seed, 16, 4)
    s = scenes.SceneData(**g, skydome_type=_capi.NOOR_SKY_HDR, env=scenes.env_map(seed, width=env_w, height=env_h),
                         name="envfield")
    s.camera = dict(scenes.frame_spheres(c, r, seed), w=64, h=48)
    s.render = dict(spp=1, bounces=5, rr=1, mis=0)
    return s


def envdist_scene() -> scenes.SceneData:
    """four small spheres under a 256 x 128 HDR map: the scene the
    distribution fixture is taken on"""
    g, (c, r) = scenes.sphere_field(9, 4, 2)
    s = scenes.SceneData(**g, skydome_type=_capi.NOOR_SKY_HDR, env=scenes.env_map(9, width=256, height=128),
                         name="envdist")
    s.camera = dict(scenes.frame_spheres(c, r, 9), w=32, h=32)
    s.render = dict(spp=1, bounces=2, rr=1, mis=0)
    return s


ENV_ROWS = np.arange(0, 1024, 64)   # rows of the sky's 1024 x 1024 tables kept in the fixture


def trace_scenes():
    """the scenes closest-hit fixtures are taken on: the C1 room (with a
    sphere light node) and a 16-sphere field at subdivision 4"""
    room = scenes.room_scene(seed=1, width=64, height=64, spp=1, bounces=5, light="sphere")
    g, (c, r) = scenes.sphere_field(7, 16, 4)
    field = scenes.SceneData(**g, skydome_type=_capi.NOOR_SKY_PHYSICAL, name="field16")
    field.camera = dict(scenes.frame_spheres(c, r, 7), w=64, h=48)
    field.render = dict(spp=1, bounces=5, rr=1, mis=0)
    field.hosek = dict(HOSEK)
    return {"room": room, "field16": field}


# ------------------------------------------------------------------ checks
# Bars shared by the oracle (CPU) and the product (GPU) parity tests against
# the reference-device fixtures.  Each takes the fixture arrays and the
# candidate's outputs for the same inputs.

def rel_err(a, b, floor=1e-6):
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def check_microfacet(ref: np.ndarray, got: np.ndarray, exact: bool):
    """D, G, Pdf within 1e-5 relative (bit-identical when `exact`); the
    sampled half vector within 1e-6 absolute at the median, 1e-4 at the 99th
    and 2e-3 at the 99.9th percentile (visible-normal sampling at grazing
    incidence and small alpha divides by alpha, amplifying libm rounding)"""
    if exact:
        assert np.array_equal(got[:, :3], ref[:, :3])
    else:
        assert rel_err(got[:, :3], ref[:, :3], 1e-30).max() < 1e-5
    assert np.array_equal(got[:, 7], ref[:, 7])
    d = np.abs(got[:, 3:6] - ref[:, 3:6]).max(1)
    q = np.quantile(d, [0.5, 0.99, 0.999])
    assert q[0] < 1e-6 and q[1] < 1e-4 and q[2] < 2e-3, q


def check_warps(ref: np.ndarray, got: np.ndarray, tol: float = 5e-7):
    """warps within `tol` absolute (the cosine warp's z, a square root of a
    difference near the disk rim, within 1e-3); Erf / ErfInv within `tol`;
    the power heuristic within 1e-6 relative where defined"""
    cols = [0, 1, 2, 3, 5, 6, 7, 8, 9, 10, 11]
    assert np.abs(got[:, cols] - ref[:, cols]).max() < tol
    assert np.abs(got[:, 4] - ref[:, 4]).max() < 1e-3
    assert np.abs(got[:, 13:15] - ref[:, 13:15]).max() < tol
    ok = np.isfinite(ref[:, 12])
    assert np.array_equal(ok, np.isfinite(got[:, 12]))
    assert rel_err(got[ok, 12], ref[ok, 12]).max() < 1e-6


def check_fresnel(ref: np.ndarray, got: np.ndarray):
    """within 1e-5 absolute, 5e-5 relative at the 99.9th percentile"""
    assert np.abs(got - ref).max() < 1e-5
    assert np.quantile(rel_err(got, ref, 1e-30), 0.999) < 5e-5


def bsdf_materials(rec: np.ndarray) -> np.ndarray:
    return np.floor(rec[:, 6] / 2.0).astype(int)


def catcher_rows(rec: np.ndarray) -> np.ndarray:
    return np.array([MATS[m]["type"] == _capi.NOOR_SHADOWCATCHER for m in bsdf_materials(rec)])


def check_bsdf(kind: int, rec: np.ndarray, ref: np.ndarray, got: np.ndarray, constant_sky: float = 0.25):
    """got: (n, 8) outputs of noor_eval_bsdf / oracle_eval_bsdf for the probe
    records (noor_eval_bsdf's shadow catcher leaves out the sky factor the
    reference's lobe multiplies in; the probe scene's sky is the constant
    0.25).  Eval and Pdf within 1e-5 relative at the 99.9th percentile for
    every material but rough glass, whose microfacet transmission cancels in
    FP32 (1e-3 there); Sample_f picks the same lobe for every sample, the
    direction within 1e-4 absolute at the 99th percentile, value and pdf
    within 1e-3 relative at the 99th."""
    g = got.copy()
    g[catcher_rows(rec), :3] *= constant_sky
    assert (ref[:, 10] == 1).all() and np.array_equal(ref[:, 11], bsdf_materials(rec))
    rough = np.array([MATS[m]["type"] == _capi.NOOR_ROUGHGLASS for m in bsdf_materials(rec)])
    if kind < 2:
        cols = [0, 1, 2] if kind == 0 else [3]
        e = rel_err(g[:, cols], ref[:, cols]).max(1)
        q = np.quantile(e[~rough], 0.999)
        assert q < 1e-5, q
        assert np.quantile(e[rough], 0.999) < 1e-3
        return
    assert np.array_equal(g[:, 7], ref[:, 7])
    hit = ref[:, 3] != 0
    assert np.array_equal(hit, g[:, 3] != 0)
    dw = np.abs(g[hit, 4:7] - ref[hit, 4:7]).max(1)
    ev = rel_err(g[hit, 0:4], ref[hit, 0:4]).max(1)
    qw, qv = np.quantile(dw, [0.5, 0.99]), np.quantile(ev, [0.5, 0.99])
    assert qw[0] < 1e-6 and qw[1] < 1e-4, qw
    assert qv[0] < 1e-6 and qv[1] < 1e-3, qv


def check_trace(ref_hits: np.ndarray, ref_any: np.ndarray, hits: np.ndarray, occ: np.ndarray):
    """closest hit: hit flag, triangle and instance index, barycentrics and
    (where hit) t identical to the bit; any hit identical"""
    assert np.array_equal(hits[:, 6], ref_hits[:, 6])
    h = ref_hits[:, 6] == 1
    for c in (0, 1, 2, 4, 5):
        assert np.array_equal(hits[h, c], ref_hits[h, c]), c
    assert np.array_equal(occ, ref_any)


def check_camera_rays(ref: np.ndarray, got: np.ndarray, tol: float = 3e-7):
    """origins identical, directions within `tol` absolute (the reference's
    normalize is v * rsqrtf(dot(v, v)), an approximate reciprocal root)"""
    assert np.array_equal(got[:, 0:3], ref[:, 0:3])
    assert np.abs(got[:, 4:7] - ref[:, 4:7]).max() < tol


def check_film(ref: np.ndarray, got: np.ndarray, q50=1e-6, q99=1e-5, q999=1e-4):
    """per-pixel relative difference (floor 1e-3) below q50 / q99 / q999 at
    the median / 99th / 99.9th percentile, and the image means within 1e-3"""
    e = rel_err(got[..., :3], ref[..., :3], 1e-3).max(-1).ravel()
    q = np.quantile(e, [0.5, 0.99, 0.999])
    assert q[0] < q50 and q[1] < q99 and q[2] < q999, q
    m_got, m_ref = float(got[..., :3].mean()), float(ref[..., :3].mean())
    assert abs(m_got - m_ref) <= 1e-3 * abs(m_ref), (m_got, m_ref)
