"""Seeded synthetic scenes for the five configurations, and the host-side
plumbing that turns them into a payload (BVH + Wald records + materials),
a camera, a spec and a sky through the C-ABI.

Scenes are generated as the loader output Noor's Model consumes
(noor/header/assetLoader.h:103-162): shared vertex/normal/uv arrays with
per-triangle index triples, per-triangle material indices, meshes with
transforms, constant materials and quad area lights.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional

import numpy as np

from . import _capi as capi

GOLD_ETA = (0.126052, 0.465040, 1.340442)   # Au, as in the reference's material presets
GOLD_K = (4.230981, 2.204432, 1.642458)
DEFAULT_BVH = dict(num_bins=16, max_height=32, Ci=1.0, Ct=0.125, min_leaf_tris=2, max_leaf_tris=4)
# the Hosek-Wilkie RGB tables (BSD-3, data/HOSEK_WILKIE_LICENSE), written by
# data/make_hosek_data.py from the model's published data header
HOSEK_DATASET = Path(__file__).resolve().parent / "data" / "hosek_rgb.npy"

IDENTITY = np.eye(4, dtype=np.float32).reshape(-1, order="F")


def material(kind: str, albedo=(0.5, 0.5, 0.5), roughness: float = 0.1, ior: float = 1.5,
             emittance=(0.0, 0.0, 0.0), distribution: int = 0, specular=(1.0, 1.0, 1.0), coat_weight: float = 1.0,
             coat_sigma: float = 0.0, coat_thickness: float = 1.0) -> dict:
    """Constant material parameters (AssetLoader getters) for one of
    'diffuse', 'metal' (gold conductor, `specular` tints it), 'glass',
    'emitter', 'mirror' (albedo is the reflectance), 'substrate' (Fresnel
    blend of the albedo under a `specular` coat), 'translucent' (albedo
    reflected and transmitted), 'glossy' (albedo under a dielectric
    microfacet coat), 'roughglass' (dielectric microfacet reflection and
    transmission), 'clearcoat' (a gold microfacet substrate tinted by
    `specular` under a dielectric coat of index `ior` whose reflection is
    tinted by `albedo`; `coat_weight` sets how often the coat is sampled,
    `coat_sigma` x `coat_thickness` its absorption) or 'shadowcatcher'
    (shows the sky where lights reach it)."""
    types = {"diffuse": capi.NOOR_DIFFUSE, "metal": capi.NOOR_METAL, "glass": capi.NOOR_GLASS,
             "emitter": capi.NOOR_EMITTER, "mirror": capi.NOOR_MIRROR, "substrate": capi.NOOR_SUBSTRATE,
             "translucent": capi.NOOR_TRANSLUCENT, "glossy": capi.NOOR_GLOSSY, "roughglass": capi.NOOR_ROUGHGLASS,
             "clearcoat": capi.NOOR_CLEARCOAT, "shadowcatcher": capi.NOOR_SHADOWCATCHER}
    gold = kind in ("metal", "clearcoat")
    return dict(diffuse=tuple(albedo), specular=tuple(float(x) for x in specular), transmission=(1.0, 1.0, 1.0),
                emittance=tuple(emittance), transparency=(1.0, 1.0, 1.0),
                ior=GOLD_ETA if gold else (ior, ior, ior), k=GOLD_K if gold else (0, 0, 0),
                roughness=(roughness, roughness), coat_weight=coat_weight, coat_roughness=0.001,
                coat_thickness=coat_thickness, coat_sigma=coat_sigma, coat_ior=ior, emitter_scale=1.0,
                type=types[kind], distribution=distribution)


@dataclass
class SceneData:
    vertices: np.ndarray           # (V,4) f32
    normals: np.ndarray            # (N,4) f32
    uvs: np.ndarray                # (U,2) f32
    vindices: np.ndarray           # (T,3) u32
    nindices: np.ndarray
    uvindices: np.ndarray
    material_indices: np.ndarray   # (T,) u32
    meshes: list
    materials: list
    area_lights: list = field(default_factory=list)
    point_lights: list = field(default_factory=list)     # dict(position, ke)
    spot_lights: list = field(default_factory=list)      # dict(position, direction, ke, cos_inner, cos_outer)
    distant_lights: list = field(default_factory=list)   # dict(direction, ke)
    skydome_type: int = capi.NOOR_SKY_CONSTANT
    env: Optional[np.ndarray] = None   # (H,W,4) f32
    images: list = field(default_factory=list)   # image maps, (H,W,4) f32 each, named by materials' "map"
    bvh: dict = field(default_factory=lambda: dict(DEFAULT_BVH))
    camera: dict = field(default_factory=dict)
    render: dict = field(default_factory=dict)
    hosek: Optional[dict] = None
    name: str = ""

    @property
    def num_triangles(self) -> int:
        return int(self.vindices.shape[0])


# ----------------------------------------------------------------- C1 room
def _quad(points, inward):
    """two triangles (a,b,c),(a,c,d) wound so cross(b-a, c-a) follows `inward`"""
    a, b, c, d = [np.asarray(p, np.float64) for p in points]
    n = np.cross(b - a, c - a)
    if np.dot(n, inward) < 0:
        a, b, c, d = a, d, c, b
    return [a, b, c, d]


def _box(center, size, angle_deg):
    """6 faces (4 corners each) of a y-rotated box with outward orientation"""
    cx, cy, cz = center
    sx, sy, sz = size
    t = np.radians(angle_deg)
    R = np.array([[np.cos(t), 0, np.sin(t)], [0, 1, 0], [-np.sin(t), 0, np.cos(t)]])
    c = np.array(center, np.float64)
    faces = []
    for axis in range(3):
        for s in (-1.0, 1.0):
            n = np.zeros(3)
            n[axis] = s
            u = np.zeros(3)
            v = np.zeros(3)
            u[(axis + 1) % 3] = 1
            v[(axis + 2) % 3] = 1
            half = np.array([sx, sy, sz]) / 2
            pts = []
            for du, dv in ((-1, -1), (1, -1), (1, 1), (-1, 1)):
                p = n * half + du * u * half + dv * v * half
                pts.append(c + R @ p)
            faces.append((_quad(pts, R @ n), R @ n))
    return faces


def room_scene(seed: int = 1, width: int = 256, height: int = 256, spp: int = 16, bounces: int = 5,
               rr: int = 1, mis: bool = False, box_materials=None, light: str = "quad") -> SceneData:
    """C1: closed room of 5 wall quads + 1 ceiling light quad + 2 rotated
    boxes = 36 triangles, one mesh; wall albedo U[0.2,0.8]^3 from `seed`.
    `box_materials`: two material dicts for the short and the tall box
    (default: one diffuse grey for both).  `light` replaces the emissive
    ceiling quad: "sphere" or "disk" (an area light under the ceiling, in
    the BVH as a light node), "point", "spot" (aimed at the floor) or
    "distant" (the ceiling removed, light from above at an angle)."""
    rng = np.random.default_rng(seed)
    faces = []   # (corners, normal, material)
    walls = [
        ([(-1, 0, 1), (1, 0, 1), (1, 0, -1), (-1, 0, -1)], (0, 1, 0)),     # floor
        ([(-1, 2, 1), (1, 2, 1), (1, 2, -1), (-1, 2, -1)], (0, -1, 0)),    # ceiling
        ([(-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1)], (0, 0, 1)),   # back
        ([(-1, 0, -1), (-1, 0, 1), (-1, 2, 1), (-1, 2, -1)], (1, 0, 0)),   # left
        ([(1, 0, -1), (1, 0, 1), (1, 2, 1), (1, 2, -1)], (-1, 0, 0)),      # right
    ]
    if light == "distant":
        walls = walls[:1] + walls[2:]
    mats = []
    for i, (pts, n) in enumerate(walls):
        mats.append(material("diffuse", albedo=tuple(rng.uniform(0.2, 0.8, 3))))
        faces.append((_quad(pts, np.array(n, np.float64)), np.array(n, np.float64), i))
    box_mat = len(mats)
    if box_materials is None:
        mats.append(material("diffuse", albedo=(0.7, 0.7, 0.7)))
        box_ids = (box_mat, box_mat)
    else:
        mats.extend(box_materials)
        box_ids = (box_mat, box_mat + 1)
    for b, corners_list in enumerate((_box((0.35, 0.3, 0.25), (0.6, 0.6, 0.6), 17.0),
                                      _box((-0.33, 0.6, -0.3), (0.6, 1.2, 0.6), -18.0))):
        for corners_n in corners_list:
            faces.append((corners_n[0], corners_n[1], box_ids[b]))
    ke = (17.0, 12.0, 4.0)
    ly, h = 1.98, 0.25
    if light == "quad":
        light_mat = len(mats)
        mats.append(material("emitter", emittance=ke))
        lpts = _quad([(-h, ly, -h), (h, ly, -h), (h, ly, h), (-h, ly, h)], np.array([0.0, -1.0, 0.0]))
        faces.append((lpts, np.array([0.0, -1.0, 0.0]), light_mat))

    verts, norms, vidx, nidx, midx = [], [], [], [], []
    for corners, n, m in faces:
        base = len(verts)
        verts.extend(corners)
        ni = len(norms)
        norms.append(n / np.linalg.norm(n))
        for tri in ((0, 1, 2), (0, 2, 3)):
            vidx.append([base + tri[0], base + tri[1], base + tri[2]])
            nidx.append([ni, ni, ni])
            midx.append(m)
    V = np.zeros((len(verts), 4), np.float32)
    V[:, :3] = np.array(verts)
    V[:, 3] = 1.0
    N = np.zeros((len(norms), 4), np.float32)
    N[:, :3] = np.array(norms)
    T = len(vidx)
    meshes = [dict(tri_start=0, tri_count=T, to_global=IDENTITY, instance=-1, light_idx=-1)]
    area, point, spot, distant = [], [], [], []
    if light == "quad":
        area.append(dict(center=(-h, ly, -h), u=(2 * h, 0.0, 0.0), v=(0.0, 0.0, 2 * h), ke=ke, two_sided=0))
    elif light == "sphere":
        area.append(dict(type="sphere", center=(-0.2, 1.45, -0.2), u=(0.4, 0.0, 0.0), v=(0.0, 0.0, 0.4),
                         ke=(6.0, 4.5, 2.0)))
        meshes.append(dict(tri_start=0, tri_count=0, to_global=IDENTITY, instance=-1, light_idx=0))
    elif light == "disk":
        area.append(dict(type="disk", center=(-0.3, 1.9, -0.3), u=(0.6, 0.0, 0.0), v=(0.0, 0.0, 0.6),
                         ke=(12.0, 9.0, 4.0)))
        meshes.append(dict(tri_start=0, tri_count=0, to_global=IDENTITY, instance=-1, light_idx=0))
    elif light == "point":
        point.append(dict(position=(0.1, 1.75, 0.2), ke=(3.0, 2.4, 1.2)))
    elif light == "spot":
        spot.append(dict(position=(0.0, 1.9, 0.3), direction=(0.0, 1.0, 0.0), ke=(5.0, 4.0, 2.5),
                         cos_inner=float(np.cos(np.radians(20.0))), cos_outer=float(np.cos(np.radians(35.0)))))
    elif light == "distant":
        distant.append(dict(direction=(0.35, 1.0, 0.25), ke=(2.0, 1.8, 1.5)))
    else:
        raise ValueError(f"unknown room light {light!r}")
    return SceneData(
        vertices=V, normals=N, uvs=np.zeros((1, 2), np.float32),
        vindices=np.array(vidx, np.uint32), nindices=np.array(nidx, np.uint32),
        uvindices=np.zeros((T, 3), np.uint32), material_indices=np.array(midx, np.uint32),
        meshes=meshes, materials=mats, area_lights=area, point_lights=point, spot_lights=spot,
        distant_lights=distant, skydome_type=capi.NOOR_SKY_CONSTANT,
        camera=dict(eye=(0.0, 1.0, 3.75), look_at=(0.0, 1.0, 0.0), up=(0.0, 1.0, 0.0), fov_deg=40.0,
                    w=width, h=height),
        render=dict(spp=spp, bounces=bounces, rr=rr, mis=int(mis)), name="room")


def _image_maps(seed: int):
    """the textured room's image maps (H, W, 4) f32: a noisy two-tone checker
    (64 x 64), a roughness map in R and G (32 x 32), a height field of
    grooves and bumps (64 x 64, in R) and an alpha map of round holes
    (32 x 32: 0 inside a hole, 1 elsewhere)"""
    rng = np.random.default_rng(seed)
    img = []
    y, x = np.mgrid[0:64, 0:64]
    chk = ((x // 8 + y // 8) % 2).astype(np.float32)[..., None]
    a, b = np.array([0.75, 0.62, 0.45], np.float32), np.array([0.18, 0.25, 0.35], np.float32)
    rgb = chk * a + (1 - chk) * b + 0.04 * rng.standard_normal((64, 64, 3)).astype(np.float32)
    img.append(np.concatenate([np.clip(rgb, 0.02, 0.98), np.ones((64, 64, 1), np.float32)], 2))
    r = 0.05 + 0.25 * rng.random((32, 32)).astype(np.float32)
    img.append(np.stack([r, r * 0.8, np.zeros_like(r), np.ones_like(r)], 2).astype(np.float32))
    hgt = 0.5 + 0.3 * np.sin(x / 64 * 2 * np.pi * 4) + 0.2 * rng.standard_normal((64, 64))
    img.append(np.stack([hgt, hgt, hgt, np.ones_like(hgt)], 2).astype(np.float32))
    yy, xx = np.mgrid[0:32, 0:32]
    holes = (((xx % 16) - 7.5) ** 2 + ((yy % 16) - 7.5) ** 2) < 5.5 ** 2
    alpha = np.where(holes, 0.0, 1.0).astype(np.float32)
    img.append(np.stack([alpha, alpha, alpha, np.ones_like(alpha)], 2).astype(np.float32))
    return img


def textured_room_scene(seed: int = 6, width: int = 128, height: int = 128, spp: int = 16, bounces: int = 5,
                        rr: int = 1, textured_light: bool = False) -> SceneData:
    """The room with texture coordinates on every face (0..1 over each quad)
    and image maps: a checker on the floor (map_Kd, uv scale 4), a rough
    gold short box whose roughness is a map (uv scale 1), a bump-mapped tall
    box (map_bump, factor 0.02, uv scale 2) and, in front of the right
    wall, an alpha-cut panel (map_d with round holes, uv scale 3).  Camera
    rays that reflect off the gold box reach the bumped box with
    differentials.  `textured_light`: the ceiling light's emittance is the
    checker map too (an emitter's texture is read at its barycentrics)."""
    base = room_scene(seed=seed, width=width, height=height, spp=spp, bounces=bounces, rr=rr)
    mats = [dict(m) for m in base.materials]
    floor, short_box, tall_box = 0, 5, 5
    faces_per_quad = 2
    # materials: floor checker; the boxes get their own materials
    unit = [(1.0, 1.0)] * 7
    def maps(**kw):
        m = [-1] * 7
        for k, v in kw.items():
            m[getattr(capi, "NOOR_MAP_" + k.upper())] = v
        return m
    mats[floor] = dict(mats[floor], map=maps(diffuse=0), map_uvscale=[(4.0, 4.0)] + unit[1:])
    gold = material("metal", roughness=0.1)
    gold.update(map=maps(roughness=1), map_uvscale=unit)
    bumped = material("diffuse", albedo=(0.65, 0.6, 0.55))
    bumped.update(map=maps(bump=2), map_uvscale=[(2.0, 2.0)] * 7, bumpfactor=0.02)
    panel = material("diffuse", albedo=(0.3, 0.55, 0.35))
    panel.update(map=maps(alpha=3), map_uvscale=[(3.0, 3.0)] * 7)
    light_mat = len(mats) - 1
    light = dict(mats[light_mat])
    if textured_light:
        light.update(map=maps(emittance=0), map_uvscale=unit, emitter_scale=20.0)
    mats = mats[:5] + [gold, bumped, light, panel]
    # triangles: 10 wall, 12 short box, 12 tall box, 2 light (as in room_scene)
    midx = base.material_indices.astype(np.int64).copy()
    midx[10:22] = 5
    midx[22:34] = 6
    midx[34:36] = 7
    # the alpha-cut panel: a quad facing the camera in front of the right wall
    V = base.vertices.copy()
    pts = _quad([(0.55, 0.0, -0.75), (0.95, 0.0, -0.2), (0.95, 1.5, -0.2), (0.55, 1.5, -0.75)],
                np.array([-0.8, 0.0, 0.6]))
    pv = np.zeros((4, 4), np.float32)
    pv[:, :3] = np.array(pts)
    pv[:, 3] = 1.0
    V = np.concatenate([V, pv])
    n = np.cross(pts[1] - pts[0], pts[2] - pts[0])
    N = np.concatenate([base.normals, np.array([[*(n / np.linalg.norm(n)), 0.0]], np.float32)])
    b0 = base.vertices.shape[0]
    vidx = np.concatenate([base.vindices, np.array([[b0, b0 + 1, b0 + 2], [b0, b0 + 2, b0 + 3]], np.uint32)])
    nidx = np.concatenate([base.nindices, np.full((2, 3), N.shape[0] - 1, np.uint32)])
    midx = np.concatenate([midx, [8, 8]]).astype(np.uint32)
    # texture coordinates: the 4 corners of every quad at (0,0) (1,0) (1,1) (0,1)
    uvs = np.array([(0.0, 0.0), (1.0, 0.0), (1.0, 1.0), (0.0, 1.0)], np.float32)
    T = vidx.shape[0]
    uvidx = np.zeros((T, 3), np.uint32)
    uvidx[0::2] = [0, 1, 2]
    uvidx[1::2] = [0, 2, 3]
    meshes = [dict(base.meshes[0], tri_count=T)]
    return SceneData(vertices=V, normals=N, uvs=uvs, vindices=vidx, nindices=nidx, uvindices=uvidx,
                     material_indices=midx, meshes=meshes, materials=mats, area_lights=base.area_lights,
                     skydome_type=base.skydome_type, images=_image_maps(seed), camera=base.camera,
                     render=base.render, name="textured_room")


# ------------------------------------------------------------- icospheres
_ICO_CACHE: dict = {}


def icosphere(level: int):
    """unit icosphere: (V,3) float64 vertices, (F,3) int faces wound outward"""
    if level in _ICO_CACHE:
        return _ICO_CACHE[level]
    t = (1.0 + 5.0 ** 0.5) / 2.0
    V = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
                  (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
                  (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
                  (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)], np.int64)
    for _ in range(level):
        e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
        es = np.sort(e, axis=1)
        uniq, inv = np.unique(es, axis=0, return_inverse=True)
        mid = V[uniq[:, 0]] + V[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = V.shape[0]
        V = np.concatenate([V, mid])
        m = inv.reshape(3, -1).T + base
        a, b, c = F[:, 0], F[:, 1], F[:, 2]
        ab, bc, ca = m[:, 0], m[:, 1], m[:, 2]
        F = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                            np.stack([ab, bc, ca], 1)])
    n = np.cross(V[F[:, 1]] - V[F[:, 0]], V[F[:, 2]] - V[F[:, 0]])
    flip = np.einsum("ij,ij->i", n, V[F].mean(axis=1)) < 0
    F[flip] = F[flip][:, [0, 2, 1]]
    _ICO_CACHE[level] = (V, F)
    return V, F


def sphere_field(seed: int, count: int, level: int, box: float = 20.0, rmin: float = 0.1, rmax: float = 1.0,
                 kinds=("diffuse", "metal", "glass"), jitter: float = 0.002):
    """`count` icospheres: radius log-U[rmin,rmax], centre U in a box^3 cube,
    vertices jittered by N(0, jitter*r), one material per object drawn from
    `kinds` (Lambert albedo U[0.1,0.9]^3, gold conductor alpha U[0.05,0.5],
    dielectric IOR 1.5).  Returns the loader arrays."""
    rng = np.random.default_rng(seed)
    Vu, F = icosphere(level)
    nv, nf = Vu.shape[0], F.shape[0]
    radii = np.exp(rng.uniform(np.log(rmin), np.log(rmax), count))
    centers = rng.uniform(-box / 2, box / 2, (count, 3))
    V = np.zeros((count * nv, 4), np.float32)
    N = np.zeros((count * nv, 4), np.float32)
    vidx = np.zeros((count * nf, 3), np.uint32)
    midx = np.zeros(count * nf, np.uint32)
    meshes, mats = [], []
    for i in range(count):
        p = centers[i] + radii[i] * Vu + rng.normal(0.0, jitter * radii[i], Vu.shape)
        V[i * nv:(i + 1) * nv, :3] = p
        V[i * nv:(i + 1) * nv, 3] = 1.0
        N[i * nv:(i + 1) * nv, :3] = Vu
        vidx[i * nf:(i + 1) * nf] = F + i * nv
        midx[i * nf:(i + 1) * nf] = i
        kind = kinds[int(rng.integers(0, len(kinds)))]
        if kind == "diffuse":
            mats.append(material("diffuse", albedo=tuple(rng.uniform(0.1, 0.9, 3))))
        elif kind == "metal":
            alpha = rng.uniform(0.05, 0.5)
            mats.append(material("metal", roughness=float(np.sqrt(alpha))))
        else:
            mats.append(material("glass", ior=1.5))
        meshes.append(dict(tri_start=i * nf, tri_count=nf, to_global=IDENTITY, instance=-1, light_idx=-1))
    T = count * nf
    return dict(vertices=V, normals=N, uvs=np.zeros((1, 2), np.float32), vindices=vidx, nindices=vidx.copy(),
                uvindices=np.zeros((T, 3), np.uint32), material_indices=midx, meshes=meshes, materials=mats), \
        (centers, radii)


SKY_CAMERA = dict(eye=(0.0, 2.0, 16.0), look_at=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0), fov_deg=50.0)


def frame_spheres(centers: np.ndarray, radii: np.ndarray, seed: int, fov_deg: float = 50.0, aspect: float = 16 / 9,
                  candidates: int = 256, clearance: float = 1.0) -> dict:
    """Camera framing a seeded sphere field (the configurations do not fix a
    camera): among seeded eye positions inside the field's box and look
    directions, pick the view whose frustum holds the largest summed solid
    angle of spheres, keeping every sphere surface at least `clearance` away
    from the eye.  Deterministic in `seed`."""
    rng = np.random.default_rng(seed + 1000)
    lo, hi = centers.min(0), centers.max(0)
    eyes = rng.uniform(lo, hi, (candidates, 3))
    k = np.arange(candidates) + 0.5
    phi = np.arccos(1 - 2 * k / candidates)
    th = np.pi * (1 + 5 ** 0.5) * k
    dirs = np.stack([np.cos(th) * np.sin(phi), np.cos(phi), np.sin(th) * np.sin(phi)], 1)
    half_v = np.radians(fov_deg) / 2
    half_d = np.arctan(np.tan(half_v) * np.sqrt(1 + aspect * aspect))
    best, best_score = None, -1.0
    for e in eyes:
        v = centers - e
        dist = np.linalg.norm(v, axis=1)
        if (dist - radii).min() < clearance:
            continue
        ang = np.arcsin(np.clip(radii / dist, 0, 1))
        solid = 2 * np.pi * (1 - np.cos(ang))
        u = v / dist[:, None]
        cosang = u @ dirs.T                         # spheres x directions
        inside = np.arccos(np.clip(cosang, -1, 1)) < (half_v * 0.9)
        score = (inside * solid[:, None]).sum(0)
        j = int(np.argmax(score))
        if score[j] > best_score:
            best_score, best = float(score[j]), (e, dirs[j])
    e, d = best
    up = np.array([0.0, 1.0, 0.0]) if abs(d[1]) < 0.95 else np.array([1.0, 0.0, 0.0])
    return dict(eye=tuple(float(x) for x in e), look_at=tuple(float(x) for x in e + d), up=tuple(up),
                fov_deg=fov_deg)


def sky_scene(seed: int = 2, width: int = 1920, height: int = 1080, spp: int = 64, bounces: int = 8,
              count: int = 32, level: int = 6, rr: int = 1, mis: bool = False) -> SceneData:
    """C2: 32 subdivision-6 icospheres (2,621,440 triangles) under a
    Hosek-Wilkie sky (turbidity 3, sun elevation 30 deg, ground albedo 0.3)."""
    g, (c, r) = sphere_field(seed, count, level)
    cam = dict(frame_spheres(c, r, seed), w=width, h=height)
    return SceneData(**g, skydome_type=capi.NOOR_SKY_PHYSICAL, camera=cam,
                     render=dict(spp=spp, bounces=bounces, rr=rr, mis=int(mis)),
                     hosek=dict(turbidity=3.0, albedo=0.3, sun_lat=float(np.radians(60.0)),
                                sun_lon=float(np.pi / 4), solar_scale=250.0, solar_radius_scale=2.0),
                     name="sky")


def env_map(seed: int, width: int = 2048, height: int = 1024, mu: float = -1.0, sigma: float = 0.5,
            lobes: int = 3, peak: float = 1e4, lobe_sigma_deg=(1.0, 3.0)) -> np.ndarray:
    """equirectangular RGB map: log-normal background plus Gaussian lobes at
    seeded directions; texel (row j, col i) is the direction at
    theta = pi (j+0.5)/H, phi = 2 pi (i+0.5)/W, y up."""
    rng = np.random.default_rng(seed)
    img = np.exp(rng.normal(mu, sigma, (height, width, 3))).astype(np.float64)
    th = (np.arange(height) + 0.5) / height * np.pi
    ph = (np.arange(width) + 0.5) / width * 2 * np.pi
    st, ct = np.sin(th)[:, None], np.cos(th)[:, None]
    dirs = np.stack([st * np.cos(ph)[None, :], np.broadcast_to(ct, (height, width)), st * np.sin(ph)[None, :]], -1)
    for _ in range(lobes):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        s = np.radians(rng.uniform(*lobe_sigma_deg))
        ang = np.arccos(np.clip(dirs @ d, -1.0, 1.0))
        img += (peak * np.exp(-ang * ang / (2 * s * s)))[..., None]
    out = np.ones((height, width, 4), np.float32)
    out[..., :3] = img
    return out


def env_scene(seed: int = 3, width: int = 1920, height: int = 1080, spp: int = 128, bounces: int = 8,
              count: int = 32, level: int = 6, env_w: int = 2048, env_h: int = 1024, rr: int = 1) -> SceneData:
    """C3: the C2 geometry lit by a 2048x1024 log-normal + lobes map, MIS on."""
    g, (c, r) = sphere_field(2, count, level)
    cam = dict(frame_spheres(c, r, 2), w=width, h=height)
    return SceneData(**g, skydome_type=capi.NOOR_SKY_HDR, env=env_map(seed, env_w, env_h), camera=cam,
                     render=dict(spp=spp, bounces=bounces, rr=rr, mis=1), name="env")


def batched_workload(seed: int = 4, n_frames: int = 64, sides=(128, 256, 512, 1024), tri_range=(1e4, 2.6e6),
                     spp_range=(4, 64), bounces: int = 6):
    """C4: `n_frames` independent frames.  Per frame: square side uniform in
    `sides`; a triangle budget T log-uniform in `tri_range`, realised as
    ceil(T / 81,920) subdivision-6 icospheres of one seeded field (the first
    N spheres of it), or one icosphere at subdivision floor(log4(T / 20))
    when T < 81,920; spp uniform in spp_range (inclusive); sky or env-map
    lighting by a coin flip.  Frames whose geometry and lighting coincide
    share one scene.  Returns (scenes: dict key -> SceneData, frames: list of
    dict(key, camera, spp, bounces))."""
    rng = np.random.default_rng(seed)
    field, (c_all, r_all) = sphere_field(seed, 32, 6)
    nf6 = 20 * 4 ** 6
    scenes_: dict = {}
    frames = []
    env = None
    for _ in range(n_frames):
        side = int(rng.choice(sides))
        T = float(np.exp(rng.uniform(np.log(tri_range[0]), np.log(tri_range[1]))))
        spp = int(rng.integers(spp_range[0], spp_range[1] + 1))
        light = "sky" if rng.random() < 0.5 else "env"
        if T >= nf6:
            geo = ("field", int(min(32, np.ceil(T / nf6))))
        else:
            geo = ("single", int(max(0, np.floor(np.log(T / 20.0) / np.log(4.0)))))
        key = (geo, light)
        if key not in scenes_:
            if geo[0] == "field":
                n = geo[1]
                nv = field["vertices"].shape[0] // 32
                g = dict(vertices=field["vertices"][: n * nv], normals=field["normals"][: n * nv],
                         uvs=field["uvs"], vindices=field["vindices"][: n * nf6],
                         nindices=field["nindices"][: n * nf6], uvindices=field["uvindices"][: n * nf6],
                         material_indices=field["material_indices"][: n * nf6], meshes=field["meshes"][:n],
                         materials=field["materials"][:n])
                cam = frame_spheres(c_all[:n], r_all[:n], seed, aspect=1.0, clearance=0.5)
            else:
                g, (c1, r1) = sphere_field(seed + 100 + geo[1], 1, geo[1], rmin=1.0, rmax=1.0)
                ctr = c1[0]
                cam = dict(eye=tuple(float(x) for x in ctr + np.array([0.0, 1.0, 3.0])),
                           look_at=tuple(float(x) for x in ctr), up=(0.0, 1.0, 0.0), fov_deg=50.0)
            cam = dict(cam, w=side, h=side)  # the first frame's size (frames set their own)
            if light == "sky":
                sd = SceneData(**g, skydome_type=capi.NOOR_SKY_PHYSICAL, camera=cam,
                               render=dict(spp=spp, bounces=bounces, rr=1, mis=0),
                               hosek=dict(turbidity=3.0, albedo=0.3, sun_lat=float(np.radians(60.0)),
                                          sun_lon=float(np.pi / 4), solar_scale=250.0, solar_radius_scale=2.0),
                               name=f"{geo[0]}{geo[1]}-sky")
            else:
                if env is None:
                    env = env_map(seed, 2048, 1024)
                sd = SceneData(**g, skydome_type=capi.NOOR_SKY_HDR, env=env, camera=cam,
                               render=dict(spp=spp, bounces=bounces, rr=1, mis=1), name=f"{geo[0]}{geo[1]}-env")
            scenes_[key] = sd
        frames.append(dict(key=key, camera=dict(scenes_[key].camera, w=side, h=side), spp=spp, bounces=bounces))
    return scenes_, frames


def adjoint_scene(seed: int = 5, width: int = 512, height: int = 512, spp: int = 16, bounces: int = 4,
                  count: int = 10, level: int = 5, n_materials: int = 64, env_w: int = 512,
                  env_h: int = 256) -> SceneData:
    """C5: `count` subdivision-`level` icospheres (10 x 20,480 = 204,800
    triangles by default) with `n_materials` materials assigned per triangle
    as (sphere * 20 + base icosahedron face) mod n_materials: the first half
    Lambert (albedo U[0.1,0.9]^3), the second half GGX gold conductors
    (tint U[0.1,0.9]^3, alpha U[0.05,0.5]); lit by an env_w x env_h map
    (log-normal background plus three lobes of peak 20, below the radiance
    clamp); MIS on, Russian roulette off (rr = bounces)."""
    g, (c, r) = sphere_field(seed, count, level, box=6.0, rmin=0.5, rmax=1.5, kinds=("diffuse",))
    rng = np.random.default_rng(seed + 77)
    nf = 20 * 4 ** level
    tri = np.arange(count * nf)
    # subdivision keeps a face's children at indices congruent mod 20
    g["material_indices"] = (((tri // nf) * 20 + (tri % nf) % 20) % n_materials).astype(np.uint32)
    mats = []
    for i in range(n_materials):
        if i < n_materials // 2:
            mats.append(material("diffuse", albedo=tuple(rng.uniform(0.1, 0.9, 3))))
        else:
            mats.append(material("metal", roughness=float(np.sqrt(rng.uniform(0.05, 0.5))),
                                 specular=tuple(rng.uniform(0.1, 0.9, 3))))
    g["materials"] = mats
    cam = dict(frame_spheres(c, r, seed, aspect=width / height, clearance=0.5), w=width, h=height)
    return SceneData(**g, skydome_type=capi.NOOR_SKY_HDR, env=env_map(seed, env_w, env_h, peak=20.0), camera=cam,
                     render=dict(spp=spp, bounces=bounces, rr=bounces, mis=1), name="adjoint")


# ------------------------------------------------------------ C-ABI glue
def _ptr(a: np.ndarray, t=C.c_float):
    return a.ctypes.data_as(C.POINTER(t))


def scene_desc(scene: SceneData):
    """The noor_scene_desc of a scene (the loader output Model::load
    consumes) and the arrays it points into, which the caller keeps alive
    while the description is in use.  Builds nothing and needs no library."""
    s = scene
    keep = []
    V = np.ascontiguousarray(s.vertices, np.float32)
    N = np.ascontiguousarray(s.normals, np.float32)
    U = np.ascontiguousarray(s.uvs, np.float32)
    vi = np.ascontiguousarray(s.vindices, np.uint32)
    ni = np.ascontiguousarray(s.nindices, np.uint32)
    ui = np.ascontiguousarray(s.uvindices, np.uint32)
    mi = np.ascontiguousarray(s.material_indices, np.uint32)
    keep += [V, N, U, vi, ni, ui, mi]
    meshes = (capi.Mesh * len(s.meshes))()
    for k, m in enumerate(s.meshes):
        meshes[k].tri_start = m["tri_start"]
        meshes[k].tri_count = m["tri_count"]
        meshes[k].to_global[:] = [float(x) for x in np.asarray(m["to_global"], np.float32)]
        meshes[k].instance = m.get("instance", -1)
        meshes[k].light_idx = m.get("light_idx", -1)
    mats = (capi.MaterialDesc * len(s.materials))()
    map_defaults = dict(map=[-1] * 7, map_uvscale=[(1.0, 1.0)] * 7, bumpfactor=1.0)
    for k, m in enumerate(s.materials):
        for f, _ in capi.MaterialDesc._fields_:
            val = m.get(f, map_defaults.get(f))
            if f == "map":
                mats[k].map[:] = [int(x) for x in val]
            elif f == "map_uvscale":
                for j, uv in enumerate(val):
                    mats[k].map_uvscale[j][:] = [float(x) for x in uv]
            elif isinstance(val, (tuple, list, np.ndarray)):
                getattr(mats[k], f)[:] = [float(x) for x in val]
            else:
                setattr(mats[k], f, val)
    lights = (capi.AreaLight * max(1, len(s.area_lights)))()
    for k, l in enumerate(s.area_lights):
        lights[k] = make_area_light(l, k)
    delta = make_delta_lights(s)
    d = capi.SceneDesc()
    d.vertices, d.num_vertices = _ptr(V), V.shape[0]
    d.normals, d.num_normals = _ptr(N), N.shape[0]
    d.uvs, d.num_uvs = _ptr(U), U.shape[0]
    d.vindices, d.nindices, d.uvindices = _ptr(vi, C.c_uint32), _ptr(ni, C.c_uint32), _ptr(ui, C.c_uint32)
    d.material_indices = _ptr(mi, C.c_uint32)
    d.num_triangles = vi.shape[0]
    d.meshes, d.num_meshes = meshes, len(s.meshes)
    d.materials, d.num_materials = mats, len(s.materials)
    d.area_lights, d.num_area_lights = lights, len(s.area_lights)
    d.point_lights, d.num_point_lights = delta[0], len(s.point_lights)
    d.spot_lights, d.num_spot_lights = delta[1], len(s.spot_lights)
    d.distant_lights, d.num_distant_lights = delta[2], len(s.distant_lights)
    d.skydome_type = s.skydome_type
    if s.env is not None:
        E = np.ascontiguousarray(s.env, np.float32)
        keep.append(E)
        d.env_width, d.env_height, d.env_rgba = E.shape[1], E.shape[0], _ptr(E)
    b = s.bvh
    d.bvh = capi.BvhSpec(b["num_bins"], b["max_height"], b["Ci"], b["Ct"], b["min_leaf_tris"], b["max_leaf_tris"])
    imgs = (capi.Image * max(1, len(s.images)))()
    for k, im in enumerate(s.images):
        a = np.ascontiguousarray(im, np.float32)
        keep.append(a)
        imgs[k].width, imgs[k].height, imgs[k].rgba = a.shape[1], a.shape[0], _ptr(a)
    d.images, d.num_images = imgs, len(s.images)
    return d, keep + [meshes, mats, lights, delta, imgs]


class BuiltPayload:
    """Owns a noor_payload_handle (host arrays the library built); `gpu`
    builds the bottom-level trees on the current CUDA device (the same
    bytes)."""

    def __init__(self, scene: SceneData, gpu: bool = False):
        self.scene = scene
        self.desc, self._keep = scene_desc(scene)
        h = C.c_void_p()
        self.stat = capi.BuildStat()
        capi.call("noor_build_payload_gpu" if gpu else "noor_build_payload", C.byref(self.desc), C.byref(h),
                  C.byref(self.stat))
        self.handle = h
        self.payload = capi.Payload()
        capi.call("noor_payload_view", h, C.byref(self.payload))

    def triangle_order(self) -> np.ndarray:
        out = np.zeros(self.payload.num_triangles, np.uint32)
        capi.call("noor_payload_triangle_order", self.handle, _ptr(out, C.c_uint32), out.size)
        return out

    def nodes(self) -> np.ndarray:
        """(n, 8) uint32: min_right_start then max_axis_count words"""
        n = self.payload.num_bvh_nodes
        lo = np.ctypeslib.as_array(self.payload.bvh_min_right_start, (n, 4))
        hi = np.ctypeslib.as_array(self.payload.bvh_max_axis_count, (n, 4))
        return np.concatenate([lo, hi], axis=1).copy()

    def array(self, name: str, cols: int, dtype=np.uint32) -> np.ndarray:
        n = self.payload.num_triangles
        return np.ctypeslib.as_array(getattr(self.payload, name), (n, cols)).copy()

    def default_spec(self, bounces: int, rr: int) -> capi.Spec:
        sp = capi.Spec()
        capi.call("noor_payload_default_spec", self.handle, bounces, rr, C.byref(sp))
        return sp

    def free(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            capi.lib().noor_free_payload(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def make_area_light(l: dict, idx: int) -> capi.AreaLight:
    """CudaShape(center, u, v, n, type) + CudaAreaLight (shape.cuh:43-69):
    `center` is the corner the edges u and v start from; a sphere or disk is
    centred at center + (u + v) / 2 with radius min(|u|, |v|) / 2.  `type`:
    "quad" (default), "sphere" or "disk"."""
    a = capi.AreaLight()
    kind = {"quad": capi.NOOR_SHAPE_QUAD, "sphere": capi.NOOR_SHAPE_SPHERE,
            "disk": capi.NOOR_SHAPE_DISK}[l.get("type", "quad")]
    c, u, v = (np.asarray(l[k], np.float32) for k in ("center", "u", "v"))
    n = np.cross(u.astype(np.float64), v.astype(np.float64))
    n = (n / np.linalg.norm(n)).astype(np.float32)
    r = np.float32(0.5) * min(np.float32(np.linalg.norm(u)), np.float32(np.linalg.norm(v)))
    r2 = np.float32(r * r)
    if kind == capi.NOOR_SHAPE_QUAD:
        area = float(np.linalg.norm(np.cross(u.astype(np.float64), v.astype(np.float64))))
    else:
        c = (c + np.float32(0.5) * (u + v)).astype(np.float32)
        area = float(np.float32(4.0 * np.pi if kind == capi.NOOR_SHAPE_SPHERE else np.pi) * r2)
    a.shape.center[:] = [float(x) for x in c]
    a.shape.u[:] = [float(x) for x in u]
    a.shape.v[:] = [float(x) for x in v]
    a.shape.n[:] = [float(x) for x in n]
    a.shape.area = area
    a.shape.radius = float(r)
    a.shape.radius2 = float(r2)
    a.shape.light_idx = idx
    a.shape.type = kind
    a.ke[:] = [float(x) for x in l["ke"]]
    a.two_sided = int(l.get("two_sided", 0))
    return a


def make_delta_lights(s: "SceneData"):
    """noor_point_light / noor_spot_light / noor_distant_light arrays (one
    element at least, so that each is a valid pointer)"""
    pts = (capi.PointLight * max(1, len(s.point_lights)))()
    for k, l in enumerate(s.point_lights):
        pts[k].ke[:] = [float(x) for x in l["ke"]]
        pts[k].position[:] = [float(x) for x in l["position"]]
    spots = (capi.SpotLight * max(1, len(s.spot_lights)))()
    for k, l in enumerate(s.spot_lights):
        spots[k].ke[:] = [float(x) for x in l["ke"]]
        spots[k].position[:] = [float(x) for x in l["position"]]
        spots[k].direction[:] = [float(x) for x in l["direction"]]
        spots[k].cos_inner = float(l["cos_inner"])
        spots[k].cos_outer = float(l["cos_outer"])
    dist = (capi.DistantLight * max(1, len(s.distant_lights)))()
    for k, l in enumerate(s.distant_lights):
        dist[k].ke[:] = [float(x) for x in l["ke"]]
        dist[k].direction[:] = [float(x) for x in l["direction"]]
    return pts, spots, dist


def make_camera(cam: dict) -> capi.Camera:
    """noor_camera_lookat's pinhole camera, or with `type` "ortho" (the
    raster mapped onto a `ortho_scale`-wide window of the z = 0 plane, rays
    along -z), "env" (360 x 180 degrees) or `lens_radius` / `focal_length`
    (thin lens) set."""
    out = capi.Camera()
    arr = lambda v: (C.c_float * 3)(*[float(x) for x in v])
    capi.call("noor_camera_lookat", arr(cam["eye"]), arr(cam["look_at"]), arr(cam["up"]),
              float(np.radians(cam["fov_deg"])), int(cam["w"]), int(cam["h"]), C.byref(out))
    kind = cam.get("type", "persp")
    if kind == "ortho":
        out.type = capi.NOOR_CAMERA_ORTHO
        w, h, half = float(cam["w"]), float(cam["h"]), 0.5 * float(cam.get("ortho_scale", 2.0))
        rows = [[2 * half / w, 0.0, 0.0, -half], [0.0, -2 * half / w, 0.0, half * h / w], [0.0, 0.0, 0.0, 0.0]]
        for r in range(3):
            out.raster_to_camera[r][:] = [float(x) for x in rows[r]]
    elif kind == "env":
        out.type = capi.NOOR_CAMERA_ENV
    out.lens_radius = float(cam.get("lens_radius", 0.0))
    out.focal_length = float(cam.get("focal_length", out.focal_length))
    return out


def hosek_dataset() -> np.ndarray:
    """RGB coefficient and radiance tables of the Hosek-Wilkie model
    (3 x 1080 + 3 x 120 floats), the package's data file."""
    if not HOSEK_DATASET.exists():
        raise FileNotFoundError(f"{HOSEK_DATASET} missing (generate with noor_b200/data/make_hosek_data.py)")
    return np.load(HOSEK_DATASET).astype(np.float32)


def make_hosek(h: Optional[dict]) -> capi.HosekSky:
    out = capi.HosekSky()
    if h is None:
        return out
    ds = np.ascontiguousarray(hosek_dataset())
    alb = (C.c_float * 3)(h["albedo"], h["albedo"], h["albedo"])
    capi.call("noor_hosek_fit", _ptr(ds), float(h["turbidity"]), alb, float(h["sun_lat"]), float(h["sun_lon"]),
              float(h["solar_scale"]), float(h["solar_radius_scale"]), C.byref(out))
    return out


class Renderer:
    """The reference-facing render context: load_cuda_data on a built
    payload, then cuda_path_tracer / noor_render_frames and film readback.
    Keeps the camera, spec and sky structs alive for update_cuda_*.
    The C-ABI keeps one current context per thread, so only the most recently
    created Renderer of a thread is usable; older ones raise."""

    _current = None

    def __init__(self, scene: SceneData, built: Optional[BuiltPayload] = None, intersector: int = 0,
                 film_mode: int = 0, hosek: Optional[capi.HosekSky] = None):
        self.scene = scene
        self.built = built or BuiltPayload(scene)
        r = scene.render
        self.spec = self.built.default_spec(r.get("bounces", 5), r.get("rr", 1))
        self.spec.mis = int(r.get("mis", 0))
        self.spec.intersector = intersector
        self.spec.film_mode = film_mode
        self.camera = make_camera(scene.camera)
        self.hosek = hosek if hosek is not None else make_hosek(scene.hosek)
        capi.call("load_cuda_data", C.byref(self.built.payload), C.byref(self.hosek), C.byref(self.camera),
                  C.byref(self.spec), None)
        Renderer._current = self
        self.frame = C.c_uint(1)
        self.w, self.h = int(scene.camera["w"]), int(scene.camera["h"])

    def _check(self):
        if Renderer._current is not self:
            raise RuntimeError("this Renderer's context was replaced by a newer one on this thread")

    def render(self, n_frames: int) -> None:
        self._check()
        capi.call("noor_render_frames", C.byref(self.frame), n_frames)

    def path_tracer(self) -> None:
        self._check()
        capi.call("cuda_path_tracer", C.byref(self.frame))

    def framebuffer(self) -> np.ndarray:
        self._check()
        out = np.zeros((self.h, self.w, 4), np.float32)
        capi.call("noor_get_framebuffer", _ptr(out), self.w * self.h)
        return out

    def counters(self, reset: bool = False):
        c = (C.c_uint64 * 3)()
        capi.call("noor_ray_counters", c, int(reset))
        return tuple(int(x) for x in c)

    def status(self, reset: bool = False) -> int:
        s = C.c_uint32()
        capi.call("noor_device_status", C.byref(s), int(reset))
        return s.value

    def update_spec(self, **kw):
        self._check()
        for k, v in kw.items():
            setattr(self.spec, k, v)
        capi.call("update_cuda_spec")
        self.frame = C.c_uint(1)

    def close(self):
        if Renderer._current is self:
            capi.call("device_free_memory")
            Renderer._current = None


# ------------------------------------------------------- batched frames
def upload_scene(scene: SceneData, built: Optional[BuiltPayload] = None, intersector: int = 0):
    """Adds a scene to the current context (noor_scene_upload); returns
    (scene_id, keep-alive tuple)."""
    built = built or BuiltPayload(scene)
    r = scene.render
    spec = built.default_spec(r.get("bounces", 5), r.get("rr", 1))
    spec.mis = int(r.get("mis", 0))
    spec.intersector = intersector
    hosek = make_hosek(scene.hosek)
    sid = C.c_uint32()
    capi.call("noor_scene_upload", C.byref(built.payload), C.byref(hosek), C.byref(spec), C.byref(sid))
    return sid.value, (built, spec, hosek)


def wf_frame(scene_id: int, cam: dict, spp: int, bounces: int = 0, first_frame: int = 1, d_film: int = 0):
    f = capi.WfFrame()
    f.scene_id = scene_id
    f.width, f.height = int(cam["w"]), int(cam["h"])
    f.spp = spp
    f.first_frame = first_frame
    f.bounces = bounces
    f.camera = make_camera(cam)
    f.d_film = C.cast(C.c_void_p(d_film), capi.pf) if d_film else capi.pf()
    return f


def wf_params(block: int = 128, capacity: int = 1 << 20, sort: int = 1, graph: int = 1,
              max_iterations: int = 0, traversal: int = 0, shade_regs: int = 0) -> capi.WfParams:
    return capi.WfParams(block, capacity, sort, graph, max_iterations, traversal, shade_regs)
