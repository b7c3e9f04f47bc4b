"""The reference arm's payload, camera and sky against the product's.

oracle.RefPayload assembles a payload around the reference's own BVH builder
and WaldTriangle (oracle/_ref/libnoor_ref.so); the bench's reference arm
renders from it with the oracle, never loading libnoor_b200.so.  These tests
hold that payload to noor_build_payload byte for byte (tree, transforms,
de-duplicated vertices, Wald records, attribute words, textures, materials,
lights, spec), the oracle's camera to noor_camera_lookat, and check that
the arm runs without the product library in the process.
"""
import ctypes as C
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from noor_b200 import _capi, scenes
from oracle import oracle as O

import refdev_probe as probe

ROOT = Path(__file__).resolve().parents[1]

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref/libnoor_ref.so not built")


def _arr(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dtype))), (n,)).copy()


def payload_arrays(p) -> dict:
    nt, nv, ni, nn = p.num_triangles, p.num_vertices, p.num_instances, p.num_bvh_nodes
    out = dict(attr=_arr(p.attribute_indices, 4 * nt, np.uint32), vtx=_arr(p.vertices, 4 * nv, np.uint32),
               nrm=_arr(p.normals, 4 * nv, np.uint32), uv=_arr(p.uvs, 2 * nv, np.uint32),
               lo=_arr(p.bvh_min_right_start, 4 * nn, np.uint32), hi=_arr(p.bvh_max_axis_count, 4 * nn, np.uint32),
               root=np.array([p.bvh_root_node]))
    for k, name in enumerate(("normal_row", "world_to_object_row", "object_to_world_row")):
        for r in range(3):
            out[f"{name}{r}"] = _arr(getattr(p, name)[r], 4 * ni, np.uint32)
    for k, name in enumerate(("wald_ax_nu_nv_nd", "wald_bnu_bnv_au_av", "wald_cnu_cnv_deg_mat")):
        out[name] = _arr(getattr(p, name), 4 * nt, np.uint32)
    out["materials"] = np.frombuffer(C.string_at(p.materials, p.num_materials * C.sizeof(_capi.Material)), np.uint8)
    tex = []
    for i in range(p.num_textures):
        t = p.textures[i]
        tex.append(np.array([t.width, t.height], np.int64))
        tex.append(_arr(t.rgba, 4 * t.width * t.height, np.uint32))
    out["textures"] = np.concatenate(tex)
    for name, cls in (("area_lights", _capi.AreaLight), ("point_lights", _capi.PointLight),
                      ("spot_lights", _capi.SpotLight), ("distant_lights", _capi.DistantLight)):
        n = getattr(p, "num_" + name)
        out[name] = np.frombuffer(C.string_at(getattr(p, name), n * C.sizeof(cls)), np.uint8) if n else np.zeros(0)
    out["counts"] = np.array([p.num_infinite_lights, p.num_textures, p.num_materials])
    return out


def instanced_scene():
    g = scenes.sphere_field(3, 2, 2)[0]
    T = np.eye(4, dtype=np.float32)
    T[:3, :3] = np.array([[0.8, -0.6, 0.0], [0.6, 0.8, 0.0], [0.0, 0.0, 1.5]], np.float32)
    T[:3, 3] = (5, 0.25, -1)
    g["meshes"].append(dict(tri_start=0, tri_count=0, to_global=T.reshape(-1, order="F"), instance=1, light_idx=-1))
    return scenes.SceneData(**g, name="inst")


SCENES = {
    "room": lambda: probe.trace_scenes()["room"],
    "field16": lambda: probe.trace_scenes()["field16"],
    "sky_small": lambda: scenes.sky_scene(width=64, height=36, count=4, level=3),
    "env_small": lambda: scenes.env_scene(width=64, height=36, count=3, level=3),
    "room_scene": lambda: scenes.room_scene(),
    "instanced": instanced_scene,
    "textured_room": lambda: scenes.textured_room_scene(),
}


@pytest.mark.parametrize("name", list(SCENES))
def test_reference_payload_matches_product(name):
    s = SCENES[name]()
    b = scenes.BuiltPayload(s)
    r = O.RefPayload(s, _capi, scenes)
    got, want = payload_arrays(r.payload), payload_arrays(b.payload)
    assert got.keys() == want.keys()
    for k in want:
        if k.endswith("_row0") or k.endswith("_row1") or k.endswith("_row2"):
            # instance transforms: glm-style FP32 inverses in the reference
            # (its normal transform keeps signed zeros), FP64 rounded once in
            # the product: equal values to 2 ulp
            a, b_ = got[k].view(np.float32), want[k].view(np.float32)
            ulp = np.spacing(np.maximum(np.abs(a), np.abs(b_)).astype(np.float32))
            assert np.all(np.abs(a - b_) <= 2 * ulp), k
        else:
            assert np.array_equal(got[k], want[k]), k
    sr = bytes(r.default_spec(5, 1))
    sb = bytes(b.default_spec(5, 1))
    assert sr == sb
    r.free()
    b.free()


@pytest.mark.parametrize("name", ["room_scene", "sky", "env", "field16", "odd"])
def test_reference_camera_matches_product(name):
    if name == "sky":
        cam = scenes.sky_scene(width=1920, height=1080, count=2, level=1).camera
    elif name == "env":
        cam = scenes.env_scene(width=640, height=960, count=2, level=1).camera
    elif name == "field16":
        cam = probe.trace_scenes()["field16"].camera
    elif name == "odd":
        cam = dict(eye=(0.3, -2.0, 7.1), look_at=(1.0, 0.5, -0.25), up=(0.0, 0.0, 1.0), fov_deg=73.3, w=333, h=97)
    else:
        cam = scenes.room_scene().camera
    assert bytes(O.camera_lookat(_capi, cam)) == bytes(scenes.make_camera(cam))


@pytest.mark.gpu
def test_reference_hosek_matches_product_fit():
    """the reference arm's sky (the reference's own fit) against the
    product's FP64 fit of the same sky (a GPU routine)"""
    sys.path.insert(0, str(ROOT))
    import bench
    h = scenes.sky_scene(width=64, height=36, count=2, level=1).hosek
    ref = bench.reference_hosek(_capi, h)
    prod = scenes.make_hosek(h)
    def used(hk):
        """the fields the sky's radiance reads: state c's configs[c] and
        radiances[c], and the sun"""
        v = [x for c in range(3) for x in list(hk.state[c].configs[c]) + [hk.state[c].radiances[c]]]
        return np.array(v + list(hk.solar_dir) + list(hk.ground_albedo) + [hk.solar_scale, hk.solar_radius])
    assert np.allclose(used(ref), used(prod), rtol=2e-5, atol=1e-6)


def test_reference_arm_never_loads_the_product_library():
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'room', '--steps', '1', "
            "'--warmup', '0', '--scale', '0.25']; sys.path.insert(0, '.'); import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'product': 'libnoor_b200' in maps, 'ref': 'libnoor_ref' in maps}))")
    env = dict(os.environ, OMP_NUM_THREADS="4")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300,
                         env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(x) for x in out.stdout.strip().splitlines() if x.startswith("{")]
    line, maps = lines[0], lines[-1]
    assert line["impl"] == "reference" and line["value"] > 0, line
    assert maps == {"product": False, "ref": True}, maps
