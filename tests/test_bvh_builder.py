"""Host scene builder (noor_build_payload) against the reference's own BVH
builder and Wald precomputation: frozen golden fixtures, and the live
reference library when this machine has the reference tree."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from noor_b200 import scenes, _capi

GOLD = Path(__file__).resolve().parent / "golden"
import importlib.util as _u
_spec = _u.spec_from_file_location("make_golden", GOLD / "make_golden.py")
make_golden = _u.module_from_spec(_spec)
_spec.loader.exec_module(make_golden)


@pytest.mark.parametrize("name", sorted(make_golden.GOLDEN_SCENES))
def test_bvh_bytes_match_golden(name):
    g = np.load(GOLD / "bvh_golden.npz")
    s = make_golden.GOLDEN_SCENES[name]()
    b = scenes.BuiltPayload(s)
    assert np.array_equal(b.nodes(), g[f"{name}_nodes"])
    assert b.payload.bvh_root_node == int(g[f"{name}_meta"][0])
    assert b.stat.height == int(g[f"{name}_meta"][1])
    assert np.array_equal(b.triangle_order(), g[f"{name}_order"])


def _wald_words(v9):
    """noor_build_payload's Wald record of one triangle"""
    V = np.ones((3, 4), np.float32)
    V[:, :3] = v9.reshape(3, 3)
    s = scenes.SceneData(vertices=V, normals=np.tile(np.array([[0, 0, 1, 0]], np.float32), (3, 1)),
                         uvs=np.zeros((1, 2), np.float32), vindices=np.array([[0, 1, 2]], np.uint32),
                         nindices=np.array([[0, 1, 2]], np.uint32), uvindices=np.zeros((1, 3), np.uint32),
                         material_indices=np.zeros(1, np.uint32),
                         meshes=[dict(tri_start=0, tri_count=1, to_global=scenes.IDENTITY, instance=-1, light_idx=-1)],
                         materials=[scenes.material("diffuse")])
    b = scenes.BuiltPayload(s)
    return np.concatenate([b.array("wald_ax_nu_nv_nd", 4)[0], b.array("wald_bnu_bnv_au_av", 4)[0],
                           b.array("wald_cnu_cnv_deg_mat", 4)[0]])


def test_wald_records_match_golden():
    g = np.load(GOLD / "wald_golden.npz")
    for tri, ref in zip(g["tris"], g["recs"]):
        mine = _wald_words(tri)
        deg = ref[10] == 1
        assert mine[10] == ref[10]
        assert mine[0] == ref[0]            # axis
        if not deg:
            assert np.array_equal(mine[:10], ref[:10])


def test_degenerate_flag_is_set():
    g = np.load(GOLD / "wald_golden.npz")
    assert (g["recs"][:8, 10] == 1).all()


def test_payload_layout_invariants():
    s = scenes.room_scene()
    b = scenes.BuiltPayload(s)
    p = b.payload
    assert p.num_triangles == 36
    attr = b.array("attribute_indices", 4)
    assert attr[:, :3].max() < p.num_vertices
    assert (attr[:, 3] < p.num_materials).all()
    # every triangle index appears exactly once across the tri leaves
    nodes = b.nodes()
    seen = np.zeros(p.num_triangles, np.int32)
    for n in nodes:
        if n[7] & _capi.TRI_LEAF_MASK:
            c = n[7] & 0x7FFFFFFF
            seen[n[3]:n[3] + c] += 1
    assert (seen == 1).all()
    # material word of the Wald record carries the material type
    w2 = b.array("wald_cnu_cnv_deg_mat", 4)
    types = np.array([m["type"] for m in s.materials])
    assert np.array_equal(w2[:, 3], types[attr[:, 3]])


def test_default_spec_follows_scene_load():
    s = scenes.room_scene()
    b = scenes.BuiltPayload(s)
    sp = b.default_spec(5, 1)
    r = b.stat.scene_radius
    assert sp.world_radius == pytest.approx(r)
    assert sp.reflection_bias == pytest.approx(1e-4 * r)
    assert sp.bvh_root_node == b.payload.bvh_root_node
    assert sp.lighting_type & _capi.NOOR_LIGHT_SKY_MASK == 0   # 2 lights -> sky off
    g = scenes.SceneData(**scenes.sphere_field(1, 2, 1)[0], name="x")
    sp2 = scenes.BuiltPayload(g).default_spec(8, 1)
    assert sp2.lighting_type & _capi.NOOR_LIGHT_SKY_MASK      # infinite light only -> sky on


def test_builder_rejects_bad_input():
    s = scenes.room_scene()
    s.vindices = s.vindices.copy()
    s.vindices[3, 1] = 10_000
    with pytest.raises(_capi.NoorError):
        scenes.BuiltPayload(s)
    s = scenes.room_scene()
    s.vertices = s.vertices.copy()
    s.vertices[2, 0] = np.nan
    with pytest.raises(_capi.NoorError):
        scenes.BuiltPayload(s)


def test_instances_and_transforms():
    """an instance shares its source's bottom-level tree; the top level sees
    the transformed boxes"""
    g = scenes.sphere_field(3, 1, 2)[0]
    T = np.eye(4, dtype=np.float32)
    T[:3, 3] = (5, 0, 0)
    g["meshes"].append(dict(tri_start=0, tri_count=0, to_global=T.reshape(-1, order="F"), instance=0, light_idx=-1))
    s = scenes.SceneData(**g, name="inst")
    b = scenes.BuiltPayload(s)
    nodes = b.nodes()
    inst = [n for n in nodes if (n[7] & _capi.MESH_INSTANCE_MASK) and not (n[7] & _capi.TRI_LEAF_MASK)]
    assert len(inst) == 2
    assert inst[0][3] == inst[1][3] == 0          # both point at the one BLAS root
    lo = np.array([n[:3] for n in inst]).view(np.float32)
    assert abs((lo[1] - lo[0])[0] - 5.0) < 1e-4 or abs((lo[0] - lo[1])[0] - 5.0) < 1e-4


def test_live_reference_builder_if_available():
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("reference tree not compiled on this machine")
    for seed, count, level in [(21, 5, 3), (22, 3, 4)]:
        s = scenes.SceneData(**scenes.sphere_field(seed, count, level)[0], name="live")
        b = scenes.BuiltPayload(s)
        nodes, root, order, height = O.ref_build_bvh(b.desc, s.num_triangles)
        assert np.array_equal(b.nodes(), nodes)
        assert np.array_equal(b.triangle_order(), order)
        assert (root, height) == (b.payload.bvh_root_node, b.stat.height)


def test_light_mesh_must_carry_no_triangles():
    s = scenes.room_scene(seed=1, light="sphere")
    s.meshes[1]["tri_count"] = 2
    with pytest.raises(_capi.NoorError):
        scenes.BuiltPayload(s)


def test_light_node_points_at_its_empty_leaf():
    """a light mesh gets a one-leaf bottom-level tree (no triangles) before
    the top level, as the reference's builder makes it, and the light node
    points at it"""
    s = scenes.room_scene(seed=1, light="disk")
    b = scenes.BuiltPayload(s)
    nodes = b.nodes()
    light = [n for n in nodes if (n[7] & 0x08000000) and not (n[7] & _capi.TRI_LEAF_MASK)]
    assert len(light) == 1 and (light[0][7] & 0x07FFFFFF) == 0
    leaf = nodes[light[0][3]]
    assert leaf[7] == _capi.TRI_LEAF_MASK and np.array_equal(leaf[:3], light[0][:3])


def test_gpu_builder_fails_cleanly_without_a_device():
    """noor_build_payload_gpu reports an error instead of falling back when
    no CUDA device is there (this test only runs where there is none)"""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(_capi.NoorError):
        scenes.BuiltPayload(scenes.room_scene(), gpu=True)


@pytest.mark.parametrize("make", [lambda: scenes.room_scene(seed=1),
                                  lambda: scenes.SceneData(**scenes.sphere_field(5, 6, 4)[0], name="f")])
def test_vertex_deduplication_is_first_occurrence_in_bvh_order(make):
    """Model::loadCudaPayload numbering (model.cpp:376-401), restated with
    numpy: the corners in BVH order, each (vertex, normal, uv) triple
    numbered by its first occurrence; the payload's attribute indices and
    vertex arrays must be exactly that"""
    s = make()
    b = scenes.BuiltPayload(s)
    order = b.triangle_order()
    keys = np.stack([s.vindices[order].reshape(-1), s.nindices[order].reshape(-1),
                     s.uvindices[order].reshape(-1)], axis=1).astype(np.int64)
    packed = (keys[:, 0] << 42) | (keys[:, 1] << 21) | keys[:, 2]
    uniq, first, inverse = np.unique(packed, return_index=True, return_inverse=True)
    rank = np.empty(len(uniq), np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(len(uniq))
    element = rank[inverse]
    attr = b.array("attribute_indices", 4)
    assert np.array_equal(attr[:, :3].reshape(-1), element)
    p = b.payload
    verts = np.ctypeslib.as_array(p.vertices, (p.num_vertices, 4))
    src = keys[np.sort(first)]
    assert p.num_vertices == len(uniq)
    assert np.array_equal(verts, np.asarray(s.vertices, np.float32)[src[:, 0]])


def test_single_large_mesh_matches_live_reference():
    """one 327,680-triangle mesh: its top levels are split over host threads
    (subtrees appended in depth-first order); the bytes must still be the
    reference builder's"""
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("reference tree not compiled on this machine")
    s = scenes.SceneData(**scenes.sphere_field(41, 1, 7)[0], name="one")
    b = scenes.BuiltPayload(s)
    nodes, root, order, height = O.ref_build_bvh(b.desc, s.num_triangles)
    assert np.array_equal(b.nodes(), nodes)
    assert np.array_equal(b.triangle_order(), order)
    assert (root, height) == (b.payload.bvh_root_node, b.stat.height)


def test_hosek_data_file_is_the_reference_table():
    """the package's Hosek-Wilkie table (parsed from the model's data header
    by noor_b200/data/make_hosek_data.py) equals the table the reference's
    compiled model holds (tests/golden/hosek_rgb_dataset.npy)"""
    golden = np.load(Path(__file__).resolve().parent / "golden" / "hosek_rgb_dataset.npy")
    assert np.array_equal(scenes.hosek_dataset(), golden)
