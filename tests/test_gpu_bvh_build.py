"""GPU payload build (noor_build_payload_gpu: bottom-level BVH trees,
vertex de-duplication, Wald records) against the host builder
(noor_build_payload, itself byte-identical to the reference builder by the
golden fixtures): every payload array the same bytes, on scenes with light
nodes, instances, many meshes, forced height limits and every bin count,
and on the 2.6M-triangle sky scene."""
import numpy as np
import pytest

from noor_b200 import scenes

pytestmark = pytest.mark.gpu


def _arrays(b: scenes.BuiltPayload):
    p = b.payload
    out = {"nodes": b.nodes(), "order": b.triangle_order(), "attr": b.array("attribute_indices", 4),
           "wald0": b.array("wald_ax_nu_nv_nd", 4), "wald1": b.array("wald_bnu_bnv_au_av", 4),
           "wald2": b.array("wald_cnu_cnv_deg_mat", 4),
           "vertices": np.ctypeslib.as_array(p.vertices, (p.num_vertices, 4)).copy()}
    meta = (p.bvh_root_node, p.num_bvh_nodes, b.stat.height, b.stat.num_inner_nodes, b.stat.num_leaf_nodes,
            b.stat.max_leaf_tris)
    return out, meta


def _same(scene):
    host, gpu = scenes.BuiltPayload(scene), scenes.BuiltPayload(scene, gpu=True)
    a, ma = _arrays(host)
    g, mg = _arrays(gpu)
    assert ma == mg, (ma, mg)
    for k in a:
        assert a[k].shape == g[k].shape, k
        if not np.array_equal(a[k].view(np.uint32), g[k].view(np.uint32)):
            bad = np.argwhere(a[k].view(np.uint32) != g[k].view(np.uint32))
            raise AssertionError(f"{k}: {len(bad)} words differ, first {bad[:4].tolist()}")
    return host, gpu


def _field(seed, count, level, **bvh):
    s = scenes.SceneData(**scenes.sphere_field(seed, count, level)[0], name="f")
    s.bvh = dict(s.bvh, **bvh)
    return s


@pytest.mark.parametrize("light", ["quad", "sphere", "disk"])
def test_rooms(light):
    _same(scenes.room_scene(seed=1, light=light))


@pytest.mark.parametrize("seed,count,level", [(11, 6, 3), (21, 5, 3), (22, 3, 4), (7, 40, 2), (8, 2, 5)])
def test_sphere_fields(seed, count, level):
    _same(_field(seed, count, level))


@pytest.mark.parametrize("bvh", [dict(num_bins=2), dict(num_bins=8), dict(num_bins=32), dict(num_bins=64),
                                 dict(min_leaf_tris=1, max_leaf_tris=8), dict(max_height=6),
                                 dict(Ci=2.0, Ct=0.5)])
def test_bvh_parameters(bvh):
    _same(_field(31, 4, 4, **bvh))


def test_instances():
    g = scenes.sphere_field(3, 2, 4)[0]
    T = np.eye(4, dtype=np.float32)
    T[:3, 3] = (5, 0, 0)
    g["meshes"].append(dict(tri_start=0, tri_count=0, to_global=T.reshape(-1, order="F"), instance=0, light_idx=-1))
    _same(scenes.SceneData(**g, name="inst"))


def test_sky_scene_full_size():
    """32 subdivision-6 icospheres, 2,621,440 triangles: large tasks take the
    chunked path"""
    s = scenes.sky_scene()
    _same(s)
    # timed again, with the CUDA context up and the builder's memory pool warm
    host, gpu = scenes.BuiltPayload(s), scenes.BuiltPayload(s, gpu=True)
    for name, b in (("host", host), ("gpu", gpu)):
        st = b.stat
        print(f"{name}: {s.num_triangles} triangles, payload {st.build_seconds:.3f} s = boxes {st.box_seconds:.3f} s"
              f" + trees {st.tree_seconds:.3f} s (device {st.tree_device_ms:.1f} ms) + vertices and Wald records "
              f"{st.tail_seconds:.3f} s (device {st.tail_device_ms:.1f} ms) + the rest")
    assert gpu.stat.tree_device_ms > 0 and gpu.stat.tail_device_ms > 0
