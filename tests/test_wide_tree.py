"""The four-wide any-hit tree scene upload builds for shadow rays (host
collapse, no GPU): it exists for every scene the builder makes, halves the
binary tree's inner levels where boxes nest, bounds the traversal stack, and
is refused -- leaving the binary traversal -- for trees it does not suit.
Its answers are held to the binary traversal's on the GPU
(test_gpu_trace.py, test_gpu_refdev.py)."""
import ctypes as C

import numpy as np
import pytest

from noor_b200 import _capi, scenes

import refdev_probe as probe


def info(payload, root=None, full=False):
    nw, ne, sn, cl = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
    root = payload.bvh_root_node if root is None else root
    _capi.call("noor_wide_tree_info", C.byref(payload), root, C.byref(nw), C.byref(ne), C.byref(sn), C.byref(cl))
    if full:
        return nw.value, ne.value, sn.value, cl.value
    return nw.value, ne.value, sn.value


def inner_nodes(payload):
    hi = np.ctypeslib.as_array(C.cast(payload.bvh_max_axis_count, C.POINTER(C.c_uint32)),
                               (payload.num_bvh_nodes, 4))
    kinds = _capi.LIGHT_NODE_MASK | _capi.MESH_INSTANCE_MASK | _capi.MESH_LEAF_MASK | _capi.TRI_LEAF_MASK
    return int(((hi[:, 3] & kinds) == 0).sum())


@pytest.mark.parametrize("name", ["room", "field16", "sky_small", "textured_room", "instanced"])
def test_wide_tree_for_built_scenes(name):
    if name in ("room", "field16"):
        s = probe.trace_scenes()[name]
    elif name == "sky_small":
        s = scenes.sky_scene(width=64, height=36, count=4, level=4)
    elif name == "textured_room":
        s = scenes.textured_room_scene()
    else:
        import test_ref_payload as trp
        s = trp.instanced_scene()
    b = scenes.BuiltPayload(s)
    try:
        nw, ne, need, closest = info(b.payload, full=True)
        n_inner = inner_nodes(b.payload)
        # the builder's trees defer no entry: closest hit uses them, with a
        # stack of at least the binary traversal's depth (rays that may not
        # skip boxes walk the binary tree)
        assert closest == 1
        assert need >= b.stat.height - 1
        # every inner node is a wide node or is held in one's slots
        assert nw + ne == n_inner, (nw, ne, n_inner)
        # nesting boxes: most children of wide nodes are expanded
        assert ne >= 0.5 * nw, (nw, ne)
        assert 0 < need <= 96
        # a deeper tree needs at most three more words per two levels than
        # the binary traversal's stack
        assert need <= 3 * (b.stat.height + 1) // 2 + 3 + b.payload.num_bvh_nodes
    finally:
        b.free()


def _payload_with(b, patch):
    """a copy of b's payload with its node words patched by `patch(lo, hi)`"""
    p = b.payload
    n = p.num_bvh_nodes
    lo = np.ctypeslib.as_array(C.cast(p.bvh_min_right_start, C.POINTER(C.c_uint32)), (n, 4)).copy()
    hi = np.ctypeslib.as_array(C.cast(p.bvh_max_axis_count, C.POINTER(C.c_uint32)), (n, 4)).copy()
    patch(lo, hi)
    q = _capi.Payload()
    C.memmove(C.byref(q), C.byref(p), C.sizeof(q))
    q.bvh_min_right_start = lo.ctypes.data_as(C.POINTER(C.c_uint32))
    q.bvh_max_axis_count = hi.ctypes.data_as(C.POINTER(C.c_uint32))
    return q, (lo, hi)


def _first_inner(hi, start):
    kinds = _capi.LIGHT_NODE_MASK | _capi.MESH_INSTANCE_MASK | _capi.MESH_LEAF_MASK | _capi.TRI_LEAF_MASK
    i = start
    while hi[i, 3] & kinds:
        i += 1
    return i


def test_wide_tree_refuses_cycles_and_nan_bounds():
    s = probe.trace_scenes()["field16"]
    b = scenes.BuiltPayload(s)
    try:
        root = b.payload.bvh_root_node

        def cycle(lo, hi):
            i = _first_inner(hi, root + 1)
            lo[i, 3] = root  # an inner node's right child is the root
        q, keep = _payload_with(b, cycle)
        with pytest.raises(_capi.NoorError, match="cycle"):
            info(q, root)

        def nan_box(lo, hi):
            lo[-1, 0] = np.float32(np.nan).view(np.uint32)
        q, keep = _payload_with(b, nan_box)
        with pytest.raises(_capi.NoorError, match="NaN"):
            info(q, root)

        # a child box that sticks out of its parent's is not expanded
        nw0, ne0, _ = info(b.payload)

        def widen(lo, hi):
            # the root's left child's left child (the builder lays a left
            # child out right after its parent)
            assert _first_inner(hi, root) == root and _first_inner(hi, root + 1) == root + 1
            hi[root + 2, 0] = np.float32(1e30).view(np.uint32)
        q, keep = _payload_with(b, widen)
        nw1, ne1, _ = info(q, root)
        assert nw1 + ne1 == nw0 + ne0 and ne1 < ne0
    finally:
        b.free()
