"""Failure paths that end in a status word, made to happen without faulting
the GPU: a traversal stack too small for the tree (the caller understates
the BVH height), and the wavefront's bounded bounce loop running out."""
import ctypes as C

import numpy as np
import pytest
import torch

from noor_b200 import _capi, scenes

from gpu_util import trace_closest

pytestmark = pytest.mark.gpu


def _deep_row(n: int = 1 << 18) -> scenes.SceneData:
    """n thin triangles side by side along x (each in the plane x = k / n,
    one per leaf): every split of the tree is on x, so a ray running along
    the row meets both children of every inner node and the traversal's
    stack grows by one entry per level (about 18 before the first leaf)"""
    x = (np.arange(n, dtype=np.float64) / n).astype(np.float32)
    V = np.zeros((3 * n, 4), np.float32)
    V[0::3, 0], V[0::3, 1], V[0::3, 2] = x, -0.5, -0.5
    V[1::3, 0], V[1::3, 1], V[1::3, 2] = x, 0.5, -0.5
    V[2::3, 0], V[2::3, 1], V[2::3, 2] = x, 0.0, 0.5
    V[:, 3] = 1.0
    tri = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    N = np.zeros((1, 4), np.float32)
    N[0, 0] = 1.0
    s = scenes.SceneData(vertices=V, normals=N, uvs=np.zeros((1, 2), np.float32), vindices=tri,
                         nindices=np.zeros((n, 3), np.uint32), uvindices=np.zeros((n, 3), np.uint32),
                         material_indices=np.zeros(n, np.uint32),
                         meshes=[dict(tri_start=0, tri_count=n, to_global=scenes.IDENTITY, instance=-1, light_idx=-1)],
                         materials=[scenes.material("diffuse")], skydome_type=_capi.NOOR_SKY_CONSTANT, name="deep")
    s.bvh = dict(scenes.DEFAULT_BVH, max_height=64, min_leaf_tris=1, max_leaf_tris=1)
    s.camera = dict(eye=(-1.0, 0.1, 0.0), look_at=(0.0, 0.1, 0.0), up=(0.0, 1.0, 0.0), fov_deg=10.0, w=32, h=32)
    s.render = dict(spp=1, bounces=2, rr=1, mis=0)
    return s


def _row_rays(n: int, seed: int = 0) -> np.ndarray:
    """rays from x = -1 along +x through the row (direction components all
    non-zero: the reference's slab test misses boxes for a zero one)"""
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 8), np.float32)
    r[:, 0] = -1.0
    r[:, 1] = rng.uniform(-0.1, 0.1, n)
    r[:, 2] = rng.uniform(-0.1, 0.1, n)
    r[:, 3] = np.inf
    d = np.array([1.0, 1e-5, 2e-5]) / np.linalg.norm([1.0, 1e-5, 2e-5])
    r[:, 4:7] = d
    return r


def test_traversal_stack_overflow_sets_the_status_bit():
    """with the spec's BVH height understated the binary traversal's stack
    (the megakernel's) holds 16 entries while a ray along the row needs one
    per level (about 18): it stops at the cap (no write past it) and sets
    NOOR_DEV_STACK_OVERFLOW.  The four-wide tree that ray batches and the
    wavefront walk sizes its stack from the tree itself, so the same spec
    leaves its hits exact and the status word clear."""
    s = _deep_row()
    built = scenes.BuiltPayload(s)
    assert built.stat.height > 18, built.stat.height
    rays = _row_rays(4096)
    r = scenes.Renderer(s, built=built)
    try:
        assert r.status(reset=True) == 0
        hits = trace_closest(rays)
        assert (hits[:, 6] == 1).all()
        assert np.allclose(hits[:, 0].view(np.float32), 1.0, atol=1e-5)
        r.render(1)
        assert r.status() == 0
        r.update_spec(bvh_height=0)
        assert np.array_equal(trace_closest(rays), hits)
        assert r.status() == 0
        r.render(1)
        assert r.status(reset=True) & _capi.NOOR_DEV_STACK_OVERFLOW
    finally:
        r.close()


@pytest.mark.parametrize("graph", [1, 0])
def test_wavefront_iteration_cap_sets_wait_timeout(graph):
    """a cap of 2 iterations ends the render's loop with paths still in
    flight: NOOR_DEV_WAIT_TIMEOUT, and the call returns; without the cap the
    same render completes with a clear status word"""
    s = scenes.room_scene(width=64, height=64, spp=4)
    r = scenes.Renderer(s)
    try:
        film = torch.zeros((64, 64, 4), dtype=torch.float32, device="cuda")
        f = scenes.wf_frame(0, s.camera, 4, s.render["bounces"], d_film=film.data_ptr())
        r.status(reset=True)
        _capi.call("noor_wavefront_render", C.byref(f), 1, C.byref(scenes.wf_params(128, 1 << 14, 1, graph, 2)))
        assert r.status(reset=True) & _capi.NOOR_DEV_WAIT_TIMEOUT
        _capi.call("noor_wavefront_render", C.byref(f), 1, C.byref(scenes.wf_params(128, 1 << 14, 1, graph, 0)))
        assert r.status(reset=True) == 0
        torch.cuda.synchronize()
        assert film[..., :3].mean().item() > 0.01
    finally:
        r.close()
