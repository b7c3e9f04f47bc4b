"""Generates the golden fixtures under tests/golden/ from the reference's own
host routines, compiled unmodified from the reference tree into
oracle/_ref/libnoor_ref.so (oracle/Makefile, target `ref`).

  hosek_rgb_dataset.npy  the Hosek-Wilkie RGB coefficient and radiance tables
                         (3 x 1080 + 3 x 120 floats) the reference vendors
                         (BSD-3, Hosek & Wilkie 2012)
  hosek_states.npz       arhosek_rgb_skymodelstate_alloc_update outputs
  bvh_golden.npz         BVH node words, root, height and triangle order of
                         the reference builder for four seeded scenes
  wald_golden.npz        WaldTriangle records for seeded triangles

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from noor_b200 import scenes  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent

# (name, scene constructor) pairs whose reference BVH is frozen
GOLDEN_SCENES = {
    "room": lambda: scenes.room_scene(seed=1),
    "spheres": lambda: scenes.SceneData(**scenes.sphere_field(11, 6, 3)[0], name="spheres"),
    # light nodes with sphere and disk bounds
    "room_sphere": lambda: scenes.room_scene(seed=1, light="sphere"),
    "room_disk": lambda: scenes.room_scene(seed=1, light="disk"),
}
HOSEK_CASES = [(3.0, 0.3, np.radians(30.0)), (2.0, 0.1, np.radians(10.0)), (5.5, 0.8, np.radians(60.0)),
               (10.0, 0.5, np.radians(45.0)), (1.0, 0.0, np.radians(85.0))]


def main() -> None:
    O.build(ref=True)
    np.save(OUT / "hosek_rgb_dataset.npy", O.ref_hosek_dataset())
    states = np.stack([O.ref_hosek_state(t, a, e) for (t, a, e) in HOSEK_CASES])
    np.savez_compressed(OUT / "hosek_states.npz", cases=np.array(HOSEK_CASES, np.float64), states=states)
    arrays = {}
    for name, make in GOLDEN_SCENES.items():
        s = make()
        b = scenes.BuiltPayload(s)
        nodes, root, order, height = O.ref_build_bvh(b.desc, s.num_triangles)
        arrays[f"{name}_nodes"] = nodes
        arrays[f"{name}_meta"] = np.array([root, height], np.uint32)
        arrays[f"{name}_order"] = order
    np.savez_compressed(OUT / "bvh_golden.npz", **arrays)
    rng = np.random.default_rng(123)
    tris = rng.normal(size=(512, 9)).astype(np.float32) * 3.0
    tris[:8, 6:9] = tris[:8, 0:3]          # degenerate (repeated vertex)
    tris[8:16, 3:6] = 2 * tris[8:16, 0:3]   # collinear through the origin
    tris[8:16, 6:9] = 3 * tris[8:16, 0:3]
    recs = np.stack([O.ref_wald(t) for t in tris])
    np.savez_compressed(OUT / "wald_golden.npz", tris=tris, recs=recs)
    print("wrote", sorted(p.name for p in OUT.glob("*.np*")))


if __name__ == "__main__":
    main()
