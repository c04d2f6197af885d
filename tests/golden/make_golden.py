"""Generates the golden fixtures in tests/golden/ (run where the reference tree is present).

Two kinds of fixture:

1. ``reference_unit_cases.json`` -- the inputs and expected outcomes of the reference's own unit
   tests for this path, transcribed from (paths relative to the Polytope source tree):
     tests/shapes/test_mesh.cpp:35-117        Wald closest hit on one triangle, both windings,
                                              and grazing rays from far away
     tests/test_bvh.cpp:6-212                 compaction offsets, bound() root / split
     tests/TestBoundingBox.cpp:10-31          slab test with an axis-aligned direction
     tests/cuda/test_bvh_traversal.cpp:16-203 ray/box cases (scene cuda-bvh-traversal1.ply)
     tests/TestIntersectionTests.cpp:10-38    WorldToLocal frame convention
     tests/shading/test_mirror_brdf.cpp:36-99 mirror sample vectors
   Each case is also checked here against the reference compiled from its sources (oracle/_ref).

2. ``*.npz`` -- outputs of the reference itself (oracle/_ref/libpolyref.so: the unmodified
   bvh::bound / compact / intersect_compact / Mesh::intersect, and the patched render loop) on
   the seeded synthetic workloads, at sizes the CPU oracle finishes in seconds.

Usage:  make -C oracle && python tests/golden/make_golden.py [batch_box_scene]
        (with the argument only batch_box_scene.npz is written)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402
import polytope_b200 as pb  # noqa: E402
from polytope_b200 import workloads as W  # noqa: E402

INF = float("inf")

UNIT_CASES = {
    "mesh_one_triangle": {
        "source": "tests/shapes/test_mesh.cpp:10-75",
        "vertices": [[0, 0, 0], [0, 1, 0], [1, 0, 0]],
        # fv0, fv1, fv2, origin z, direction z, expected normal z; Location (0.2, 0.2, 0) within 4 ulps
        "cases": [[0, 1, 2, -10, 1, -1], [0, 2, 1, -10, 1, -1], [0, 1, 2, 10, -1, 1], [0, 2, 1, 10, -1, 1]],
        "expected_location": [0.2, 0.2, 0.0],
    },
    "mesh_stay_above_surface": {
        "source": "tests/shapes/test_mesh.cpp:77-117",
        "plane_z": 0.2,
        "hit_point": [0.2, 0.2, 0.2],
        "origin_xy": [1.464552, 3.635245],
        "origin_z_per_k": -1.0364,
        # The reference test loops k over [100, 1e7) expecting a hit; the reference's own
        # Mesh::intersect (compiled from its sources) accepts only up to k ~ 337152 and rejects the
        # farther rays (the deltaT bound, mesh.cpp:312-322).  Parity is with the compiled reference:
        "k_values": [100, 101, 1000, 12345, 100000, 300000, 337152],
        "k_values_reference_misses": [337268, 777777, 1000000, 5000000, 9999999],
        "expected_normal": [0, 0, -1],
        "expected_location_z": 0.2,
    },
    "bvh_compact": {
        "source": "tests/test_bvh.cpp:6-163",
        # low / high child index per hand-built node (node index == tag bb.p1.x); expected
        # (tag, high_child_offset of interior nodes) in compacted order
        "trees": {
            "compact1": {"low": [-1], "high": [-1], "expect_tags": [0], "expect_offsets": {}},
            "compact3": {"low": [1, -1, -1], "high": [2, -1, -1], "expect_tags": [0, 1, 2], "expect_offsets": {"0": 2}},
            "compact5left": {"low": [1, 2, -1, -1, -1], "high": [4, 3, -1, -1, -1], "expect_tags": [0, 1, 2, 3, 4],
                             "expect_offsets": {"0": 4, "1": 2}},
            "compact5right": {"low": [1, -1, 3, -1, -1], "high": [2, -1, 4, -1, -1], "expect_tags": [0, 1, 2, 3, 4],
                              "expect_offsets": {"0": 2, "2": 2}},
            "compact7full": {"low": [1, 2, -1, -1, 5, -1, -1], "high": [4, 3, -1, -1, 6, -1, -1],
                             "expect_tags": [0, 1, 2, 3, 4, 5, 6], "expect_offsets": {"0": 4, "1": 2}},
        },
    },
    "bvh_bound": {
        "source": "tests/test_bvh.cpp:165-212",
        "one_triangle": [[0, 0, 0], [1, 0, 0], [0, 1, 0]],
        "four_triangles_offset": 2.0,
    },
    "bbox_hits": {
        "source": "tests/TestBoundingBox.cpp:10-31, tests/cuda/test_bvh_traversal.cpp:16-203",
        # box min, box max, origin, direction, expected
        "cases": [
            [[0, 0, 0], [1, 1, 1], [0.5, 0.5, 10], [0, 0, -1], True],
            [[-3, -1, -1], [3, 2, 1], [2, 0, 10], [0, 0, -1], True],
            [[-3, -1, -1], [-1, 2, 1], [2, 0, 10], [0, 0, -1], False],
            [[1, -1, -1], [3, 2, 1], [2, 0, 10], [0, 0, -1], True],
            [[-3, -1, -1], [3, 2, 1], [2, 0, 0], [-1, 0, 0], True],
            [[-3, -1, -1], [-1, 2, 1], [2, 0, 0], [-1, 0, 0], True],
            [[1, -1, -1], [3, 2, 1], [2, 0, 0], [-1, 0, 0], True],
            [[-3, -1, -1], [3, 2, 1], [-1.701634, -0.397628, -0.295537], [0.985882, -0.038071, 0.163058], True],
            [[-3, -1, -1], [-1, 2, 1], [-1.701634, -0.397628, -0.295537], [0.985882, -0.038071, 0.163058], True],
            [[1, -1, -1], [3, 2, 1], [-1.701634, -0.397628, -0.295537], [0.985882, -0.038071, 0.163058], True],
        ],
    },
    "world_to_local": {
        "source": "tests/TestIntersectionTests.cpp:10-38",
        # bent_normal, Tangent1, Tangent2, world, expected local (exact)
        "cases": [
            [[0, 0, 1], [1, 0, 0], [0, 1, 0], [0, 0, -1], [0, -1, 0]],
            [[0, 0, 1], [0, 1, 0], [1, 0, 0], [0, 0, -1], [0, -1, 0]],
        ],
    },
    "mirror_sample": {
        "source": "tests/shading/test_mirror_brdf.cpp:36-99",
        # incoming (normalized before the call), expected (normalized), exact equality
        "cases": [[[1, -1, 0], [1, 1, 0]], [[2, -1, 0], [2, 1, 0]], [[0, -1, 0], [0, 1, 0]]],
    },
    "philox4x32_10_kat": {
        "source": "Random123 known-answer vectors for philox4x32_10 (Salmon et al., SC'11)",
        # counter (4), key (2), expected (4) -- hex
        "cases": [
            [["00000000", "00000000", "00000000", "00000000"], ["00000000", "00000000"],
             ["6627e8d5", "e169c58d", "bc57ac4c", "9b00dbd8"]],
            [["ffffffff", "ffffffff", "ffffffff", "ffffffff"], ["ffffffff", "ffffffff"],
             ["408f276d", "41c83b0e", "a20bc7c6", "6d5451fd"]],
            [["243f6a88", "85a308d3", "13198a2e", "03707344"], ["a4093822", "299f31d0"],
             ["d16cfe09", "94fdcceb", "5001e420", "24126ea1"]],
        ],
    },
}


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def random_rays(n, seed, lo=-5.0, hi=5.0, anyhit_tmax=None):
    rng = np.random.default_rng(seed)
    rays = np.zeros(n, po.RAY_DTYPE)
    rays["org"] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    rays["dir"] = d / np.linalg.norm(d, axis=1)[:, None]
    rays["tmax"] = np.inf
    if anyhit_tmax is not None:
        rays["tmax"][1::2] = anyhit_tmax
        rays["flags"][1::2] = 1
    return rays


def stay_above_rays(c, ks):
    hp = np.asarray(c["hit_point"], np.float32)
    rays = np.zeros(len(ks), po.RAY_DTYPE)
    for i, k in enumerate(ks):
        o = np.array([c["origin_xy"][0], c["origin_xy"][1], np.float32(c["origin_z_per_k"]) * np.float32(k)], np.float32)
        rays["org"][i] = o
        rays["dir"][i] = po.normalize(hp - o)
    rays["tmax"] = np.inf
    return rays


def stay_above_mesh(c):
    z = np.float32(c["plane_z"])
    v = np.array([[0, 0, z], [0, 1, z], [1, 0, z]], np.float32)
    return pb.Mesh(v[:, 0], v[:, 1], v[:, 2], np.array([[0, 1, 2]], np.uint32))


def check_unit_cases_against_ref():
    """Sanity: the reference itself reproduces the transcribed cases."""
    for bmin, bmax, o, d, exp in UNIT_CASES["bbox_hits"]["cases"]:
        got = po.bbox_hits("ref", bmin + bmax, o, d)
        assert got == exp, (bmin, bmax, o, d, exp, got)
    c = UNIT_CASES["mesh_stay_above_surface"]
    ref = po.RefScene([stay_above_mesh(c)])
    assert (ref.trace(stay_above_rays(c, c["k_values"]))["prim"] == 0).all()
    assert (ref.trace(stay_above_rays(c, c["k_values_reference_misses"]))["prim"] == po.PRIM_NONE).all()


def scene_inputs_digest(meshes) -> str:
    return sha(*[a for m in meshes for a in (m.x, m.y, m.z, m.faces, m.object_to_world)])


def box_edge_rays(mesh, n_corner: int, n_edge: int, seed: int) -> np.ndarray:
    """Closest-hit rays from random origins toward exact box corners and edge midpoints of a
    boxes mesh (batched workload), where Wald edge functions can come out exactly zero."""
    rng = np.random.default_rng(seed)
    v = np.stack([mesh.x, mesh.y, mesh.z], 1).astype(np.float32)
    tgt = np.concatenate([v[rng.integers(0, len(v), n_corner)],
                          (0.5 * (v[0::8][:n_edge] + v[1::8][:n_edge])).astype(np.float32)])
    org = rng.uniform(-6, 6, (len(tgt), 3)).astype(np.float32)
    rays = np.zeros(len(tgt), po.RAY_DTYPE)
    rays["org"] = org
    d = tgt - org
    rays["dir"] = (d / np.linalg.norm(d, axis=1)[:, None]).astype(np.float32)
    rays["tmax"] = np.inf
    return rays


BOX_SCENE_INDEX = 12  # scene 12 of the 256-scene batched workload: 1,570 faces (104 boxes), 64x64, 64 spp


def make_box_scene_fixture():
    """Scene 12 of the batched workload (seed 23) rendered by the reference's patched render loop at
    its own resolution, spp and depth (64x64, 64 spp, depth 6, NEE), plus closest hits and per-ray
    node/face test counts of rays aimed at its box corners and edges."""
    meshes, env, d = W.batched_workload(256)[BOX_SCENE_INDEX]
    ref = po.RefScene(meshes, env)
    nodes, pairs = ref.tree()
    rays = box_edge_rays(meshes[1], 2048, 1024, 61)
    hits, nt, tt = ref.trace(rays, counts=True)
    rgb, prim = ref.render(dict(d, flags=1))
    np.savez_compressed(os.path.join(HERE, "batch_box_scene.npz"), inputs_sha=scene_inputs_digest(meshes),
                        tree_sha=sha(nodes, pairs), num_nodes=len(nodes), rays=rays, hits=hits, node_tests=nt,
                        tri_tests=tt, rgb=rgb, prim=prim, width=d["width"], height=d["height"], spp=d["spp"],
                        max_depth=d["max_depth"], seed=d["seed"])


def main():
    if not po.ref_available():
        raise SystemExit("oracle/_ref/libpolyref.so is not built; run `make -C oracle` where the reference is present")
    if sys.argv[1:] == ["batch_box_scene"]:  # regenerate only this fixture
        make_box_scene_fixture()
        return
    check_unit_cases_against_ref()
    with open(os.path.join(HERE, "reference_unit_cases.json"), "w") as f:
        json.dump(UNIT_CASES, f, indent=1)

    # small scene: tree, camera rays, hits on random rays, a small render (NEE on and off)
    meshes, env = W.small_scene()
    ref = po.RefScene(meshes, env)
    nodes, pairs = ref.tree()
    rays = random_rays(8192, 5, -4.0, 4.0, anyhit_tmax=3.0)
    hits, nt, tt = ref.trace(rays, counts=True)
    frames = ref.hit_frames(rays[rays["flags"] == 0][:2048])
    small = dict(width=80, height=60, spp=4, max_depth=4, seed=1, camera=W.SMALL_CAMERA)
    cam = po.camera_rays_ref(small)
    rgb_nee, prim_nee = ref.render(dict(small, flags=1))
    rgb_bsdf, prim_bsdf = ref.render(dict(small, flags=0))
    np.savez_compressed(os.path.join(HERE, "small_scene.npz"), inputs_sha=scene_inputs_digest(meshes),
                        tree_sha=sha(nodes, pairs), num_nodes=len(nodes), rays=rays, hits=hits, node_tests=nt,
                        tri_tests=tt, frames=frames, camera_rays=cam, rgb_nee=rgb_nee, prim_nee=prim_nee,
                        rgb_bsdf=rgb_bsdf, prim_bsdf=prim_bsdf)

    # microbench mesh: tree digest and the first 65536 rays of the ray set
    mm, mrays = W.microbench(n_rays=65536)
    ref2 = po.RefScene(mm)
    n2, p2 = ref2.tree()
    h2, nt2, tt2 = ref2.trace(mrays, counts=True)
    np.savez_compressed(os.path.join(HERE, "microbench.npz"), inputs_sha=scene_inputs_digest(mm),
                        rays_sha=sha(mrays), tree_sha=sha(n2, p2), num_nodes=len(n2), hits=h2, node_tests=nt2,
                        tri_tests=tt2)

    # instanced scene (5 instances, small icosphere level to keep the fixture quick)
    im, ienv = W.instanced_scene(level=4)
    ref3 = po.RefScene(im, ienv)
    n3, p3 = ref3.tree()
    inst = dict(width=64, height=40, spp=2, max_depth=8, seed=1, camera=W.INSTANCED_CAMERA, flags=1)
    rgb3, prim3 = ref3.render(inst)
    np.savez_compressed(os.path.join(HERE, "instanced_small.npz"), inputs_sha=scene_inputs_digest(im),
                        tree_sha=sha(n3, p3), num_nodes=len(n3), rgb=rgb3, prim=prim3)
    make_box_scene_fixture()
    print("wrote fixtures:", sorted(f for f in os.listdir(HERE) if f.endswith((".npz", ".json"))))


if __name__ == "__main__":
    main()
