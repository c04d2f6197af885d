"""The ray-query device code run on the CPU (tests/cpp/traverse_host_check.cu compiles
polytope_b200/csrc/traverse.cuh for the host): both forms of the walk the kernels use -- traverse()
(fused path kernels, one-thread-per-ray queries; the box form chosen once per ray) and the resumable
walk_step / walk_leaf (persistent kernels; two children pushed at once) -- against the oracle,
bit for bit on hit id, t, u, v and count for count on node and face tests.  Covers the min/max and
the compare-and-select box forms (exact_tree forces the latter), NaN / negative / zero tmax, zero,
negative-zero and NaN direction components, origins inside boxes, any-hit rays, and rays aimed at box
corners and edges, where Wald's edge functions come out zero.  The sm_100 packed form of the box
test is device-only and is pinned by the GPU parity tests."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from golden.make_golden import box_edge_rays, random_rays
import polytope_b200 as pb
from polytope_b200 import workloads as W
from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else None)

pytestmark = pytest.mark.skipif(NVCC is None, reason="needs nvcc (host compilation only)")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    exe = tmp_path_factory.mktemp("trav") / "traverse_host_check"
    subprocess.run([NVCC, "-O2", "-std=c++17", "-Xcompiler", "-ffp-contract=off,-fno-fast-math",
                    "-I", os.path.join(ROOT, "polytope_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "traverse_host_check.cu"), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    return exe


def leaf_ordered_faces(meshes, pairs, world):
    """The device's 48-byte face records in leaf order: world vertices, then (prim, mesh, 0)."""
    base = np.concatenate([[0], np.cumsum([len(m.faces) for m in meshes])[:-1]]).astype(np.uint32)
    prim = base[pairs[:, 0]] + pairs[:, 1]
    rec = np.zeros((len(pairs), 12), np.float32)
    rec[:, 0:9] = world[prim].reshape(-1, 9)
    rec[:, 9] = prim.view(np.float32)
    rec[:, 10] = pairs[:, 0].astype(np.uint32).view(np.float32)
    return rec


def edge_case_rays(n, seed):
    rng = np.random.default_rng(seed)
    rays = random_rays(n, seed, -4, 4, anyhit_tmax=3.0)
    k = np.arange(n)
    rays["tmax"][k % 11 == 3] = np.nan
    rays["tmax"][k % 11 == 5] = -1.0
    rays["tmax"][k % 11 == 7] = 0.0
    rays["dir"][k % 13 == 1, 0] = 0.0
    rays["dir"][k % 13 == 2, 1] = -0.0
    rays["dir"][k % 97 == 4, 2] = np.nan
    rays["org"][k % 17 == 6] = rng.uniform(-0.2, 0.2, (int((k % 17 == 6).sum()), 3))  # inside the scene's boxes
    return rays


def run(harness, tmp_path, meshes, env, rays, exact):
    nodes, pairs = pb.bvh_build(meshes)
    o = po.OracleScene(meshes, env)
    faces = leaf_ordered_faces(meshes, pairs, o.world_triangles())
    paths = [tmp_path / f for f in ("nodes.bin", "tris.bin", "rays.bin", "out.bin")]
    nodes.tofile(paths[0])
    faces.tofile(paths[1])
    np.ascontiguousarray(rays, po.RAY_DTYPE).tofile(paths[2])
    p = subprocess.run([str(harness)] + [str(x) for x in paths] + [str(int(exact))], capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr
    out = np.fromfile(paths[3], np.uint32).reshape(-1, 12)
    hits, nt, tt = o.trace(rays, counts=True)
    return out, hits, nt, tt


def check(out, hits, nt, tt, rays, what):
    ref = np.stack([hits["prim"], hits["t"].view(np.uint32), hits["u"].view(np.uint32), hits["v"].view(np.uint32)], 1)
    closest = (rays["flags"] & 1) == 0
    for form, cols in (("traverse", slice(0, 6)), ("walk_step", slice(6, 12))):
        got = out[:, cols]
        assert (got[:, 0] != 0xFFFFFFFE).all(), f"{what} {form}: guard failure"
        assert (got[closest, 0:4] == ref[closest]).all(), f"{what} {form}: closest hits differ"
        assert (got[:, 0] == ref[:, 0]).all(), f"{what} {form}: first accepted any-hit faces differ"
        assert (got[:, 4] == nt).all() and (got[:, 5] == tt).all(), f"{what} {form}: node / face test counts differ"


@pytest.mark.parametrize("exact", [False, True])
def test_device_walks_on_the_small_scene_match_the_oracle(harness, tmp_path, exact):
    meshes, env = W.small_scene()
    rays = edge_case_rays(40_000, 5)
    out, hits, nt, tt = run(harness, tmp_path, meshes, env, rays, exact)
    check(out, hits, nt, tt, rays, f"small scene, exact_tree={exact}")
    assert (hits["prim"][(rays["flags"] & 1) == 0] != pb.PRIM_NONE).mean() > 0.2


@pytest.mark.parametrize("exact", [False, True])
def test_device_walks_on_a_box_scene_match_the_oracle(harness, tmp_path, exact):
    meshes, env = W.batch_scene(30_000, np.random.default_rng(3))
    boxes = meshes[1]
    rays = np.concatenate([box_edge_rays(boxes, 4000, 2000, 9), edge_case_rays(20_000, 6)])
    out, hits, nt, tt = run(harness, tmp_path, meshes, env, rays, exact)
    check(out, hits, nt, tt, rays, f"box scene, exact_tree={exact}")
    assert (hits["prim"][:6000] != pb.PRIM_NONE).mean() > 0.5
