"""The CPU oracle (oracle/oracle.cpp) against the reference's own unit-test vectors and against
fixtures produced by running the reference's code (tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, assert_bit_equal, load_golden
from oracle import pyoracle as po
import polytope_b200 as pb
from polytope_b200 import workloads as W
from golden.make_golden import scene_inputs_digest, sha  # noqa: E402

CASES = json.load(open(os.path.join(GOLDEN, "reference_unit_cases.json")))
ULP4 = 4


def ulps(a, b):
    a, b = np.float32(a), np.float32(b)
    ia, ib = int(a.view(np.int32)), int(b.view(np.int32))
    if ia < 0:
        ia = -0x80000000 - ia
    if ib < 0:
        ib = -0x80000000 - ib
    return abs(ia - ib)


def one_triangle_mesh(verts, f):
    v = np.asarray(verts, np.float32)
    return pb.Mesh(v[:, 0], v[:, 1], v[:, 2], np.asarray([f], np.uint32))


def single_ray(o, d, tmax=np.inf, flags=0):
    r = np.zeros(1, po.RAY_DTYPE)
    r["org"] = o
    r["dir"] = d
    r["tmax"] = tmax
    r["flags"] = flags
    return r


def test_mesh_one_triangle_both_windings():
    c = CASES["mesh_one_triangle"]
    for f0, f1, f2, oz, dz, nz in c["cases"]:
        s = po.OracleScene([one_triangle_mesh(c["vertices"], (f0, f1, f2))])
        ray = single_ray((0.2, 0.2, oz), (0, 0, dz))
        hit = s.trace(ray)[0]
        assert hit["prim"] == 0
        fr = s.hit_frames(ray)[0]
        loc, n = fr[0:3], fr[3:6]
        assert tuple(n) == (0.0, 0.0, float(nz)) or (ulps(n[0], 0) <= ULP4 and ulps(n[1], 0) <= ULP4 and ulps(n[2], nz) <= ULP4)
        for k in range(3):
            assert ulps(loc[k], c["expected_location"][k]) <= ULP4, (loc, f0, f1, f2)


def test_mesh_stay_above_surface():
    from golden.make_golden import stay_above_mesh, stay_above_rays
    c = CASES["mesh_stay_above_surface"]
    s = po.OracleScene([stay_above_mesh(c)])
    rays = stay_above_rays(c, c["k_values"])
    assert (s.trace(rays)["prim"] == 0).all()
    for fr in s.hit_frames(rays):
        for j in range(3):
            assert ulps(fr[3 + j], c["expected_normal"][j]) <= ULP4, fr[3:6]
        # The reference test compares Location.z with 0.2 only at k = 9999999, a ray its own
        # Wald test rejects; the compiled reference's spawn point sits 6-8 ulps below the plane
        # (the robust offset toward the incoming side, mesh.cpp:419-436).
        assert ulps(fr[2], c["expected_location_z"]) <= 16, fr[0:3]
    # farther rays: the compiled reference rejects them, so must the restatement
    assert (s.trace(stay_above_rays(c, c["k_values_reference_misses"]))["prim"] == po.PRIM_NONE).all()


def test_bvh_compact_offsets():
    for name, t in CASES["bvh_compact"]["trees"].items():
        got = po.compact_shape(t["low"], t["high"])
        assert [g[0] for g in got] == t["expect_tags"], name
        for idx, off in t["expect_offsets"].items():
            assert got[int(idx)][1] == off, (name, idx, got)


def test_bvh_bound_root_and_split():
    c = CASES["bvh_bound"]
    s = po.OracleScene([one_triangle_mesh(c["one_triangle"], (0, 1, 2))])
    nodes, _ = s.tree()
    assert len(nodes) == 1 and nodes[0]["num_faces"] == 1
    off = c["four_triangles_offset"]
    v = np.array([[0 + i * off, 0, 0] for i in range(4)] + [[1 + i * off, 0, 0] for i in range(4)] +
                 [[0 + i * off, 1, 0] for i in range(4)], np.float32)
    faces = np.array([[i, 4 + i, 8 + i] for i in range(4)], np.uint32)
    s = po.OracleScene([pb.Mesh(v[:, 0], v[:, 1], v[:, 2], faces)])
    nodes, _ = s.tree()
    assert nodes[0]["num_faces"] == 0 and len(nodes) >= 3  # root split into low and high children


def test_bbox_hits_cases():
    for bmin, bmax, o, d, exp in CASES["bbox_hits"]["cases"]:
        assert po.bbox_hits("orc", bmin + bmax, o, d) == exp, (bmin, bmax, o, d)


def test_world_to_local_and_mirror():
    for n, t1, t2, w, exp in CASES["world_to_local"]["cases"]:
        got = po.world_to_local(t1, n, t2, w)
        assert tuple(got) == tuple(np.float32(exp)), (got, exp)
    for inc, exp in CASES["mirror_sample"]["cases"]:
        got = po.mirror_sample(po.normalize(inc))
        assert_bit_equal(got, po.normalize(exp), "mirror")


def test_philox_known_answers():
    for ctr, key, exp in CASES["philox4x32_10_kat"]["cases"]:
        c = [int(x, 16) for x in ctr]
        k = [int(x, 16) for x in key]
        got = po.philox(c, k[0] | (k[1] << 32))
        assert [int(x) for x in got] == [int(x, 16) for x in exp]


def test_small_scene_fixture():
    g = load_golden("small_scene.npz")
    meshes, env = W.small_scene()
    assert scene_inputs_digest(meshes) == str(g["inputs_sha"])
    s = po.OracleScene(meshes, env)
    nodes, pairs = s.tree()
    assert len(nodes) == int(g["num_nodes"]) and sha(nodes, pairs) == str(g["tree_sha"])
    hits, nt, tt = s.trace(g["rays"], counts=True)
    closest = g["rays"]["flags"] == 0
    for f in ("prim", "t", "u", "v"):
        assert_bit_equal(hits[f][closest], g["hits"][f][closest], f)
    assert_bit_equal((hits["prim"] != po.PRIM_NONE)[~closest], (g["hits"]["prim"] != po.PRIM_NONE)[~closest], "any")
    assert_bit_equal(nt[closest], g["node_tests"][closest], "node tests")
    assert_bit_equal(tt[closest], g["tri_tests"][closest], "tri tests")
    rays_c = g["rays"][closest][:2048]
    assert_bit_equal(s.hit_frames(rays_c), g["frames"], "frames")


def test_small_scene_camera_and_render_fixture():
    g = load_golden("small_scene.npz")
    meshes, env = W.small_scene()
    s = po.OracleScene(meshes, env)
    small = dict(width=80, height=60, spp=4, max_depth=4, seed=1, camera=W.SMALL_CAMERA)
    assert_bit_equal(po.camera_rays_oracle(small).view(np.uint32), g["camera_rays"].view(np.uint32), "camera")
    for flags, key in ((1, "nee"), (0, "bsdf")):
        rgb, prim = s.render(dict(small, flags=flags))
        assert_bit_equal(rgb, g[f"rgb_{key}"], f"rgb {key}")
        assert_bit_equal(prim, g[f"prim_{key}"], f"prim {key}")
    assert g["rgb_nee"].mean() > 0


def test_microbench_fixture():
    g = load_golden("microbench.npz")
    mm, rays = W.microbench(n_rays=65536)
    assert scene_inputs_digest(mm) == str(g["inputs_sha"]) and sha(rays) == str(g["rays_sha"])
    s = po.OracleScene(mm)
    nodes, pairs = s.tree()
    assert sha(nodes, pairs) == str(g["tree_sha"])
    hits, nt, tt = s.trace(rays, counts=True)
    closest = rays["flags"] == 0
    for f in ("prim", "t", "u", "v"):
        assert_bit_equal(hits[f][closest], g["hits"][f][closest], f)
    assert_bit_equal((hits["prim"] != po.PRIM_NONE)[~closest], (g["hits"]["prim"] != po.PRIM_NONE)[~closest], "any")
    assert_bit_equal(nt[closest], g["node_tests"][closest], "nodes")
    assert_bit_equal(tt[closest], g["tri_tests"][closest], "tris")


def test_instanced_fixture():
    g = load_golden("instanced_small.npz")
    im, env = W.instanced_scene(level=4)
    assert scene_inputs_digest(im) == str(g["inputs_sha"])
    s = po.OracleScene(im, env)
    nodes, pairs = s.tree()
    assert sha(nodes, pairs) == str(g["tree_sha"])
    rgb, prim = s.render(dict(width=64, height=40, spp=2, max_depth=8, seed=1, camera=W.INSTANCED_CAMERA, flags=1))
    assert_bit_equal(rgb, g["rgb"], "rgb")
    assert_bit_equal(prim, g["prim"], "prim")


def test_batch_box_scene_fixture():
    """Scene 12 of the 256-scene batched workload (icosphere among 104 boxes, 64x64, 64 spp, depth
    6, NEE): tree, box corner/edge hits with per-ray counts and the whole film equal the
    reference's."""
    from golden.make_golden import BOX_SCENE_INDEX
    g = load_golden("batch_box_scene.npz")
    meshes, env, d = W.batched_workload(256)[BOX_SCENE_INDEX]
    assert scene_inputs_digest(meshes) == str(g["inputs_sha"])
    s = po.OracleScene(meshes, env)
    nodes, pairs = s.tree()
    assert sha(nodes, pairs) == str(g["tree_sha"])
    hits, nt, tt = s.trace(g["rays"], counts=True)
    for f in ("prim", "t", "u", "v"):
        assert_bit_equal(hits[f], g["hits"][f], f)
    assert_bit_equal(nt, g["node_tests"], "nodes")
    assert_bit_equal(tt, g["tri_tests"], "tris")
    rgb, prim = s.render(dict(d, flags=1))
    assert_bit_equal(rgb, g["rgb"], "rgb")
    assert_bit_equal(prim, g["prim"], "prim")


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref is only built where the reference tree is present")
def test_oracle_matches_reference_on_random_multimesh_scene():
    rng = np.random.default_rng(7)
    meshes = []
    for k in range(3):
        c = rng.uniform(-3, 3, (1500, 3)).astype(np.float32)
        v = (c[:, None, :] + rng.normal(0, 0.2, (1500, 3, 3))).astype(np.float32).reshape(-1, 3)
        M = np.eye(4, dtype=np.float32)
        M[:3, 3] = rng.uniform(-1, 1, 3)
        M[0, 1] = 0.25 * k
        meshes.append(pb.Mesh(v[:, 0], v[:, 1], v[:, 2], np.arange(4500, dtype=np.uint32).reshape(-1, 3),
                              object_to_world=M, material=1 + (k % 2), is_light=(k == 2), emission=(900,) * 3 if k == 2 else (0,) * 3))
    o, r = po.OracleScene(meshes, (30, 40, 50)), po.RefScene(meshes, (30, 40, 50))
    no, po_ = o.tree()
    nr, pr = r.tree()
    assert no.tobytes() == nr.tobytes() and (po_ == pr).all()
    from golden.make_golden import random_rays
    rays = random_rays(20000, 3, anyhit_tmax=2.5)
    ho, nto, tto = o.trace(rays, counts=True)
    hr, ntr, ttr = r.trace(rays, counts=True)
    c = rays["flags"] == 0
    for f in ("prim", "t", "u", "v"):
        assert_bit_equal(ho[f][c], hr[f][c], f)
    assert_bit_equal(nto[c], ntr[c], "nodes")
    assert ((ho["prim"] != po.PRIM_NONE) == (hr["prim"] != po.PRIM_NONE)).all()
    assert_bit_equal(o.hit_frames(rays[c][:3000]), r.hit_frames(rays[c][:3000]), "frames")
    desc = dict(width=40, height=30, spp=3, max_depth=5, seed=9, flags=3,
                camera=dict(eye=(0, 1, 9), look_at=(0, 0, 0), up=(0, 1, 0), fov=50.0))
    a, pa = o.render(desc)
    b, pb_ = r.render(desc)
    assert_bit_equal(a, b, "render")
    assert_bit_equal(pa, pb_, "prim")


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref is only built where the reference tree is present")
@pytest.mark.parametrize("flags", [1, 0, 3], ids=["nee", "bsdf", "nee_jitter"])
def test_oracle_matches_reference_on_the_full_small_config(flags):
    """The small configuration at its full size (320x240, 8 spp, depth 4): the restatement's film
    and primary ids equal the compiled reference's render loop bit for bit."""
    meshes, env = W.small_scene()
    o, r = po.OracleScene(meshes, env), po.RefScene(meshes, env)
    d = dict(W.SMALL_RENDER, flags=flags)
    a, pa = o.render(d)
    b, pb_ = r.render(d)
    assert_bit_equal(a, b, "film")
    assert_bit_equal(pa, pb_, "primary ids")
    assert a.mean() > 1.0


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref is only built where the reference tree is present")
def test_full_instanced_scene_tree_and_band_match_reference():
    """The instanced path-trace configuration at full size (5 displaced icosphere-8 instances and a
    ground, 6,553,604 faces): the library's parallel SAH build, the restatement and the reference's
    bvh::bound + compact give the same tree byte for byte, and a 4-row band of the 1920x1080 frame
    (4 spp, depth 8, NEE) renders identically in the restatement and the reference."""
    meshes, env = W.instanced_scene()
    nodes, pairs = pb.bvh_build(meshes)
    r = po.RefScene(meshes, env)
    nr, pr = r.tree()
    assert nodes.tobytes() == nr.tobytes() and (pairs == pr).all()
    o = po.OracleScene(meshes, env)
    no, po_ = o.tree()
    assert no.tobytes() == nr.tobytes() and (po_ == pr).all()
    d = dict(W.INSTANCED_RENDER, spp=4, flags=1)
    a, pa = o.render(d, rows=(530, 534))
    b, pb_ = r.render(d, rows=(530, 534))
    assert_bit_equal(a, b, "band film")
    assert_bit_equal(pa, pb_, "band primary ids")
    assert a[530:534].mean() > 1.0 and (pa[530:534] != po.PRIM_NONE).any()


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref is only built where the reference tree is present")
def test_oracle_matches_reference_on_the_full_microbench():
    """All 16,777,216 microbench rays on the 1,310,720-face displaced icosphere: closest hits (id, t,
    u, v) bit-exact and any-hit outcomes equal between the restatement and the reference's
    bvh::intersect_compact; per-ray node and face test counts equal on the first 1,048,576 rays."""
    mm, rays = W.microbench()
    o, r = po.OracleScene(mm), po.RefScene(mm)
    ho, hr = o.trace(rays), r.trace(rays)
    c = rays["flags"] == 0
    for f in ("prim", "t", "u", "v"):
        assert_bit_equal(ho[f][c], hr[f][c], f)
    assert ((ho["prim"] != po.PRIM_NONE) == (hr["prim"] != po.PRIM_NONE)).all()
    sub = rays[:1 << 20]
    _, nto, tto = o.trace(sub, counts=True)
    _, ntr, ttr = r.trace(sub, counts=True)
    cs = sub["flags"] == 0
    assert_bit_equal(nto[cs], ntr[cs], "node tests")
    assert_bit_equal(tto[cs], ttr[cs], "face tests")


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref is only built where the reference tree is present")
def test_oracle_matches_reference_on_batch_scenes_with_boxes():
    """Scenes of the batched workload (a displaced icosphere among axis-aligned boxes, 12 faces
    each, a quad light, environment 0.2), with rays aimed at box corners and edge midpoints, where
    edge functions can come out exactly zero and the Wald test takes its FP64 branch; trees, closest
    hits with counts,
    and a 64x64, 4 spp, depth 6 film with NEE are bit-exact between the restatement and the
    reference."""
    work = W.batched_workload(3, seed=41, min_tris=20_000, max_tris=60_000, resolutions=(64,), spps=(4,))
    rng = np.random.default_rng(43)
    for meshes, env, d in work:
        o, r = po.OracleScene(meshes, env), po.RefScene(meshes, env)
        no, po_ = o.tree()
        nr, pr = r.tree()
        assert no.tobytes() == nr.tobytes() and (po_ == pr).all()
        # rays aimed at box corners and edge midpoints (exact vertex coordinates) plus random ones
        bx = meshes[1]
        v = np.stack([bx.x, bx.y, bx.z], 1).astype(np.float32)
        tgt = np.concatenate([v[rng.integers(0, len(v), 6000)],
                              (0.5 * (v[0::8][:3000] + v[1::8][:3000])).astype(np.float32)])
        org = rng.uniform(-6, 6, (len(tgt), 3)).astype(np.float32)
        rays = np.zeros(len(tgt), po.RAY_DTYPE)
        rays["org"] = org
        dd = tgt - org
        rays["dir"] = (dd / np.linalg.norm(dd, axis=1)[:, None]).astype(np.float32)
        rays["tmax"] = np.inf
        ho, nto, tto = o.trace(rays, counts=True)
        hr, ntr, ttr = r.trace(rays, counts=True)
        for f in ("prim", "t", "u", "v"):
            assert_bit_equal(ho[f], hr[f], f)
        assert_bit_equal(nto, ntr, "node tests")
        assert_bit_equal(tto, ttr, "face tests")
        assert (ho["prim"] != po.PRIM_NONE).mean() > 0.3
        desc = dict(d, flags=1)
        a, pa = o.render(desc)
        b, pb_ = r.render(desc)
        assert_bit_equal(a, b, "film")
        assert_bit_equal(pa, pb_, "primary ids")


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref is only built where the reference tree is present")
def test_oracle_matches_reference_with_vertex_normals(tmp_path):
    """A scene read from a PBRT file whose meshes mix vertex normals (interpolated in the post-hit
    frame, mesh.cpp:385-410) with face normals, mirrors, area lights and instances: hit frames and
    a rendered film with NEE are bit-exact between the restatement and the reference."""
    from test_pbrt_cpu import write_scene
    s = pb.load_pbrt(write_scene(tmp_path))
    assert any(m.normals is not None for m in s.meshes) and any(m.normals is None for m in s.meshes)
    o, r = po.OracleScene(s.meshes, s.env), po.RefScene(s.meshes, s.env)
    # closest-hit rays from random points toward random points of faces of the normal-bearing meshes
    rng = np.random.default_rng(5)
    base = np.cumsum([0] + [len(m.faces) for m in s.meshes])
    prims = np.concatenate([np.arange(base[k], base[k + 1]) for k, m in enumerate(s.meshes) if m.normals is not None])
    tri = o.world_triangles()[rng.choice(prims, 6000)]
    bary = rng.dirichlet((1, 1, 1), 6000).astype(np.float32)
    tgt = (tri * bary[:, :, None]).sum(1).astype(np.float32)
    org = rng.uniform(-6, 6, (6000, 3)).astype(np.float32)
    rays = np.zeros(6000, po.RAY_DTYPE)
    rays["org"] = org
    dd = tgt - org
    rays["dir"] = (dd / np.linalg.norm(dd, axis=1)[:, None]).astype(np.float32)
    rays["tmax"] = np.inf
    ho, hr = o.trace(rays), r.trace(rays)
    for f in ("prim", "t", "u", "v"):
        assert_bit_equal(ho[f], hr[f], f)
    hit = ho["prim"][ho["prim"] != po.PRIM_NONE]
    assert np.isin(hit, prims).sum() > 2000  # most hits land on meshes with vertex normals
    assert_bit_equal(o.hit_frames(rays), r.hit_frames(rays), "frames")
    d = dict(s.render_args(), seed=5, flags=1)
    a, pa = o.render(d)
    b, pb_ = r.render(d)
    assert_bit_equal(a, b, "film")
    assert_bit_equal(pa, pb_, "primary ids")
    assert a.mean() > 0.5


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref is only built where the reference tree is present")
@pytest.mark.parametrize("w,h,spp,depth", [(1, 1, 1, 0), (7, 3, 2, 1), (13, 9, 3, 2), (2, 17, 1, 9)])
@pytest.mark.parametrize("flags", [0, 1, 3], ids=["bsdf", "nee", "nee_jitter"])
def test_oracle_matches_reference_on_edge_render_shapes(w, h, spp, depth, flags):
    """Degenerate frame shapes and depths (one pixel, odd sizes, max depth 0 and 1, a deeper path
    than the configurations use): films and primary ids equal the reference's render loop."""
    meshes, env = W.small_scene(level=3)
    o, r = po.OracleScene(meshes, env), po.RefScene(meshes, env)
    d = dict(width=w, height=h, spp=spp, max_depth=depth, seed=17, camera=W.SMALL_CAMERA, flags=flags)
    a, pa = o.render(d)
    b, pb_ = r.render(d)
    assert_bit_equal(a, b, "film")
    assert_bit_equal(pa, pb_, "primary ids")


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref is only built where the reference tree is present")
def test_oracle_matches_reference_on_edge_rays():
    """The edge-case ray set of the device tests (both windings, axis-aligned directions with
    infinite inverses, rays through edges and vertices, tmax 0 and just short of the hit, origins
    inside boxes) plus directions with signed zeros: closest hits and per-ray counts equal the
    reference's bvh::intersect_compact, and any-hit outcomes equal its closest-hit predicate."""
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1]], np.float32)
    meshes = [pb.Mesh(v[:, 0], v[:, 1], v[:, 2], np.array([[0, 1, 2], [0, 2, 1], [1, 3, 4], [0, 3, 1]], np.uint32))]
    cases = []
    for o, d in [((0.25, 0.25, 5), (0, 0, -1)), ((0.25, 0.25, -5), (0, 0, 1)), ((0.5, 0, 5), (0, 0, -1)),
                 ((0, 0, 5), (0, 0, -1)), ((0.5, 0.5, 5), (0, 0, -1)), ((1, 0, 5), (0, 0, -1)),
                 ((0.3, 0.3, 0.1), (0, 0, -1)), ((0.2, 0.2, 0.2), (1, 0, 0)), ((-1, 0.5, 0.5), (1, 0, 0)),
                 ((0.5, 0.5, 0.5), (0, 1, 0)), ((0.25, 0.25, 5), (0, 0, 1)), ((2, 2, 2), (-1, -1, -1)),
                 ((0.25, 0.25, 5), (-0.0, 0.0, -1)), ((0.25, 0.25, 5), (0.0, -0.0, -1)),
                 ((0.5, 0.5, -2), (-0.0, -0.0, 1)), ((1, 1, 1), (-0.57735026, -0.57735026, -0.57735026))]:
        for tmax in (np.inf, 0.0, 4.9999, 5.0):
            for flags in (0, 1):
                cases.append((o, d, tmax, flags))
    rays = np.zeros(len(cases), po.RAY_DTYPE)
    for i, (o, d, tmax, flags) in enumerate(cases):
        rays["org"][i], rays["dir"][i], rays["tmax"][i], rays["flags"][i] = o, d, tmax, flags
    o_, r_ = po.OracleScene(meshes), po.RefScene(meshes)
    ho, nto, tto = o_.trace(rays, counts=True)
    hr, ntr, ttr = r_.trace(rays, counts=True)
    c = rays["flags"] == 0
    for f in ("prim", "t", "u", "v"):
        assert_bit_equal(ho[f][c], hr[f][c], f)
    assert_bit_equal(nto[c], ntr[c], "nodes")
    assert_bit_equal(tto[c], ttr[c], "faces")
    assert ((ho["prim"] != po.PRIM_NONE) == (hr["prim"] != po.PRIM_NONE)).all()
    assert (ho["prim"][c] != po.PRIM_NONE).sum() >= 10


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref is only built where the reference tree is present")
def test_oracle_matches_reference_on_serving_pool_scenes():
    """The two smallest of the first four resident scenes of the serving workload (the displaced
    sphere instanced with seeded rigid transforms, Lambert or mirror, over a ground quad, a 3x3
    light and environment 0.2): trees byte for byte, and an 8-row band of a 256x256, 4 spp, depth 5
    request with NEE renders identically."""
    pool = sorted(W.serving_pool(4), key=lambda s: sum(len(m.faces) for m in s[0]))[:2]
    for meshes, env in pool:
        o, r = po.OracleScene(meshes, env), po.RefScene(meshes, env)
        no, po_ = o.tree()
        nr, pr = r.tree()
        assert no.tobytes() == nr.tobytes() and (po_ == pr).all()
        d = dict(width=256, height=256, spp=4, max_depth=5, seed=23, camera=W.SERVE_CAMERA, flags=1)
        a, pa = o.render(d, rows=(124, 132))
        b, pb_ = r.render(d, rows=(124, 132))
        assert_bit_equal(a, b, "band film")
        assert_bit_equal(pa, pb_, "band primary ids")
        assert a[124:132].mean() > 0.1
