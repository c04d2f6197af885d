"""GPU parity of the ray-query path (pt_trace through the C ABI) against the CPU oracle and the
reference fixtures: hit id, t, u, v bit-exact for closest-hit rays, identical any-hit booleans,
identical per-ray node / face test counts (which pins the traversal order)."""
import numpy as np
import pytest

from conftest import assert_bit_equal, load_golden
import polytope_b200 as pb
from polytope_b200 import workloads as W
from oracle import pyoracle as po
from golden.make_golden import random_rays

pytestmark = pytest.mark.gpu


def compare(hits, ref, rays, what):
    c = rays["flags"] == 0
    for f in ("prim", "t", "u", "v"):
        assert_bit_equal(hits[f][c], ref[f][c], f"{what} {f}")
    assert_bit_equal(hits["prim"][~c] != pb.PRIM_NONE, ref["prim"][~c] != pb.PRIM_NONE, f"{what} any-hit")


def test_exact_helpers_on_device(cuda_device):
    from test_host_cpu import f64_cases, f64_reference
    q = f64_cases(5000, 2)
    got = pb.selftest_device(0, q, len(q))
    exp = f64_reference(q)
    ok = ~np.isnan(exp)
    assert_bit_equal(got[ok], exp[ok], "device f64 emulation")
    u = (np.arange(1 << 16, dtype=np.uint32) << 8).astype(np.float32) * np.float32(2 ** -24)
    sc = pb.selftest_device(1, u, len(u))
    host = np.array([po.sincos_2pi(float(x)) for x in u[::97]], np.float32)
    assert_bit_equal(sc[::97], host, "sincos")
    assert np.abs(sc[:, 0] - np.sin(2 * np.pi * u.astype(np.float64))).max() < 3e-7
    ctr = np.random.default_rng(1).integers(0, 2 ** 32, (4096, 4), dtype=np.uint64).astype(np.uint32)
    dev = pb.selftest_device(2, ctr, len(ctr), seed=0x0123456789ABCDEF)
    host = np.array([po.philox(c, 0x0123456789ABCDEF) for c in ctr[:256]])
    assert (dev[:256] == host).all()


def test_box_test_on_device_matches_reference_semantics(cuda_device):
    """BoundingBox::Hits with its inside early-out, against the device test that skips the early-out
    when it cannot change the answer: origins inside, outside and on faces; zero, negative-zero and
    NaN direction components; tmax of inf, 0, positive, negative and NaN."""
    rng = np.random.default_rng(17)
    n = 20000
    lo = rng.uniform(-2, 1, (n, 3)).astype(np.float32)
    hi = (lo + rng.uniform(0, 2, (n, 3))).astype(np.float32)
    o = rng.uniform(-3, 3, (n, 3)).astype(np.float32)
    inside = rng.random(n) < 0.3
    o[inside] = ((lo + hi) / 2)[inside]
    on_face = rng.random(n) < 0.1
    o[on_face, 0] = lo[on_face, 0]
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d[rng.random(n) < 0.1, 1] = 0.0
    d[rng.random(n) < 0.05, 2] = -0.0
    d[rng.random(n) < 0.01, 0] = np.nan
    tmax = rng.choice(np.array([np.inf, 0.0, 1.5, 100.0, -1.0, np.nan], np.float32), n).astype(np.float32)
    case = np.zeros((n, 16), np.float32)
    case[:, 0:3], case[:, 3:6], case[:, 6:9], case[:, 9:12], case[:, 12] = lo, hi, o, d, tmax
    got = pb.selftest_device(3, case, n)
    exp = np.array([po.bbox_hits("orc", np.concatenate([lo[i], hi[i]]), o[i], d[i], float(tmax[i])) for i in range(n)])
    assert (got.astype(bool) == exp).all(), np.nonzero(got.astype(bool) != exp)[0][:10]


def test_box_test_on_device_keeps_subnormals(cuda_device):
    """The min/max box test of finite rays (packed f32x2 slab products on the device) on boxes,
    origins and far bounds of subnormal size, where flushing a difference or a product to zero
    would change the answer (it would on 86 % of these cases); unit directions aimed near each
    box, so about one case in seven hits."""
    rng = np.random.default_rng(23)
    n = 20000
    tiny = np.float32(1e-39)  # below FLT_MIN (1.18e-38)
    lo = (rng.uniform(-2, 1, (n, 3)) * tiny).astype(np.float32)
    hi = (lo + rng.uniform(0, 2, (n, 3)).astype(np.float32) * tiny).astype(np.float32)
    o = (rng.uniform(-3, 3, (n, 3)) * tiny).astype(np.float32)
    aim = ((lo + hi) / 2 - o).astype(np.float64) + rng.normal(size=(n, 3)) * 1e-39
    d = (aim / np.linalg.norm(aim, axis=1)[:, None]).astype(np.float32)
    d[d == 0] = np.float32(1e-20)
    tmax = rng.choice(np.array([np.inf, 1e-39, 5e-40, 1e-30, 1.0], np.float32), n).astype(np.float32)
    case = np.zeros((n, 16), np.float32)
    case[:, 0:3], case[:, 3:6], case[:, 6:9], case[:, 9:12], case[:, 12] = lo, hi, o, d, tmax
    assert (np.abs(case[:, 0:9]) < 1.18e-38).mean() > 0.9
    got = pb.selftest_device(3, case, n)
    exp = np.array([po.bbox_hits("orc", np.concatenate([lo[i], hi[i]]), o[i], d[i], float(tmax[i])) for i in range(n)])
    assert 0.05 < exp.mean() < 0.95, exp.mean()
    assert (got.astype(bool) == exp).all(), np.nonzero(got.astype(bool) != exp)[0][:10]


def test_small_scene_random_rays_match_fixture_and_oracle(cuda_device):
    g = load_golden("small_scene.npz")
    meshes, env = W.small_scene()
    scene = pb.Scene(meshes, env)
    rays = g["rays"]
    hits, nt, tt = scene.intersect(rays, counts=True)
    compare(hits, g["hits"], rays, "fixture")
    c = rays["flags"] == 0
    assert_bit_equal(nt[c], g["node_tests"][c], "node tests")
    assert_bit_equal(tt[c], g["tri_tests"][c], "tri tests")
    # any-hit rays stop early: their counts match the oracle's early-exit traversal
    o = po.OracleScene(meshes, env)
    oh, ont, ott = o.trace(rays, counts=True)
    assert_bit_equal(hits["prim"], oh["prim"], "prims incl. first any-hit")
    assert_bit_equal(nt, ont, "all node tests")
    assert_bit_equal(tt, ott, "all tri tests")


def test_microbench_prefix_matches_reference_fixture(cuda_device):
    g = load_golden("microbench.npz")
    mm, rays = W.microbench(n_rays=65536)
    scene = pb.Scene(mm)
    hits, nt, tt = scene.intersect(rays, counts=True)
    compare(hits, g["hits"], rays, "microbench")
    c = rays["flags"] == 0
    assert_bit_equal(nt[c], g["node_tests"][c], "nodes")
    assert_bit_equal(tt[c], g["tri_tests"][c], "tris")


def test_microbench_full_size_matches_oracle(cuda_device):
    """All 16,777,216 rays of the microbench against the CPU oracle (multi-threaded)."""
    mm, rays = W.microbench()
    scene = pb.Scene(mm)
    hits = scene.intersect(rays)
    o = po.OracleScene(mm)
    oh = o.trace(rays)
    compare(hits, oh, rays, "full microbench")
    assert_bit_equal(hits["prim"], oh["prim"], "first accepted any-hit prims")
    hit_rate = (hits["prim"][0::2] != pb.PRIM_NONE).mean()
    assert 0.5 < hit_rate <= 1.0
    # t error of the closest hits against an FP64 recomputation of the same Wald hit point
    tri = o.world_triangles()
    sel = np.nonzero((hits["prim"] != pb.PRIM_NONE) & (rays["flags"] == 0))[0][:200000]
    v = tri[hits["prim"][sel]].astype(np.float64)
    org, d = rays["org"][sel].astype(np.float64), rays["dir"][sel].astype(np.float64)
    n = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
    t64 = ((v[:, 0] - org) * n).sum(1) / (d * n).sum(1)
    rel = np.abs(hits["t"][sel] - t64) / np.abs(t64)
    assert rel.max() < 1e-5, rel.max()


def test_device_pointer_path_and_host_paths_agree(cuda_device):
    import torch
    meshes, env = W.small_scene()
    scene = pb.Scene(meshes, env)
    rays = random_rays(300_000, 11, -4, 4, anyhit_tmax=2.0)
    host = scene.intersect(rays)
    # pinned host buffers
    pr = torch.from_numpy(rays.view(np.uint8)).pin_memory()
    ph = torch.zeros(len(rays) * 16, dtype=torch.uint8).pin_memory()
    pb.check(pb.lib.pt_trace(scene.handle, pr.data_ptr(), len(rays), ph.data_ptr(), 0, None))
    assert ph.numpy().tobytes() == host.tobytes()
    # device buffers, asynchronous on a torch stream
    dr = torch.from_numpy(rays.view(np.uint8)).to(cuda_device)
    dh = torch.zeros(len(rays) * 16, dtype=torch.uint8, device=cuda_device)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        pb.check(pb.lib.pt_trace(scene.handle, dr.data_ptr(), len(rays), dh.data_ptr(), pb.MEM_DEVICE, s.cuda_stream))
    s.synchronize()
    assert dh.cpu().numpy().tobytes() == host.tobytes()


def test_edge_cases(cuda_device):
    # one triangle: both windings, axis-aligned rays (infinite inverse), rays on edges and
    # vertices (the FP64 edge fallback), tmax = 0, rays starting inside boxes, zero-length queries
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1]], np.float32)
    m = pb.Mesh(v[:, 0], v[:, 1], v[:, 2], [[0, 1, 2], [0, 2, 1], [1, 3, 4], [0, 3, 1]])
    scene = pb.Scene([m])
    cases = []
    for o, d in [((0.25, 0.25, 5), (0, 0, -1)), ((0.25, 0.25, -5), (0, 0, 1)), ((0.5, 0, 5), (0, 0, -1)),
                 ((0, 0, 5), (0, 0, -1)), ((0.5, 0.5, 5), (0, 0, -1)), ((1, 0, 5), (0, 0, -1)),
                 ((0.3, 0.3, 0.1), (0, 0, -1)), ((0.2, 0.2, 0.2), (1, 0, 0)), ((-1, 0.5, 0.5), (1, 0, 0)),
                 ((0.5, 0.5, 0.5), (0, 1, 0)), ((0.25, 0.25, 5), (0, 0, 1)), ((2, 2, 2), (-1, -1, -1))]:
        for tmax in (np.inf, 0.0, 4.9999, 5.0):
            for flags in (0, 1):
                cases.append((o, d, tmax, flags))
    rays = np.zeros(len(cases), pb.RAY_DTYPE)
    for i, (o, d, tmax, flags) in enumerate(cases):
        rays[i] = (o, tmax, d, flags)
    hits, nt, tt = scene.intersect(rays, counts=True)
    oh, ont, ott = po.OracleScene([m]).trace(rays, counts=True)
    for f in ("prim", "t", "u", "v"):
        assert_bit_equal(hits[f], oh[f], f)
    assert_bit_equal(nt, ont, "nodes")
    assert_bit_equal(tt, ott, "tris")
    assert (hits["prim"] != pb.PRIM_NONE).any()
    empty = np.zeros(0, pb.RAY_DTYPE)
    assert len(scene.intersect(empty)) == 0


def test_reference_built_tree_passthrough(cuda_device):
    """The drop-in path: the caller hands over the tree its own bvh::compact() produced."""
    meshes, env = W.small_scene()
    nodes, pairs = pb.bvh_build(meshes)
    a = pb.Scene(meshes, env)
    b = pb.Scene(meshes, env, nodes=nodes, leaf_pairs=pairs)
    rays = random_rays(50_000, 4, -4, 4, anyhit_tmax=3.0)
    assert a.intersect(rays).tobytes() == b.intersect(rays).tobytes()
    bad = nodes.copy()
    bad["offset"][0] = len(nodes) + 5
    with pytest.raises(pb.PolytopeError) as e:
        pb.Scene(meshes, env, nodes=bad, leaf_pairs=pairs)
    assert e.value.code == pb.PT_EINVAL


def test_device_intersect_takes_counts_from_byte_sizes(cuda_device):
    """Device buffers of any element type: the ray count is bytes / 32, and a hits buffer too small
    for it is refused before anything reaches the GPU."""
    import torch
    meshes, rays = W.microbench(n_rays=4096, level=4)
    scene = pb.Scene(meshes)
    exp = scene.intersect(rays)
    as_bytes = torch.from_numpy(rays.view(np.uint8)).cuda()
    as_float = torch.from_numpy(rays.view(np.float32)).cuda()
    for dr in (as_bytes, as_float):
        hits = torch.zeros(len(rays) * 16, dtype=torch.uint8, device="cuda")
        scene.intersect(dr, hits, device=True)
        torch.cuda.synchronize()
        assert hits.cpu().numpy().tobytes() == exp.tobytes()
    with pytest.raises(ValueError):
        scene.intersect(as_bytes, torch.zeros(len(rays) * 16 - 1, dtype=torch.uint8, device="cuda"), device=True)
    with pytest.raises(ValueError):
        scene.intersect(as_bytes[:-4], torch.zeros(len(rays) * 16, dtype=torch.uint8, device="cuda"), device=True)



def test_coincident_faces_that_raise_min_t(cuda_device):
    """Every face twice, the copy with its vertices rotated: the copy's Wald t can round one ulp
    above the running MinT and still be accepted (the range check compares T with MinT * det
    before the division), so MinT rises during the walk and ties are decided by rounding.  Hits
    and per-ray test counts must still equal the oracle's.  Rays aim at face interiors, so most
    meet such a pair."""
    x, y, z, f = pb.icosphere(4, 1.0, 0.05, 7)
    m = pb.Mesh(x, y, z, np.concatenate([f, f[:, [1, 2, 0]]]))
    scene = pb.Scene([m])
    rng = np.random.default_rng(9)
    n = 100_000
    fi = f[rng.integers(0, len(f), n)]
    w = rng.dirichlet([1, 1, 1], n).astype(np.float32)
    tgt = sum(w[:, k:k + 1] * np.stack([x[fi[:, k]], y[fi[:, k]], z[fi[:, k]]], 1) for k in range(3))
    o = rng.normal(size=(n, 3))
    o = 3 * o / np.linalg.norm(o, axis=1)[:, None]
    d = tgt - o
    rays = np.zeros(n, pb.RAY_DTYPE)
    rays["org"] = o
    rays["dir"] = d / np.linalg.norm(d, axis=1)[:, None]
    rays["tmax"] = np.inf
    rays["flags"][1::4] = 1
    rays["tmax"][1::4] = 3.5
    hits, nt, tt = scene.intersect(rays, counts=True)
    oh, ont, ott = po.OracleScene([m]).trace(rays, counts=True)
    for fld in ("prim", "t", "u", "v"):
        assert_bit_equal(hits[fld], oh[fld], fld)
    assert_bit_equal(nt, ont, "nodes")
    assert_bit_equal(tt, ott, "tris")
    plain = scene.intersect(rays)
    assert plain.tobytes() == hits.tobytes()
