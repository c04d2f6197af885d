"""Host-side product code without a GPU: the C-ABI library's exports, error paths, the identical
BVH build, the exact-arithmetic helpers and the generators."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, assert_bit_equal, load_golden
import polytope_b200 as pb
from polytope_b200 import workloads as W
from oracle import pyoracle as po
from golden.make_golden import scene_inputs_digest, sha


def header_symbols():
    text = open(os.path.join(ROOT, "include", "polytope_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pt_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    syms = header_symbols()
    assert len(syms) >= 10
    lib = C.CDLL(pb.LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_no_gpu_error_path():
    assert "sm_100a" in pb.version()
    import torch
    if torch.cuda.is_available():
        pytest.skip("this checks the no-device error path")
    x, y, z, f = pb.icosphere(1)
    with pytest.raises(pb.PolytopeError) as e:
        pb.Scene([pb.Mesh(x, y, z, f)])
    assert e.value.code == pb.PT_ECUDA and "no CUDA device" in str(e.value)


def test_invalid_arguments():
    lib = pb.lib
    assert lib.pt_scene_create(None, None) == pb.PT_EINVAL
    assert lib.pt_trace(None, None, 1, None, 0, None) == pb.PT_EINVAL
    assert "NULL" in pb.last_error()
    n = C.c_uint32(0)
    assert lib.pt_bvh_build(None, 0, 0, None, C.byref(n), None) == pb.PT_EINVAL
    # vertex index out of range
    bad = pb.Mesh([0, 1, 0], [0, 0, 1], [0, 0, 0], [[0, 1, 5]])
    with pytest.raises(pb.PolytopeError) as e:
        pb.bvh_build([bad])
    assert e.value.code == pb.PT_EINVAL and "out of range" in str(e.value)
    # no faces at all: the reference's bound() is undefined there, the library refuses
    empty = pb.Mesh([0.0], [0.0], [0.0], np.zeros((0, 3), np.uint32))
    with pytest.raises(pb.PolytopeError):
        pb.bvh_build([empty])
    # server configuration is checked before any device call
    cfg = pb.ServerConfig()
    cfg.max_inflight, cfg.tuning, cfg.policy = 4, pb.default_tuning(), 7
    h = C.c_void_p()
    assert lib.pt_server_create(C.byref(cfg), C.byref(h)) == pb.PT_EINVAL and "policy" in pb.last_error()
    cfg.policy, cfg.max_inflight = pb.SERVE_FAIR_SHARE, 0
    assert lib.pt_server_create(C.byref(cfg), C.byref(h)) == pb.PT_EINVAL


def soup(seed, meshes=3, faces=2000):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(meshes):
        c = rng.uniform(-3, 3, (faces, 3)).astype(np.float32)
        v = (c[:, None, :] + rng.normal(0, 0.2, (faces, 3, 3))).astype(np.float32).reshape(-1, 3)
        M = np.eye(4, dtype=np.float32)
        M[:3, 3] = rng.uniform(-1, 1, 3)
        M[1, 2] = 0.3 * k
        out.append(pb.Mesh(v[:, 0], v[:, 1], v[:, 2], np.arange(3 * faces, dtype=np.uint32).reshape(-1, 3), object_to_world=M))
    # degenerate leaf: many copies of one triangle (same centroid: stop case 3)
    v = np.tile(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), (37, 1))
    out.append(pb.Mesh(v[:, 0], v[:, 1], v[:, 2], np.arange(111, dtype=np.uint32).reshape(-1, 3)))
    # zero-area faces (all at one point: stop case 2)
    z = np.zeros(30, np.float32)
    out.append(pb.Mesh(z + 5, z + 5, z + 5, np.arange(30, dtype=np.uint32).reshape(-1, 3)))
    return out


@pytest.mark.parametrize("threads", [1, 0, 3, 32])
def test_bvh_build_identical_to_oracle(threads):
    for meshes in (W.small_scene()[0], soup(1), soup(2, meshes=1, faces=1)):
        nodes, pairs = pb.bvh_build(meshes, threads=threads)
        o = po.OracleScene(meshes)
        on, op = o.tree()
        assert nodes.tobytes() == on.tobytes()
        assert (pairs == op).all()


def coincident_soup(seed=0):
    """Two meshes whose many degenerate faces share one centroid: leaves of more than 16 faces that
    mix meshes, where the reference's std::sort with its leaf comparator is undefined."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(3000, 3)).astype(np.float32)
    v[::7] = 0.0
    v[1::11] *= -0.0
    return [pb.Mesh(v[:, 0], v[:, 1], v[:, 2], rng.integers(0, 3000, (20000, 3))),
            pb.Mesh(v[:, 0], v[:, 1], v[:, 2], rng.integers(0, 3000, (500, 3)),
                    object_to_world=np.diag([1, -1, 1, 1]).astype(np.float32))]


@pytest.mark.parametrize("threads", [1, 0])
def test_long_mixed_leaves_build_safely_and_match_the_oracle(threads):
    meshes = coincident_soup()
    nodes, pairs = pb.bvh_build(meshes, threads=threads)
    big = nodes[nodes["num_faces"] > 16]
    assert len(big) > 0
    mixed = 0
    for nd in big:
        leaf = pairs[nd["offset"]:nd["offset"] + nd["num_faces"]]
        if len(set(leaf[:, 0])) > 1:  # the defined order: by (mesh, face)
            mixed += 1
            assert [tuple(p) for p in leaf] == sorted(tuple(p) for p in leaf)
    assert mixed > 0
    on, op = po.OracleScene(meshes).tree()
    assert nodes.tobytes() == on.tobytes() and (pairs == op).all()


def test_parallel_build_is_deterministic():
    """The parallel phases (baking, face boxes, subtree tasks, compaction) give the same bytes on
    every run and for every thread count."""
    meshes = W.instanced_scene(level=5)[0]
    ref_nodes, ref_pairs = pb.bvh_build(meshes, threads=1)
    for threads in (0, 2, 5, 16, 0, 16):
        nodes, pairs = pb.bvh_build(meshes, threads=threads)
        assert nodes.tobytes() == ref_nodes.tobytes() and pairs.tobytes() == ref_pairs.tobytes()


def test_leaf_beyond_the_record_limit_is_refused():
    z = np.zeros(3, np.float32)
    m = pb.Mesh(z, z, z, np.zeros((70000, 3), np.uint32))  # 70,000 copies of one point-face
    with pytest.raises(pb.PolytopeError) as e:
        pb.bvh_build([m])
    assert e.value.code == pb.PT_EINVAL and "65535" in str(e.value)


def test_bvh_build_matches_reference_fixtures():
    g = load_golden("small_scene.npz")
    meshes, _ = W.small_scene()
    nodes, pairs = pb.bvh_build(meshes)
    assert sha(nodes, pairs) == str(g["tree_sha"])
    g2 = load_golden("instanced_small.npz")
    im, _ = W.instanced_scene(level=4)
    n2, p2 = pb.bvh_build(im)
    assert sha(n2, p2) == str(g2["tree_sha"])


def test_bvh_build_microbench_tree_matches_reference():
    g = load_golden("microbench.npz")
    mm, _ = W.microbench(n_rays=1)
    nodes, pairs = pb.bvh_build(mm)
    assert len(nodes) == int(g["num_nodes"])
    assert sha(nodes, pairs) == str(g["tree_sha"])


def test_generators_match_fixture_inputs():
    g = load_golden("microbench.npz")
    mm, rays = W.microbench(n_rays=65536)
    assert scene_inputs_digest(mm) == str(g["inputs_sha"]) and sha(rays) == str(g["rays_sha"])
    x, y, z, f = pb.icosphere(3)
    assert len(x) == 10 * 4 ** 3 + 2 and len(f) == 20 * 4 ** 3
    v = np.stack([x, y, z], 1).astype(np.float64)
    n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 1]])
    c = v[f].mean(axis=1)
    assert ((n * c).sum(1) > 0).all()  # outward winding
    assert np.allclose(np.linalg.norm(v, axis=1), 1.0, atol=1e-6)
    r = rays
    assert np.allclose(np.linalg.norm(r["org"], axis=1), 3.0, atol=1e-5)
    assert np.allclose(np.linalg.norm(r["dir"], axis=1), 1.0, atol=1e-6)
    assert (r["flags"][1::2] == 1).all() and np.isinf(r["tmax"][0::2]).all() and (r["tmax"][1::2] > 1.9).all()


def test_gamma_constants_match_host_folding():
    # bit patterns hard-coded in exact_math.h against the host compiler's constant folding
    lib = po.oracle_lib()
    exp = {2: 0x34000001, 3: 0x34400002, 5: 0x34A00003, 7: 0x34E00006, 0: 0x3F800003}
    for n, b in exp.items():
        assert np.float32(lib.orc_gamma(n)).view(np.uint32) == b, n
    src = open(os.path.join(ROOT, "polytope_b200", "csrc", "exact_math.h")).read()
    for name, b in (("GAMMA2", 0x34000001), ("GAMMA3", 0x34400002), ("GAMMA5", 0x34A00003), ("GAMMA7", 0x34E00006),
                    ("GAMMA_MUL", 0x3F800003)):
        assert re.search(rf"PT_{name}_BITS 0x{b:08X}u", src), name


def f64_cases(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    # general random magnitudes
    e = rng.integers(-60, 60, (n, 4))
    m = rng.uniform(1, 2, (n, 4)) * rng.choice([-1, 1], (n, 4))
    out.append((m * 2.0 ** e).astype(np.float32))
    # near cancellation: a*b ~= c*d
    a = rng.uniform(-4, 4, n).astype(np.float32)
    b = rng.uniform(-4, 4, n).astype(np.float32)
    c = (a * (1 + rng.normal(0, 1e-6, n))).astype(np.float32)
    d = (b * (1 + rng.normal(0, 1e-6, n))).astype(np.float32)
    out.append(np.stack([a, b, c, d], 1))
    out.append(np.stack([a, b, a, b], 1))  # exact cancellation
    out.append(np.stack([a, b, b, a], 1))
    # subnormal / huge ranges and wide exponent gaps
    e = rng.integers(-149, 127, (n, 4))
    m = rng.uniform(1, 2, (n, 4)) * rng.choice([-1, 1], (n, 4))
    out.append(np.clip(m * 2.0 ** e, -3e38, 3e38).astype(np.float32))
    sub = (rng.integers(1, 1 << 23, (n, 4)) * rng.choice([-1, 1], (n, 4))).astype(np.int64)
    out.append(np.where(sub < 0, (-sub) | (1 << 31), sub).astype(np.uint32).view(np.float32).reshape(n, 4))
    # zeros with signs
    z = np.array([[0.0, 1.0, 0.0, 1.0], [-0.0, 1.0, 0.0, 1.0], [0.0, -1.0, 0.0, 1.0], [-0.0, 1.0, -0.0, -1.0],
                  [0.0, 0.0, 2.0, 3.0], [2.0, 3.0, 0.0, -0.0], [1e-30, 1e-30, 0.0, 0.0]], np.float32)
    out.append(z)
    return np.concatenate(out)


def f64_reference(q):
    q = q.astype(np.float64)
    with np.errstate(over="ignore", invalid="ignore"):
        return (q[:, 0] * q[:, 1] - q[:, 2] * q[:, 3]).astype(np.float32)


def test_f64_emulation_host_matches_double():
    q = f64_cases(20000, 1)
    lib = pb.lib
    got = np.array([lib.pt_host_f64_diff_emulated(*map(float, row)) for row in q], np.float32)
    exp = f64_reference(q)
    ok = np.isnan(exp)
    assert_bit_equal(got[~ok], exp[~ok], "f64 emulation")
    # the oracle's real-double version agrees too
    o = np.array([po.f64_diff(*map(float, row)) for row in q[:2000]], np.float32)
    assert_bit_equal(o, exp[:2000], "oracle double")


def test_f64_emulation_double_rounding_ties():
    # values where rounding to double then to float differs from a single rounding
    rng = np.random.default_rng(3)
    rows = []
    for _ in range(4000):
        a = np.float32(rng.uniform(1, 2))
        b = np.float32(rng.uniform(1, 2))
        p = np.float64(a) * np.float64(b)
        # c*d chosen so that the exact difference is just off a float midpoint
        c = np.float32(rng.uniform(1, 2)) * np.float32(2.0 ** -rng.integers(20, 40))
        d = np.float32(rng.uniform(1, 2))
        rows.append([a, b, c, d])
    q = np.array(rows, np.float32)
    got = np.array([pb.f64_diff_emulated_host(*map(float, r)) for r in q], np.float32)
    assert_bit_equal(got, f64_reference(q), "double rounding")


def _read_png(path):
    """Minimal PNG reader for the test: chunks with CRC check, zlib inflate, filter-0 scanlines."""
    import struct
    import zlib
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, chunks = 8, []
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        typ, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]
        assert zlib.crc32(typ + body) & 0xFFFFFFFF == crc
        chunks.append((typ, body))
        pos += 12 + n
    assert [c[0] for c in chunks] == [b"IHDR", b"IDAT", b"IEND"]
    w, h, depth, ctype = struct.unpack(">IIBB", chunks[0][1][:10])
    assert (depth, ctype) == (8, 6)
    raw = zlib.decompress(chunks[1][1])
    rows = np.frombuffer(raw, np.uint8).reshape(h, 1 + 4 * w)
    assert (rows[:, 0] == 0).all()
    return rows[:, 1:].reshape(h, w, 4)


@pytest.mark.parametrize("w,h", [(1, 1), (37, 5), (300, 250)])
def test_png_writer_round_trip(tmp_path, w, h):
    rng = np.random.default_rng(w * 7 + h)
    rgba = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    path = tmp_path / "film.png"
    pb.write_png(path, rgba)
    assert np.array_equal(_read_png(path), rgba)


def test_png_quantisation_oracle_known_answers():
    # PNGFilm::Output: clamp at 255, truncate toward zero, alpha 255
    rgb = np.array([[[0.0, 0.5, 254.99], [255.0, 300.0, 1e9], [1.0, 127.9999, 128.0]]], np.float32)
    exp = np.array([[[0, 0, 254, 255], [255, 255, 255, 255], [1, 127, 128, 255]]], np.uint8)
    assert np.array_equal(po.film_to_rgba8(rgb), exp)


def test_nan_inf_and_signed_zero_geometry_builds_deterministically():
    """Faces with NaN or infinite coordinates (which the reference's bucket index cannot handle:
    its unsigned conversion of a NaN is undefined) and coordinates of both zero signs: the build
    stays in bounds, gives the same bytes for every thread count, and lists every face once."""
    rng = np.random.default_rng(11)
    nf = 150_000
    v = rng.normal(size=(3 * nf, 3)).astype(np.float32)
    v[rng.integers(0, len(v), 200), rng.integers(0, 3, 200)] = np.nan
    v[rng.integers(0, len(v), 50), rng.integers(0, 3, 50)] = np.inf
    v[rng.integers(0, len(v), 50), rng.integers(0, 3, 50)] = -np.inf
    z = rng.integers(0, len(v), 5000)
    v[z, rng.integers(0, 3, 5000)] = np.where(rng.random(5000) < 0.5, np.float32(0.0), np.float32(-0.0))
    meshes = [pb.Mesh(v[:, 0], v[:, 1], v[:, 2], np.arange(3 * nf, dtype=np.uint32).reshape(-1, 3)),
              pb.Mesh(v[::-1, 0].copy(), v[::-1, 1].copy(), v[::-1, 2].copy(),
                      np.arange(3 * nf, dtype=np.uint32).reshape(-1, 3)[:40_000])]
    ref_nodes, ref_pairs = pb.bvh_build(meshes, threads=1)
    for threads in (0, 3, 16):
        nodes, pairs = pb.bvh_build(meshes, threads=threads)
        assert nodes.tobytes() == ref_nodes.tobytes() and pairs.tobytes() == ref_pairs.tobytes()
    ids = ref_pairs[:, 0].astype(np.int64) * (1 << 32) + ref_pairs[:, 1]
    assert len(np.unique(ids)) == nf + 40_000
    leaves = ref_nodes[ref_nodes["num_faces"] > 0]
    assert int(leaves["num_faces"].sum()) == nf + 40_000


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref is only built where the reference tree is present")
@pytest.mark.parametrize("w,h", [(1, 1), (37, 5), (160, 120)])
def test_png_output_matches_the_reference_film_output(tmp_path, w, h):
    """The output step against the reference's own: a float film written by PNGFilm::Output
    (BoxFilter of one sample per pixel, clamp and truncation, lodepng encoding) and the same film
    quantised by the restatement and written by pt_write_png decode, with the reference's lodepng,
    to the same RGBA8 pixels (the GPU tests pin pt_film_to_rgba8 to the restatement)."""
    rng = np.random.default_rng(w * 31 + h)
    rgb = rng.uniform(0, 400, (h, w, 3)).astype(np.float32)  # films are >= 0 (negative casts are undefined in C++)
    rgb[0, 0] = (255.0, 254.99998, 0.0)
    po.ref_png_film(rgb, tmp_path / "ref.png")
    pb.write_png(tmp_path / "ours.png", po.film_to_rgba8(rgb))
    want = po.ref_png_decode(tmp_path / "ref.png")
    got = po.ref_png_decode(tmp_path / "ours.png")
    assert want.shape == (h, w, 4) and np.array_equal(got, want)
