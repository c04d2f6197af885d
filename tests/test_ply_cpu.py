"""Scene ingest: pt_load_ply against the arrays the test wrote and against the reference's own
ply_parser::parse_file (oracle/_ref, src/common/parsers/mesh_parsers.cpp) on generated PLY files
in every format the reference reads: ascii, binary little and big endian, with and without vertex
normals and uv, extra vertex properties, permuted property order, faces before vertices."""
import struct

import numpy as np
import pytest

import polytope_b200 as pb
from oracle import pyoracle as po

TYPES = {"float": "f", "int": "i", "uchar": "B", "double": "d"}


def write_ply(path, fmt, verts, faces, props, face_first=False, list_types=("uchar", "int")):
    """verts: dict name -> (N,) array; props: [(type, name)] in file order."""
    n, f = len(next(iter(verts.values()))), len(faces)
    head = ["ply", f"format {fmt} 1.0", "comment generated by the test"]
    vdecl = [f"element vertex {n}"] + [f"property {t} {nm}" for t, nm in props]
    fdecl = [f"element face {f}", f"property list {list_types[0]} {list_types[1]} vertex_indices"]
    head += (fdecl + vdecl) if face_first else (vdecl + fdecl)
    head.append("end_header")
    out = ("\n".join(head) + "\n").encode()
    if fmt == "ascii":
        vlines = "".join(" ".join(repr(float(verts[nm][i])) if t in ("float", "double") else str(int(verts[nm][i]))
                                  for t, nm in props) + " \n" for i in range(n))
        flines = "".join(f"3 {a} {b} {c} \n" for a, b, c in faces)
        body = (flines + vlines) if face_first else (vlines + flines)
        out += body.encode()
    else:
        e = "<" if fmt == "binary_little_endian" else ">"
        vbody = b"".join(b"".join(struct.pack(e + TYPES[t], verts[nm][i] if t in ("float", "double") else int(verts[nm][i]))
                                  for t, nm in props) for i in range(n))
        fbody = b"".join(struct.pack(e + TYPES[list_types[0]], 3) + struct.pack(e + TYPES[list_types[1]] * 3, *map(int, fc))
                         for fc in faces)
        out += (fbody + vbody) if face_first else (vbody + fbody)
    path.write_bytes(out)


def mesh_arrays(seed, n=50, f=70):
    rng = np.random.default_rng(seed)
    v = {k: rng.normal(size=n).astype(np.float32) for k in ("x", "y", "z", "nx", "ny", "nz", "u", "v", "confidence")}
    v["flags"] = rng.integers(0, 100, n)
    faces = rng.integers(0, n, (f, 3))
    return v, faces


CASES = [
    # (format, properties in file order, face_first)
    ("ascii", [("float", "x"), ("float", "y"), ("float", "z")], False),
    ("ascii", [("float", "x"), ("float", "z"), ("float", "y"), ("float", "confidence")], False),
    ("ascii", [("float", "x"), ("float", "y"), ("float", "z"), ("float", "nx"), ("float", "ny"), ("float", "nz"),
               ("int", "flags")], True),
    ("binary_little_endian", [("float", "x"), ("float", "y"), ("float", "z"), ("float", "nx"), ("float", "ny"),
                              ("float", "nz"), ("float", "u"), ("float", "v")], False),
    ("binary_big_endian", [("float", "x"), ("float", "y"), ("float", "z"), ("float", "nx"), ("float", "ny"),
                           ("float", "nz")], False),
]


def check_against_written(m, v, faces, props):
    names = [nm for _, nm in props]
    assert np.array_equal(m.x, v["x"]) and np.array_equal(m.y, v["y"]) and np.array_equal(m.z, v["z"])
    assert np.array_equal(m.faces, faces.astype(np.uint32))
    if "nx" in names:
        assert np.array_equal(m.normals, np.stack([v["nx"], v["ny"], v["nz"]], 1))
    else:
        assert m.normals is None
    if "u" in names:
        assert np.array_equal(m.uv, np.stack([v["u"], v["v"]], 1))


@pytest.mark.parametrize("k", range(len(CASES)))
def test_ply_matches_written_arrays_and_reference_parser(tmp_path, k):
    fmt, props, face_first = CASES[k]
    v, faces = mesh_arrays(k)
    path = tmp_path / f"mesh{k}.ply"
    write_ply(path, fmt, v, faces, props, face_first)
    m = pb.load_ply(path)
    check_against_written(m, v, faces, props)
    if not po.ref_available():
        pytest.skip("oracle/_ref not built")
    x, y, z, f, n = po.ref_load_ply(path)
    assert np.array_equal(m.x, x) and np.array_equal(m.y, y) and np.array_equal(m.z, z)
    assert np.array_equal(m.faces, f)
    if n is None:
        assert m.normals is None
    else:
        assert np.array_equal(m.normals, n)


def test_binary_without_normals_reads_each_vertex_once(tmp_path):
    """The reference's own test parse_ply.Binary (tests/parsers/test_ply_parser.cpp:110-133) expects
    one packed vertex per file vertex; the compiled reference appends each twice for binary files
    without normals (mesh_parsers.cpp:470-473).  The library follows the test."""
    v, faces = mesh_arrays(11, n=8, f=4)
    props = [("float", "x"), ("float", "y"), ("float", "z")]
    path = tmp_path / "floor.ply"
    write_ply(path, "binary_little_endian", v, faces, props)
    m = pb.load_ply(path)
    assert len(m.x) == 8
    check_against_written(m, v, faces, props)
    ascii_path = tmp_path / "floor_ascii.ply"
    write_ply(ascii_path, "ascii", v, faces, props)
    assert np.array_equal(pb.load_ply(ascii_path).x, m.x)
    if po.ref_available():
        x, _, _, f, _ = po.ref_load_ply(path)
        assert len(x) == 16 and np.array_equal(x[0::2], m.x) and np.array_equal(x[1::2], m.x)
        assert np.array_equal(f, m.faces)


def test_declared_binary_types_are_honoured(tmp_path):
    v, faces = mesh_arrays(5, n=20, f=10)
    props = [("double", "x"), ("double", "y"), ("double", "z"), ("uchar", "flags")]
    path = tmp_path / "typed.ply"
    write_ply(path, "binary_little_endian", v, faces, props, list_types=("uchar", "uchar") if faces.max() < 256 else ("uchar", "int"))
    m = pb.load_ply(path)
    assert np.array_equal(m.x, v["x"].astype(np.float64).astype(np.float32))
    assert np.array_equal(m.faces, faces.astype(np.uint32))


@pytest.mark.parametrize("bad", [
    "ply\nformat ascii 2.0\nend_header\n",
    "ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nproperty float y\nend_header\n0 0\n",
    "ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nproperty float y\nproperty float z\nproperty float nx\nend_header\n0 0 0 0\n",
    "ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\nproperty float z\n"
    "element face 1\nproperty list uchar int vertex_indices\nend_header\n0 0 0\n1 0 0\n0 1 0\n4 0 1 2 0\n",
    "ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nproperty float y\nproperty float z\n",
    "nope\n",
])
def test_malformed_files_are_rejected(tmp_path, bad):
    path = tmp_path / "bad.ply"
    path.write_text(bad)
    with pytest.raises(pb.PolytopeError) as e:
        pb.load_ply(path)
    assert e.value.code == pb.PT_EINVAL


def test_loaded_mesh_builds_the_same_tree(tmp_path):
    """An ingested mesh feeds the identical host SAH build."""
    v, faces = mesh_arrays(3, n=200, f=300)
    props = [("float", "x"), ("float", "y"), ("float", "z")]
    path = tmp_path / "tree.ply"
    write_ply(path, "binary_little_endian", v, faces, props)
    m = pb.load_ply(path)
    direct = pb.Mesh(v["x"], v["y"], v["z"], faces)
    a, b = pb.bvh_build([m]), pb.bvh_build([direct])
    assert all(np.array_equal(p, q) for p, q in zip(a, b))
