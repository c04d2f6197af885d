"""Scene ingest: pt_load_obj against the reference's own obj_parser::parse_file (oracle/_ref,
src/common/parsers/mesh_parsers.cpp:547-598) on generated OBJ files, including the lines the
reference reads in its own way (vn / vt lines as vertices, polygons cut to their first three
corners, "v/vt/vn" index triples, short lines), and an objmesh shape in a PBRT scene."""
import numpy as np
import pytest

import polytope_b200 as pb
from oracle import pyoracle as po
from test_pbrt_cpu import assert_same_as_reference, write_assets


def write_obj(path, seed=0):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(40, 3)).astype(np.float32)
    lines = ["# generated", "o thing", "g group"]
    for i, p in enumerate(v):
        lines.append("v " + " ".join(repr(float(c)) for c in p))
        if i % 9 == 0:
            lines.append("vn 0 0 1")  # read as a vertex by the reference too
        if i % 13 == 0:
            lines.append("vt 0.5 0.25")  # short line: the last word is read again
    n = len(v) + len(range(0, 40, 9)) + len(range(0, 40, 13))
    for k in range(60):
        a, b, c, d = rng.integers(1, n + 1, 4)
        style = k % 4
        if style == 0:
            lines.append(f"f {a} {b} {c}")
        elif style == 1:
            lines.append(f"f {a}/{b} {b}/{c} {c}/{a}")
        elif style == 2:
            lines.append(f"f {a}/1/2 {b}//3 {c}/4/5 {d}/6/7")  # a quad: first three corners only
        else:
            lines.append(f"f  {a}\t{b}   {c}   # trailing comment")
    lines.append("s off")
    lines.append("usemtl nothing")
    path.write_text("\n".join(lines) + "\n")


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_obj_matches_reference_parser(tmp_path, seed):
    path = tmp_path / f"m{seed}.obj"
    write_obj(path, seed)
    m = pb.load_obj(path)
    assert len(m.x) > 40 and len(m.faces) == 60
    if not po.ref_available():
        pytest.skip("oracle/_ref not built")
    x, y, z, f = po.ref_load_obj(path)
    assert np.array_equal(m.x, x) and np.array_equal(m.y, y) and np.array_equal(m.z, z)
    assert np.array_equal(m.faces, f)


@pytest.mark.parametrize("text,why", [
    ("v 1 2 3\nv 1 2 3\nv 1 2 3\nf 1 2 4\n", "does not exist"),
    ("v 1 2 3\nv 1 2 3\nv 1 2 3\nf 0 1 2\n", "does not exist"),
    ("v 1 x 3\n", "not a number"),
    ("v 1 2 3\nf a b c\n", "not an index"),
])
def test_malformed_obj_is_rejected(tmp_path, text, why):
    path = tmp_path / "bad.obj"
    path.write_text(text)
    with pytest.raises(pb.PolytopeError) as e:
        pb.load_obj(path)
    assert e.value.code == pb.PT_EINVAL and why in str(e.value)


def test_objmesh_in_pbrt_scene_matches_reference(tmp_path):
    write_assets(tmp_path)
    write_obj(tmp_path / "thing.obj", 4)
    (tmp_path / "s.pbrt").write_text(
        'LookAt 0 2 9 0 0 0 0 1 0\nCamera "perspective" "float fov" [ 40 ]\nWorldBegin\n'
        'Material "matte" "rgb Kd" [ .5 .6 .7 ]\n'
        'AttributeBegin\n  Translate 0 1 0\n  Shape "objmesh" "string filename" [ "thing.obj" ]\nAttributeEnd\n'
        'ObjectBegin "both"\n  Shape "objmesh" "string filename" [ "thing.obj" ]\n'
        '  Shape "plymesh" "string filename" [ "quad.ply" ]\nObjectEnd\n'
        'Translate 2 0 0\nObjectInstance "both"\nWorldEnd\n')
    s = pb.load_pbrt(tmp_path / "s.pbrt")
    assert len(s.meshes) == 2
    if not po.ref_available():
        pytest.skip("oracle/_ref not built")
    assert_same_as_reference(s, po.ref_load_pbrt(tmp_path / "s.pbrt"))
