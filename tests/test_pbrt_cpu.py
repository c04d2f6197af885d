"""Scene ingest: pt_load_pbrt against the reference's own pbrt_parser::parse_file (oracle/_ref,
src/common/parsers/pbrt_parser.cpp) -- render settings, camera, and per shape the packed geometry,
object-to-world and world-to-object matrices, material and radiance, all bit for bit -- on
generated scenes that exercise the reference's scoping rules (a scope's transform and area light
updated in place after shapes use them, ObjectBegin / ObjectInstance, named materials, UV spheres,
Rotate) and on the reference's own example scenes when its tree is present."""
import os

import numpy as np
import pytest

from conftest import reference_path

import polytope_b200 as pb
from oracle import pyoracle as po
from test_ply_cpu import write_ply

REF_SCENES = reference_path("scenes")
# example scenes of the reference that it parses and whose geometry files it ships
MATCHING = ["bunny/bunny.pbrt", "bvh-test/bvh-test.pbrt", "lighttest/lighttest.pbrt", "minimum.pbrt",
            "minimum-emptyworld.pbrt", "teapot/teapot.pbrt", "test/cuda/bvh-traversal.pbrt",
            "triangle-one/triangle-one.pbrt", "two-balls.pbrt"]

SCENE = """Integrator "path" "integer maxdepth" [ 6 ]
LookAt 1 2 8   0 0.5 0   0 1 0 # eye, target, up
Sampler "halton" "integer pixelsamples" [ 4 ]
PixelFilter "box" "float xwidth" [ 1 ] "float ywidth" [ 1 ]
Film "image" "integer xresolution" [ 96 ] "integer yresolution" [ 72 ] "string filename" [ "out.png" ]
Camera "perspective" "float fov" [ 40 ]
WorldBegin
  LightSource "infinite" "rgb L" [ .1 .12 .15 ]
  AttributeBegin
    AreaLightSource "diffuse" "rgb L" [ 4 4 3.5 ]
    Translate 0 4 0
    Shape "plymesh" "string filename" [ "quad.ply" ]
    AreaLightSource "diffuse" "rgb L" [ 5 5 5 ]
    Rotate 15 0 0 1
    Shape "plymesh" "string filename" [ "quad.ply" ]
  AttributeEnd
  Material "matte" "rgb Kd" [ .6 .5 .4 ]
  AttributeBegin
    Translate -1.5 1 0
    Rotate 30 1 1 0
    Scale 0.8 0.7 0.8
    Shape "plymesh" "string filename" [ "blob.ply" ]
  AttributeEnd
  AttributeBegin
    Material "mirror" "color Kr" [ .9 .85 .8 ]
    Translate 1.5 1 0
    Shape "sphere" "float radius" [ 0.7 ]
    TransformBegin
      Translate 0 1.2 0.5
      Shape "sphere" "float radius" [ 24 ]
    TransformEnd
  AttributeEnd
  MakeNamedMaterial "grey" "string type" [ "matte" ] "rgb Kd" [ .9 .1 .1 ]
  NamedMaterial "grey"
  ObjectBegin "blobs"
    Shape "plymesh" "string filename" [ "blob.ply" ]
  ObjectEnd
  AttributeBegin
    Translate 0 0.5 -2
    ObjectInstance "blobs"
    Translate 0 0 -2
    ObjectInstance "blobs"
  AttributeEnd
  Shape "plymesh" "string filename" [ "ground.ply" ]
WorldEnd
"""


def write_assets(d):
    """quad.ply (ascii light quad), blob.ply (binary little endian with normals), ground.ply (ascii)."""
    quad = {"x": np.float32([-0.5, 0.5, 0.5, -0.5]), "y": np.zeros(4, np.float32), "z": np.float32([-0.5, -0.5, 0.5, 0.5])}
    write_ply(d / "quad.ply", "ascii", quad, np.array([[0, 2, 1], [0, 3, 2]]), [("float", k) for k in "xyz"])
    x, y, z, f = pb.icosphere(2, 0.5, 0.05, 3)
    n = np.stack([x, y, z], 1)
    n = (n / np.linalg.norm(n, axis=1)[:, None]).astype(np.float32)
    blob = {"x": x, "y": y, "z": z, "nx": n[:, 0], "ny": n[:, 1], "nz": n[:, 2]}
    write_ply(d / "blob.ply", "binary_little_endian", blob, f, [("float", k) for k in ("x", "y", "z", "nx", "ny", "nz")])
    g = {"x": np.float32([-6, 6, 6, -6]), "y": np.zeros(4, np.float32), "z": np.float32([-6, -6, 6, 6])}
    write_ply(d / "ground.ply", "ascii", g, np.array([[0, 1, 2], [0, 2, 3]]), [("float", k) for k in "xyz"])


def write_scene(d, text=SCENE):
    write_assets(d)
    (d / "scene.pbrt").write_text(text)
    return d / "scene.pbrt"


def assert_same_as_reference(s, r):
    assert (s.width, s.height, s.spp, s.max_depth) == (r["width"], r["height"], r["spp"], r["max_depth"])
    assert np.float32(s.camera["fov"]) == np.float32(r["fov"])
    if np.array_equal(r["camera_to_world"], np.eye(4, dtype=np.float32)):
        assert s.camera["eye"] == (0, 0, 0) and s.camera["look_at"] == (0, 0, 1) and s.camera["up"] == (0, 1, 0)
    else:
        for k in ("eye", "look_at", "up"):
            assert np.array_equal(np.float32(s.camera[k]), r[k]), k
    assert (s.env is None) == (r["env"] is None)
    if s.env is not None:
        assert np.array_equal(np.float32(s.env), np.float32(r["env"]))
    assert len(s.meshes) == len(r["meshes"])
    for i, (a, b) in enumerate(zip(s.meshes, r["meshes"])):
        for k in ("x", "y", "z"):
            assert np.array_equal(getattr(a, k), b[k]), (i, k)
        assert np.array_equal(a.faces, b["faces"]), i
        assert np.array_equal(a.object_to_world, b["object_to_world"]), i
        # the matrix vertex normals are transformed with: the stored inverse of the (final)
        # object-to-world transform, as Transform::ApplyInPlace(Normal&) reads it
        assert np.array_equal(a.world_to_object, b["normal_inverse"]), i
        assert a.is_light == b["is_light"], i
        assert np.array_equal(np.float32(a.emission), b["emission"]), i
        if not a.is_light:
            assert a.material == b["material"] and np.array_equal(np.float32(a.albedo), b["albedo"]), i
        assert (a.normals is None) == (b["normals"] is None), i
        if a.normals is not None:
            assert np.array_equal(a.normals, b["normals"]), i


def test_generated_scene_reads_as_expected(tmp_path):
    s = pb.load_pbrt(write_scene(tmp_path))
    assert (s.width, s.height, s.spp, s.max_depth) == (96, 72, 4, 6)
    assert s.camera == dict(eye=(1.0, 2.0, 8.0), look_at=(0.0, 0.5, 0.0), up=(0.0, 1.0, 0.0), fov=40.0)
    assert np.array_equal(np.float32(s.env), np.float32([.1, .12, .15]) * np.float32(255))
    assert len(s.meshes) == 8
    lights = [m for m in s.meshes if m.is_light]
    assert len(lights) == 2
    # both lights share the scope's radiance and transform, updated after the first shape
    assert lights[0].emission == lights[1].emission == (5 * 255.0,) * 3
    assert np.array_equal(lights[0].object_to_world, lights[1].object_to_world)
    assert np.array_equal(lights[0].world_to_object, lights[1].world_to_object)
    # UV spheres: radius only sets the tessellation (max(int(r), 20) meridians and parallels)
    spheres = [m for m in s.meshes if m.material == pb.MAT_MIRROR]
    assert [len(m.faces) for m in spheres] == [2 * 20 * 20, 2 * 24 * 24]
    assert np.float32(spheres[0].albedo[1]) == np.float32(.85)
    # named matte materials take reflectance 0.5; both instances share one transform
    inst = s.meshes[5:7]
    assert all(m.albedo == (0.5, 0.5, 0.5) for m in inst)
    assert np.array_equal(inst[0].object_to_world, inst[1].object_to_world)
    assert inst[0].object_to_world[2, 3] == np.float32(-4.0)


def test_generated_scene_matches_reference_parser(tmp_path):
    if not po.ref_available():
        pytest.skip("oracle/_ref not built")
    path = write_scene(tmp_path)
    assert_same_as_reference(pb.load_pbrt(path), po.ref_load_pbrt(path))


@pytest.mark.parametrize("scene", MATCHING)
def test_reference_example_scenes_match(scene):
    path = os.path.join(REF_SCENES, scene)
    if not os.path.exists(path) or not po.ref_available():
        pytest.skip("reference scenes or oracle/_ref not available")
    assert_same_as_reference(pb.load_pbrt(path), po.ref_load_pbrt(path))


SCOPES = """LookAt 0 3 9  0 1 0  0 1 0
Camera "perspective" "float fov" [ 35 ]
WorldBegin
  Material "matte" "rgb Kd" [ .2 .3 .4 ]
  AttributeBegin
    AreaLightSource "diffuse" "rgb L" [ 1 2 3 ]
    AttributeBegin
      Material "mirror" "rgb Kr" [ .5 .5 .5 ]
      AreaLightSource "diffuse" "rgb L" [ 7 7 7 ]
      Translate 0 2 0
      Shape "plymesh" "string filename" [ "quad.ply" ]
    AttributeEnd
    Translate 1 0 0
    Shape "plymesh" "string filename" [ "quad.ply" ]
    TransformBegin
      Rotate -40 0 1 0
      Scale 2 1 2
      Shape "plymesh" "string filename" [ "blob.ply" ]
    TransformEnd
  AttributeEnd
  Shape "plymesh" "string filename" [ "blob.ply" ]
  AttributeEnd
  Material "glass"
  Translate 0 -1 0
  Shape "plymesh" "string filename" [ "ground.ply" ]
  Material "mirror" "rgb Kr" [ .7 .8 .9 ]
  AttributeBegin
    Rotate 90 1 0 0
    Shape "sphere" "float radius" [ 3 ]
  AttributeEnd
WorldEnd
"""


def test_nested_scopes_match_reference_parser(tmp_path):
    """Lights and materials saved only when set, a light rewritten inside a nested scope (and so
    for the outer scope's shapes), an unbalanced AttributeEnd, an unknown material (no material),
    TransformBegin inside an attribute scope."""
    path = write_scene(tmp_path, SCOPES)
    s = pb.load_pbrt(path)
    assert len(s.meshes) == 6
    assert s.meshes[0].emission == s.meshes[1].emission == (7 * 255.0,) * 3
    assert s.meshes[4].material == 0  # after Material "glass": no material
    if not po.ref_available():
        pytest.skip("oracle/_ref not built")
    assert_same_as_reference(s, po.ref_load_pbrt(path))


def test_defaults_and_identity_camera(tmp_path):
    write_assets(tmp_path)
    (tmp_path / "s.pbrt").write_text('WorldBegin\nMaterial "matte" "rgb Kd" [ .5 .5 .5 ]\n'
                                     'Shape "plymesh" "string filename" [ "quad.ply" ]\nWorldEnd\n')
    s = pb.load_pbrt(tmp_path / "s.pbrt")
    assert (s.width, s.height, s.spp, s.max_depth) == (640, 360, 8, 5)
    assert s.camera == dict(eye=(0.0, 0.0, 0.0), look_at=(0.0, 0.0, 1.0), up=(0.0, 1.0, 0.0), fov=90.0)
    assert s.env is None and len(s.meshes) == 1


@pytest.mark.parametrize("text,why", [
    ('LookAt 0 0 5 0 0 0 0 1 0\nWorldBegin\nTexture "t" "color" "imagemap" "string filename" [ "a.png" ]\nWorldEnd\n',
     "Texture"),
    ('LookAt 0 0 5 0 0 0 0 1 0\nWorldBegin\nMaterial "plastic" "rgb Kd" [ .5 .5 .5 ]\nWorldEnd\n', "plastic"),
    ('LookAt 0 0 5 0 0 0 0 1 0\nWorldBegin\nShape "objmesh" "string filename" [ "a.obj" ]\nWorldEnd\n', "a.obj"),
    ('Scale -1 1 1\nLookAt 0 0 5 0 0 0 0 1 0\nWorldBegin\nWorldEnd\n', "LookAt"),
    ('LookAt 0 0 5 0 0 0 0 1 0\nLookAt 0 0 5 0 0 0 0 1 0\nWorldBegin\nWorldEnd\n', "LookAt"),
    ('LookAt 0 0 5 0 0 0\nWorldBegin\nWorldEnd\n', "LookAt"),
    ('LookAt 0 0 5 0 0 0 0 1 0\nWorldBegin\nObjectInstance "nothing"\nWorldEnd\n', "nothing"),
    ('LookAt 0 0 5 0 0 0 0 1 0\nWorldBegin\nShape "plymesh" "string filename" [ "missing.ply" ]\nWorldEnd\n', "missing"),
    ('LookAt 0 0 5 0 0 0 0 1 0\nWorldBegin\nWorldEn\n', "WorldEn"),
    ('LookAt 0 0 5 0 0 0 0 1 0\nCamera "perspective" "float fov [ 30 ]\n', "unterminated"),
    # the reference's lexer tests ScaleDirective2 / ScaleDirective3 (tests/parsers/pbrt/test_lex.cpp:54-62)
    # expect its process to exit with status 1 for these; the reader returns PT_EINVAL instead
    ('LookAt 0 0 5 0 0 0 0 1 0\nWorldBegin\nScale 1 2\nWorldEnd\n', "Scale takes 3 numbers"),
    ('LookAt 0 0 5 0 0 0 0 1 0\nWorldBegin\nScale 1 2 3 4\nWorldEnd\n', "Scale takes 3 numbers"),
    ('LookAt 0 0 5 0 0 0 0 1 0\nWorldBegin\nTranslate 1 2\nWorldEnd\n', "Translate takes 3 numbers"),
    ('LookAt 0 0 5 0 0 0 0 1 0\nWorldBegin\nRotate 30 0 1\nWorldEnd\n', "Rotate takes 4 numbers"),
])
def test_unsupported_or_malformed_files_are_rejected(tmp_path, text, why):
    (tmp_path / "bad.pbrt").write_text(text)
    with pytest.raises(pb.PolytopeError) as e:
        pb.load_pbrt(tmp_path / "bad.pbrt")
    assert e.value.code == pb.PT_EINVAL and why in str(e.value)


def test_huge_sphere_radius_is_refused(tmp_path):
    (tmp_path / "s.pbrt").write_text('LookAt 0 0 5 0 0 0 0 1 0\nWorldBegin\nMaterial "matte" "rgb Kd" [ .5 .5 .5 ]\n'
                                     'Shape "sphere" "float radius" [ 1e9 ]\nWorldEnd\n')
    with pytest.raises(pb.PolytopeError) as e:
        pb.load_pbrt(tmp_path / "s.pbrt")
    assert e.value.code == pb.PT_EINVAL and "sphere radius" in str(e.value)


def test_mutated_files_fail_cleanly(tmp_path):
    """Random byte mutations of valid scene, OBJ and PLY files: every load either succeeds or
    raises PolytopeError (PT_EINVAL / PT_ENOMEM) -- never a crash or another exception."""
    import random
    from test_obj_cpu import write_obj
    from test_ply_cpu import CASES, mesh_arrays
    write_scene(tmp_path)
    write_obj(tmp_path / "t.obj", 0)
    fmt, props, ff = CASES[3]
    v, faces = mesh_arrays(3)
    write_ply(tmp_path / "t.ply", fmt, v, faces, props, ff)
    seeds = {"pbrt": (tmp_path / "scene.pbrt").read_bytes(), "obj": (tmp_path / "t.obj").read_bytes(),
             "ply": (tmp_path / "t.ply").read_bytes()}
    rng = random.Random(7)
    loaders = {"pbrt": pb.load_pbrt, "obj": pb.load_obj, "ply": pb.load_ply}
    for it in range(150):
        kind = ("pbrt", "obj", "ply")[it % 3]
        b = bytearray(seeds[kind])
        for _ in range(rng.randint(1, 6)):
            i = rng.randrange(len(b))
            r = rng.random()
            if r < 0.4:
                b[i] = rng.randrange(256)
            elif r < 0.6:
                del b[i:i + rng.randint(1, 40)]
            else:
                b[i:i] = rng.choice([b" [ ", b" ] ", b'"', b"\n", b" 1e38 ", b" -1 ", b" 4294967295 ", b" nan ",
                                     b"AttributeEnd\n", b'ObjectInstance "x"\n'])
        path = tmp_path / ("scene.pbrt" if kind == "pbrt" else f"fz.{kind}")
        path.write_bytes(bytes(b))
        try:
            loaders[kind](path)
        except pb.PolytopeError as e:
            assert e.code in (pb.PT_EINVAL, pb.PT_ENOMEM)
    (tmp_path / "scene.pbrt").write_bytes(seeds["pbrt"])


SPACING = ["[ 40 ]", "[40]", "40", "[ 40]", "[40 ]"]
ARRAYS = ["[.6 .5 .4]", "[ .6 .5 .4 ]", "[ .6 .5 .4]", "[.6 .5 .4 ]"]


@pytest.mark.parametrize("fov", SPACING)
@pytest.mark.parametrize("kd", ARRAYS)
def test_bracket_spacing_variants(tmp_path, fov, kd):
    """The reference's scanner tests (tests/parsers/pbrt/test_scan.cpp:49-104: single values in
    brackets with and without spaces or without brackets, arrays with and without inner spaces)
    restated on whole files: every spelling reads the same, and the same as the reference parser."""
    write_assets(tmp_path)
    path = tmp_path / "s.pbrt"
    path.write_text(f'LookAt 0 0 5  0 0 0  0 1 0\nCamera "perspective" "float fov" {fov}\nWorldBegin\n'
                    f'Material "matte" "rgb Kd" {kd}\nShape "plymesh" "string filename" [ "quad.ply" ]\nWorldEnd\n')
    s = pb.load_pbrt(path)
    assert np.float32(s.camera["fov"]) == np.float32(40)
    assert np.array_equal(np.float32(s.meshes[0].albedo), np.float32([.6, .5, .4]))
    if po.ref_available():
        assert_same_as_reference(s, po.ref_load_pbrt(str(path)))
