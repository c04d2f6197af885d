"""The reference-side binding (polytope_b200/examples/reference_binding.h: poly::Scene ->
pt_scene_desc, make_gpu_scene, GpuRunner) compiled against the reference's own headers and classes
and run on PBRT scenes parsed by the reference's pbrt_parser (tests/binding/check_reference_binding.cpp).
It checks that the library's SAH build of the converted meshes equals the tree the reference built
(nodes and leaf pairs, bit for bit), that the converted descriptors equal pt_load_pbrt's reading of
the same file, and that without a device the device calls fail with the library's status instead of
ending the process.  Needs the reference tree (headers) and oracle/_ref/libpolyref.so, so it runs
where the reference is present and is skipped elsewhere."""
import os
import shutil
import subprocess

import pytest

from conftest import reference_path

from test_pbrt_cpu import MATCHING, REF_SCENES, write_scene

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SRC = reference_path("src")
REF_LIB = os.path.join(ROOT, "oracle", "_ref")
LIBDIR = os.path.join(ROOT, "polytope_b200", "lib")

pytestmark = pytest.mark.skipif(
    not (os.path.isdir(REF_SRC) and os.path.exists(os.path.join(REF_LIB, "libpolyref.so")) and shutil.which("g++")),
    reason="needs the reference's headers, oracle/_ref and g++")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = tmp_path_factory.mktemp("binding") / "check_reference_binding"
    subprocess.run(["g++", "-O1", "-std=c++14", "-include", "limits", "-I", REF_SRC, "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "polytope_b200", "examples"),
                    os.path.join(ROOT, "tests", "binding", "check_reference_binding.cpp"), "-o", str(exe),
                    "-L", REF_LIB, "-lpolyref", "-L", LIBDIR, "-lpolytope_b200",
                    f"-Wl,-rpath,{REF_LIB}", f"-Wl,-rpath,{LIBDIR}"], check=True, capture_output=True, text=True)
    return exe


def run(exe, scene):
    p = subprocess.run([str(exe), str(scene)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    f = p.stdout.split()
    return dict(meshes=int(f[1]), faces=int(f[3]), nodes=int(f[5]), device=f[7])


def test_binding_on_generated_scene(checker, tmp_path):
    """Area lights updated in place, mirror and matte materials, UV spheres, named materials and
    object instances: the binding's descriptors equal pt_load_pbrt's and the trees match."""
    import torch
    r = run(checker, write_scene(tmp_path))
    assert r["meshes"] == 8 and r["faces"] > 1000 and r["nodes"] > r["faces"] // 2
    if not torch.cuda.is_available():
        assert r["device"] == "no"


@pytest.mark.parametrize("scene", MATCHING)
def test_binding_on_reference_example_scenes(checker, scene):
    r = run(checker, os.path.join(REF_SCENES, scene))
    if scene == "minimum-emptyworld.pbrt":
        assert r["meshes"] == 0 and r["nodes"] == 0
    else:
        assert r["meshes"] >= 1 and r["nodes"] >= 1
