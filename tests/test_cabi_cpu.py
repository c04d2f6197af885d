"""The C ABI from C and C++ callers: include/polytope_b200.h compiles as C99 and as C++17, and a
program linked against the library reads a PBRT scene, its meshes and a PLY file, builds the
reference tree and round-trips a tuning-cache entry through the exported entry points (calls that
need no GPU), with the same results as the Python binding."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import polytope_b200 as pb
from test_pbrt_cpu import write_scene

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.dirname(pb.LIB_PATH)

C_SRC = r"""
#include <stdio.h>
#include <stdlib.h>
#include "polytope_b200.h"

int main(int argc, char **argv) {
    pt_pbrt_scene *ps = NULL;
    if (pt_load_pbrt(argv[1], &ps) != PT_OK) { printf("error %s\n", pt_last_error()); return 1; }
    pt_pbrt_info info;
    const pt_mesh_desc *meshes = NULL;
    pt_pbrt_get_info(ps, &info);
    pt_pbrt_get_meshes(ps, &meshes);
    unsigned faces = 0;
    for (unsigned i = 0; i < info.num_meshes; ++i) faces += meshes[i].num_faces;
    unsigned num_nodes = 2 * faces;
    pt_bvh_node *nodes = (pt_bvh_node *)malloc(sizeof(pt_bvh_node) * num_nodes);
    unsigned *pairs = (unsigned *)malloc(2 * sizeof(unsigned) * faces);
    int rc = pt_bvh_build(meshes, info.num_meshes, 0, nodes, &num_nodes, pairs);
    printf("%u %u %u %u %u %u %d %.6g %u %u\n", info.num_meshes, faces, info.width, info.height, info.spp,
           info.max_depth, rc, info.camera.fov_deg, num_nodes, nodes[0].offset);
    pt_pbrt_free(ps);
    free(nodes);
    free(pairs);
    pt_mesh_data ply;
    if (pt_load_ply(argv[2], &ply) != PT_OK) { printf("error %s\n", pt_last_error()); return 1; }
    printf("%u %u %d\n", ply.num_vertices, ply.num_faces, ply.nx != NULL);
    pt_mesh_data_free(&ply);
    pt_tuning_class cls = {0};
    snprintf(cls.device, sizeof cls.device, "%s", "C caller GPU");
    cls.sm_count = 148;
    cls.compute_capability = 100;
    cls.items_log2 = 3;
    pt_batch_tuning t, back;
    pt_batch_default_tuning(&t);
    t.queue_chunk = 96;
    double ms = 0;
    int found = 0;
    const int put = pt_tuning_cache_put(argv[3], &cls, &t, 2.5);
    const int get = pt_tuning_cache_get(argv[3], &cls, &back, &ms, &found);
    printf("%d %d %d %.3g %u\n", put, get, found, ms, back.queue_chunk);
    printf("%s\n", pt_version());
    return 0;
}
"""


def build_and_run(tmp_path, compiler, std, name, args):
    exe = tmp_path / name
    src = tmp_path / (name + (".c" if compiler == "gcc" else ".cpp"))
    src.write_text(C_SRC)
    cmd = [compiler, f"-std={std}", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
           "-L", LIBDIR, "-lpolytope_b200", f"-Wl,-rpath,{LIBDIR}"]
    if compiler == "g++":
        cmd.insert(1, "-x")
        cmd.insert(2, "c++")
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)] + [str(a) for a in args], check=True, capture_output=True, text=True).stdout
    return out.strip().splitlines()


@pytest.mark.parametrize("compiler,std", [("gcc", "c99"), ("g++", "c++17")])
def test_c_and_cpp_callers(tmp_path, compiler, std):
    if not shutil.which(compiler):
        pytest.skip(f"{compiler} not available")
    scene = write_scene(tmp_path)
    lines = build_and_run(tmp_path, compiler, std, "caller", [scene, tmp_path / "blob.ply", tmp_path / "tune.json"])
    s = pb.load_pbrt(scene)
    nodes, pairs = pb.bvh_build(s.meshes)
    faces = sum(len(m.faces) for m in s.meshes)
    f = lines[0].split()
    assert [int(v) for v in f[:6]] == [len(s.meshes), faces, s.width, s.height, s.spp, s.max_depth]
    assert int(f[6]) == pb.PT_OK and float(f[7]) == s.camera["fov"]
    assert int(f[8]) == len(nodes) and int(f[9]) == int(nodes[0]["offset"])
    m = pb.load_ply(tmp_path / "blob.ply")
    assert lines[1].split() == [str(len(m.x)), str(len(m.faces)), "1"]
    assert lines[2].split() == ["0", "0", "1", "2.5", "96"]  # the tuning cache from C
    assert lines[3] == pb.version()


def test_render_example_builds_and_fails_cleanly_without_a_device(tmp_path):
    """polytope_b200/examples/render_pbrt.cpp compiles against the header; here, without a CUDA
    device, it stops at pt_scene_create with the library's PT_ECUDA message."""
    import torch
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    exe = tmp_path / "render_pbrt"
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "polytope_b200", "examples", "render_pbrt.cpp"), "-o", str(exe),
                    "-L", LIBDIR, "-lpolytope_b200", f"-Wl,-rpath,{LIBDIR}"], check=True, capture_output=True)
    if torch.cuda.is_available():
        pytest.skip("this checks the no-device path")
    scene = write_scene(tmp_path)
    p = subprocess.run([str(exe), str(scene), str(tmp_path / "out.png")], capture_output=True, text=True)
    assert p.returncode == 1 and "pt_scene_create" in p.stderr and "no CUDA device" in p.stderr
