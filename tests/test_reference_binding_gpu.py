"""The reference-side binding on the device: the reference's own render call (main.cpp:187-220 --
parse the PBRT file with pbrt_parser, bvh::bound + compact, spawn the runner's threads, join,
Output()) with polytope_b200/examples/reference_binding.h's GpuRunner in place of TileRunner.

The driver oracle/_ref/check_reference_binding is compiled by oracle/Makefile against the
reference's headers and classes (oracle/_ref/libpolyref.so) where the reference tree is present;
here it only runs.  The scene is the generated PBRT file of tests/test_pbrt_cpu.py (area lights
updated in place, mirror and matte materials, UV spheres, named materials, object instances).
Checked bit for bit:
  * the float film GpuRunner rendered equals pt_load_pbrt + pt_render's film of the same file;
  * the PNG the reference's PNGFilm wrote from that film (BoxFilter, lodepng) and the PNG that
    DevicePNGFilm wrote (pt_render_rgba8: quantised on the device, pt_write_png) decode to the
    same pixels, equal to the oracle's restatement of PNGFilm::Output on the film."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, assert_bit_equal
import polytope_b200 as pb
from oracle import pyoracle as po
from test_pbrt_cpu import write_scene

pytestmark = pytest.mark.gpu

CHECKER = os.path.join(ROOT, "oracle", "_ref", "check_reference_binding")


def test_reference_render_call_with_gpu_runner(cuda_device, tmp_path):
    assert os.path.exists(CHECKER), "oracle/_ref/check_reference_binding is built by `make -C oracle` with the reference tree"
    scene_file = write_scene(tmp_path)
    p = subprocess.run([CHECKER, str(scene_file), "--render", str(tmp_path), "4"], capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.split()[7] == "yes", p.stdout
    s = pb.load_pbrt(scene_file)
    scene = pb.Scene(s.meshes, s.env)
    rgb, _ = pb.render(scene, s.width, s.height, s.spp, s.max_depth, s.camera, seed=1, flags=pb.RENDER_NEE)
    film = np.fromfile(tmp_path / "film.bin", np.float32).reshape(s.height, s.width, 3)
    assert_bit_equal(film, rgb, "GpuRunner film vs pt_render")
    assert rgb.mean() > 1.0
    exp = po.film_to_rgba8(rgb)
    assert_bit_equal(po.ref_png_decode(tmp_path / "float_film.png"), exp, "reference PNGFilm output")
    assert_bit_equal(po.ref_png_decode(tmp_path / "device_film.png"), exp, "DevicePNGFilm output")
    rgba, _ = pb.render_rgba8(scene, s.width, s.height, s.spp, s.max_depth, s.camera, seed=1, flags=pb.RENDER_NEE)
    assert_bit_equal(rgba, exp, "pt_render_rgba8")
