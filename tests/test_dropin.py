"""The reference-named C++ classes of include/prr_dropin.hpp: a C++ program
written like the reference's scene setup compiles against them, and on the
GPU renders the same image as the Python API."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "dropin_example.cpp"
GLTF_SRC = ROOT / "tests" / "cpp" / "gltf_example.cpp"
OBJ_SRC = ROOT / "tests" / "cpp" / "obj_example.cpp"
LIBDIR = ROOT / "photorealisticrender4610_b200"


def build_example(tmp_path, src=SRC):
    exe = tmp_path / src.stem
    cmd = ["/usr/bin/g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"),
           "-I", "/usr/local/cuda/include", str(src), "-o", str(exe), "-L", str(LIBDIR), "-lprr",
           f"-Wl,-rpath,{LIBDIR}", "-L", "/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_dropin_example_compiles(tmp_path, lib):
    assert build_example(tmp_path).exists()
    assert build_example(tmp_path, GLTF_SRC).exists()
    assert build_example(tmp_path, OBJ_SRC).exists()


@pytest.mark.gpu
def test_dropin_renders_like_the_python_api(tmp_path, cuda):
    import photorealisticrender4610_b200 as prr
    from photorealisticrender4610_b200 import scenes
    exe = build_example(tmp_path)
    out = tmp_path / "fb.bin"
    r = subprocess.run([str(exe), str(out)], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    fb = np.fromfile(out, np.float32).reshape(64, 64, 3)
    s = prr.Scene.from_desc(scenes.cornell_box(64, 64))
    want, _ = s.render(16, 5, seed=1)
    assert np.array_equal(fb.view(np.uint32), want.cpu().numpy().view(np.uint32))
    for name in ("output", "output_raw", "sample_count"):
        assert (tmp_path / f"{name}.ppm").exists() and (tmp_path / f"{name}.png").exists()
    # output.png is the tone-mapped framebuffer (the drop-in's default AgX, exposure 1)
    from PIL import Image
    _, u8 = prr.tonemap(want, "agx", 1.0)
    png = np.asarray(Image.open(tmp_path / "output.png").convert("RGB"))
    assert np.array_equal(png, u8.cpu().numpy())
    assert "hit 1 obj 2" in r.stdout  # the back wall


@pytest.mark.gpu
def test_gltf_dropin_renders_like_the_python_api(tmp_path, cuda):
    """GLTFLoader::load of the drop-in header on a file written by the test
    writer, rendered by Renderer::Render, equals the Python API's add_gltf
    scene rendered in the same mode and seed."""
    import sys
    sys.path.insert(0, str(ROOT / "tests"))
    import gltf_writer
    import photorealisticrender4610_b200 as prr
    from photorealisticrender4610_b200 import scenes
    path = tmp_path / "features.glb"
    gltf_writer.feature_file(path)
    exe = build_example(tmp_path, GLTF_SRC)
    out = tmp_path / "fb.bin"
    r = subprocess.run([str(exe), str(path), str(out)], cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    fb = np.fromfile(out, np.float32).reshape(72, 96, 3)
    s = prr.Scene()
    s.add_gltf(path)
    lm = s.add_material(1, [0.8, 0.8, 0.8, 0.5, 0.0, 1.5, 20.0, 20.0, 20.0])
    s.add_sphere((0.3, 1.4, 0.2), 0.25, lm)
    s.set_camera(scenes.Camera(eye=(0.0, 2.0, 2.6), target=(0, 0, 0), up=(0, 1, 0), fovv=50.0,
                               fovh=60.0), 96, 72)
    s.buildBVH()
    want, _ = s.render(64, 6, seed=3, mode="wavefront")
    assert np.array_equal(fb.view(np.uint32), want.cpu().numpy().view(np.uint32))


@pytest.mark.gpu
def test_obj_dropin_renders_like_the_python_api(tmp_path, cuda):
    """MeshTriangle(filename, offset, m) of the drop-in header on an OBJ
    height field, rendered by Renderer::Render, equals the Python API's
    add_obj scene at the same seed (plain mode, one slice per pixel)."""
    import sys
    sys.path.insert(0, str(ROOT / "tests"))
    from test_obj import grid_obj
    import photorealisticrender4610_b200 as prr
    from photorealisticrender4610_b200 import scenes
    path = tmp_path / "grid.obj"
    path.write_text(grid_obj(9, seed=2))
    exe = build_example(tmp_path, OBJ_SRC)
    out = tmp_path / "fb.bin"
    r = subprocess.run([str(exe), str(path), str(out)], cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    # the diagonal ray enters the box at 2*sqrt(3) and leaves at 4*sqrt(3); the
    # reference's intersect misses axis-aligned rays (their zero components)
    assert "medium 1 3.4641 6.9282 active 1" in r.stdout, r.stdout
    assert "axis-aligned 0" in r.stdout
    fb = np.fromfile(out, np.float32).reshape(60, 80, 3)
    s = prr.Scene()
    m = s.add_material(0, [0.7, 0.6, 0.5, 0.5, 0.0, 1.5, 0.0, 0.0, 0.0])
    s.add_obj(path, m, (-0.5, 0.0, -0.5))
    lm = s.add_material(1, [0.8, 0.8, 0.8, 0.5, 0.0, 1.5, 15.0, 15.0, 15.0])
    s.add_sphere((0.0, 1.2, 0.0), 0.2, lm)
    s.set_camera(scenes.Camera(eye=(0.0, 1.6, 1.8), target=(0, 0, 0), up=(0, 1, 0), fovv=50.0,
                               fovh=60.0), 80, 60)
    s.buildBVH()
    want, _ = s.render(32, 5, seed=5)
    assert np.array_equal(fb.view(np.uint32), want.cpu().numpy().view(np.uint32))
