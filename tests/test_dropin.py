"""The reference-named C++ classes of include/prr_dropin.hpp: a C++ program
written like the reference's scene setup compiles against them, and on the
GPU renders the same image as the Python API."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "dropin_example.cpp"
LIBDIR = ROOT / "photorealisticrender4610_b200"


def build_example(tmp_path):
    exe = tmp_path / "dropin_example"
    cmd = ["/usr/bin/g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"),
           "-I", "/usr/local/cuda/include", str(SRC), "-o", str(exe), "-L", str(LIBDIR), "-lprr",
           f"-Wl,-rpath,{LIBDIR}", "-L", "/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_dropin_example_compiles(tmp_path, lib):
    assert build_example(tmp_path).exists()


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
    assert (tmp_path / "output.ppm").exists() and (tmp_path / "output_raw.ppm").exists()
    assert "hit 1 obj 2" in r.stdout  # the back wall
