"""The output files of Renderer::Render (Renderer.cpp:163-211): PNG and PPM of
the tone-mapped framebuffer, and the adaptive-sampling visualisation. Host-only
entry points; the PNG is checked by decoding it with an independent reader."""
import numpy as np
import pytest

import photorealisticrender4610_b200 as prr


def test_png_and_ppm_round_trip(tmp_path):
    from PIL import Image
    rng = np.random.default_rng(0)
    img = (rng.random((37, 53, 3)) * 255).astype(np.uint8)
    prr.write_image(tmp_path / "out.png", img)
    back = np.asarray(Image.open(tmp_path / "out.png").convert("RGB"))
    assert np.array_equal(back, img)
    prr.write_image(tmp_path / "out.ppm", img)
    data = (tmp_path / "out.ppm").read_bytes()
    header = b"P6\n53 37\n255\n"
    assert data.startswith(header) and data[len(header):] == img.tobytes()
    with pytest.raises(prr.PrrError):
        prr.write_image(tmp_path / "out.bmp", img)


def test_sample_count_image_formula():
    spp = np.array([[1, 7, 64], [255, 256, 100]], np.int32)
    out = prr.sample_count_image(spp, 256)
    want = (255 * spp.astype(np.float32) / np.float32(256)).astype(np.uint8)
    assert np.array_equal(out[..., 0], want) and (out[..., 0] == out[..., 2]).all()
