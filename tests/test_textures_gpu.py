"""Per-corner mesh data and material textures on the GPU path against the
reference: Triangle::finalize's interpolated normals, uvs and tangents
(Triangle.cpp:34-59), ShadingData with base-colour, metallic-roughness and
normal-map textures (Material.cpp:3-26, Material.hpp:57-70,
TextureUtils.hpp:22-136), on a scene the reference renders through the same
fields its glTF loader fills (GLTFLoader.cpp:224-262).

Texture lookups use powf for the sRGB decode (CUDA's, not libm's), so paths
agree with the reference up to last-ulp differences; images are gated by
relative MSE = sum((gpu - ref)^2) / sum(ref^2) <= 1e-3, as elsewhere.
"""
import numpy as np
import pytest
import torch

import photorealisticrender4610_b200 as prr
from photorealisticrender4610_b200 import scenes

pytestmark = pytest.mark.gpu

REL_MSE_TOL = 1e-3


def rel_mse(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-30))


@pytest.fixture(scope="module")
def showcase():
    return scenes.textured_showcase(160, 120)


def test_smooth_normals_and_hits_match_reference(ref, cuda, showcase):
    s = prr.Scene.from_desc(showcase)
    rs = ref.scene(showcase)
    rng = np.random.default_rng(3)
    n = 20000
    o = np.tile(np.array([[0.0, 2.2, 5.0]], np.float32), (n, 1))
    tgt = np.column_stack([rng.uniform(-2.5, 2.5, n), rng.uniform(0.0, 2.0, n),
                           rng.uniform(-2.5, 1.5, n)]).astype(np.float32)
    d = (tgt - o) / np.linalg.norm(tgt - o, axis=1, keepdims=True)
    d = d.astype(np.float32)
    obj, prim, t, geo = s.intersect(torch.from_numpy(o).to(cuda), torch.from_numpy(d).to(cuda),
                                    geo=True)
    robj, rprim, rt, rgeo = rs.intersect(o, d, geo=True)
    assert np.array_equal(obj.cpu().numpy(), robj)
    assert np.array_equal(prim.cpu().numpy(), rprim)
    assert np.array_equal(t.cpu().numpy().view(np.uint32), rt.view(np.uint32))
    # coordinates and the interpolated (smooth) normals of the hits, bit for bit
    hit = robj >= 0
    assert np.array_equal(geo.cpu().numpy()[hit].view(np.uint32), rgeo[hit].view(np.uint32))
    on_ball = robj == 1
    assert on_ball.sum() > 1000
    # the smooth normal differs from the face normal inside the triangles
    face = showcase.objects[1].verts.reshape(-1, 3, 3)
    fn = np.cross(face[:, 1] - face[:, 0], face[:, 2] - face[:, 0])
    fn /= np.linalg.norm(fn, axis=1, keepdims=True)
    assert np.abs(rgeo[on_ball, 3:] - fn[rprim[on_ball]]).max() > 1e-3


def test_textured_paths_lockstep(ref, cuda, showcase):
    s = prr.Scene.from_desc(showcase)
    rs = ref.scene(showcase)
    rng = np.random.default_rng(5)
    n = 4096
    px = rng.integers(0, showcase.width, n).astype(np.int32)
    py = rng.integers(0, showcase.height, n).astype(np.int32)
    sm = rng.integers(0, 1000, n).astype(np.int32)
    out = s.cast_samples(px, py, sm, max_depth=8, seed=2).cpu().numpy()
    rout, _ = rs.cast_samples(8, 2, px, py, sm)
    err = np.abs(out - rout).max(1) / np.maximum(np.abs(rout).max(1), 1e-3)
    assert (err < 1e-3).mean() > 0.95, (err < 1e-3).mean()


@pytest.mark.parametrize("mode", ["plain", "wavefront"])
def test_textured_4096spp_against_reference(ref, cuda, showcase, mode):
    """A 24x24 crop covering the normal-mapped ball, its shadow and the
    textured floor at 4096 spp against the reference on the same streams."""
    win = (56, 58, 80, 82)
    s = prr.Scene.from_desc(showcase)
    img, _ = s.render(4096, 8, seed=1, window=win, mode=mode)
    rimg, _ = ref.scene(showcase).render(8, 4096, 1, window=win)
    err = rel_mse(img.cpu().numpy(), rimg)
    print(f"textured 4096 spp crop rMSE vs reference ({mode}): {err:.3e}")
    assert err < REL_MSE_TOL


def test_textured_wavefront_equals_plain(cuda, showcase):
    s = prr.Scene.from_desc(showcase)
    a, _ = s.render(16, 8, seed=9, slices=1)
    npix = showcase.width * showcase.height
    s.set_wavefront(paths_per_pass=npix * 4, block_size=128, ordered=True)
    b, _ = s.render(16, 8, seed=9, mode="wavefront")
    assert np.array_equal(a.cpu().numpy().view(np.uint32), b.cpu().numpy().view(np.uint32))


def test_texture_arguments_rejected(cuda):
    s = prr.Scene()
    m = s.add_material(0, [0.8, 0.8, 0.8, 0.5, 0.0, 1.5, 0.0, 0.0, 0.0])
    with pytest.raises(prr.PrrError):
        s.add_texture(np.zeros((4, 4, 2), np.uint8))  # needs 3 or 4 channels
    t = s.add_texture(np.zeros((4, 4, 3), np.uint8))
    with pytest.raises(prr.PrrError):
        s.set_material_textures(m, base_color=t + 1)
    s.set_material_textures(m, base_color=t)
