"""glTF ingest (prr_scene_add_gltf) against the reference's own GLTFLoader
(GLTFLoader.cpp, on tinygltf, compiled into the oracle): for every primitive
the same triangles, normalized corner normals, uvs and tangents bit for bit,
the same material class and parameters, and the same decoded texels. Files are
written by tests/gltf_writer.py to cover the accessor, index, image and
material variants; the reference's own .glb assets are read too when the
reference tree is present. On the GPU, a glTF scene renders as the reference
renders it."""
from pathlib import Path

import numpy as np
import pytest

import gltf_writer
import photorealisticrender4610_b200 as prr
from oracle import loader

REF_ASSETS = loader.REFERENCE_ROOT / "assets" / "models"

pytestmark = pytest.mark.skipif(not loader.reference_available(),
                                reason="reference oracle library not built")


@pytest.fixture(scope="module")
def ref_oracle():
    return loader.ReferenceOracle()


def compare(path, ref_oracle, material_type="diffuse"):
    s = prr.Scene()
    info = s.add_gltf(path, material_type)
    rg = loader.RefGltf(ref_oracle, path, material_type)
    assert info["count"] == rg.count
    for k in range(rg.count):
        ours = s.export_mesh(info["first"] + k)
        ref = rg.mesh(k)
        assert np.array_equal(ours["verts"].view(np.uint32), ref["verts"].view(np.uint32)), k
        assert ("normals" in ours) == bool(ref["attr"] & 1), k
        if "normals" in ours:
            assert np.array_equal(ours["normals"].view(np.uint32), ref["normals"].view(np.uint32))
        if "uvs" in ours:
            assert np.array_equal(ours["uvs"].view(np.uint32), ref["uvs"].view(np.uint32)), k
        else:
            assert not ref["uvs"].any()
        assert ("tangents" in ours) == bool(ref["attr"] & 4), k
        if "tangents" in ours:
            assert np.array_equal(ours["tangents"].view(np.uint32),
                                  ref["tangents"].view(np.uint32))
        m = s.export_material(k)  # one material per primitive, in primitive order
        rm = rg.material(k)
        assert m["kind"] == rm["kind"], k
        assert np.array_equal(m["params"].view(np.uint32), rm["params"].view(np.uint32)), k
        for slot in range(4):
            t = m["textures"][slot]
            rt = rm["textures"][slot]
            assert (t >= 0) == (rt is not None), (k, slot)
            if t < 0:
                continue
            texels = s.export_texture(int(t))
            if slot == 3 and rt.size != texels.size:  # bytes, not texels
                # the reference keeps a 16-bit emissive image undecimated
                # (GLTFLoader.cpp:131-137); the path never samples it
                assert texels.shape[:2] == rt.shape[:2]
                continue
            assert np.array_equal(texels, rt), (k, slot)
    return s, info


@pytest.mark.parametrize("as_gltf", [False, True])
def test_feature_file_matches_reference_loader(tmp_path, ref_oracle, as_gltf):
    path = tmp_path / ("features.gltf" if as_gltf else "features.glb")
    gltf_writer.feature_file(path, as_gltf=as_gltf)
    s, info = compare(path, ref_oracle)
    assert info["count"] == 4 and info["undecoded_images"] == 0
    # grey, palette and 16-bit images arrive as 8-bit RGBA
    kinds = [s.export_texture(t).shape for t in range(5)]
    assert all(k[2] == 4 for k in kinds)


@pytest.mark.parametrize("material_type", ["glass", "mirror", "emit"])
def test_material_types_match_reference_loader(tmp_path, ref_oracle, material_type):
    path = tmp_path / "features.glb"
    gltf_writer.feature_file(path)
    compare(path, ref_oracle, material_type)


@pytest.mark.skipif(not REF_ASSETS.exists(), reason="reference assets not present")
@pytest.mark.parametrize("name", ["floor", "left", "right", "light", "shortbox", "tallbox"])
def test_reference_assets(ref_oracle, name):
    compare(REF_ASSETS / f"{name}.glb", ref_oracle)


def test_bad_files_fail_cleanly(tmp_path):
    s = prr.Scene()
    with pytest.raises(prr.PrrError):
        s.add_gltf(tmp_path / "missing.glb")
    bad = tmp_path / "bad.glb"
    bad.write_bytes(b"glTF\x02\x00\x00\x00\x10\x00\x00\x00garbage!")
    with pytest.raises(prr.PrrError):
        s.add_gltf(bad)
    junk = tmp_path / "junk.gltf"
    junk.write_text('{"asset": {"version": "2.0"}, "meshes": [{"primitives": [{"attributes": '
                    '{"POSITION": 7}}]}]}')
    with pytest.raises(prr.PrrError):
        s.add_gltf(junk)


@pytest.mark.gpu
def test_gltf_scene_renders_like_reference(tmp_path, ref_oracle, cuda):
    """The feature file plus an emissive sphere and a camera, rendered on the
    GPU and by the reference (meshes from its own loader) on the same RNG
    streams: image rMSE <= 1e-3, and the wavefront film equal to the plain one."""
    path = tmp_path / "features.glb"
    gltf_writer.feature_file(path)
    W, H = 96, 72
    light = [0.8, 0.8, 0.8, 0.5, 0.0, 1.5, 20.0, 20.0, 20.0]
    eye, target, up = (0.0, 2.0, 2.6), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0)

    s = prr.Scene()
    s.add_gltf(path)
    lm = s.add_material(1, light)
    s.add_sphere((0.3, 1.4, 0.2), 0.25, lm)
    from photorealisticrender4610_b200 import scenes
    cam = scenes.Camera(eye=eye, target=target, up=up, fovv=50.0, fovh=60.0)
    s.set_camera(cam, W, H)
    s.buildBVH()

    rg = loader.RefGltf(ref_oracle, path)
    L = ref_oracle.L
    f32 = lambda v: np.ascontiguousarray(v, np.float32)  # noqa: E731
    rlm = L.prr_ref_scene_add_material(rg.h, 1, f32(light))
    L.prr_ref_scene_add_sphere(rg.h, f32((0.3, 1.4, 0.2)), 0.25, rlm)
    L.prr_ref_scene_set_camera(rg.h, f32(eye), f32(target), f32(up), 50.0, 60.0, 0.0, -1.0, W, H)
    L.prr_ref_scene_build(rg.h)

    rimg = np.empty((W * H, 3), np.float32)
    cnt = np.empty(W * H, np.int32)
    L.prr_ref_render(rg.h, 6, 256, 256, 0.05, 3, 0, 0, W, H, rimg, cnt.ctypes.data, 0)
    img, _ = s.render(256, 6, seed=3)
    img = img.cpu().numpy().reshape(-1, 3)
    err = float(((img.astype(np.float64) - rimg) ** 2).sum() / (rimg.astype(np.float64) ** 2).sum())
    print(f"glTF scene 256 spp rMSE vs reference: {err:.3e}")
    assert err < 1e-3
    one, _ = s.render(256, 6, seed=3, slices=1)  # one thread per pixel: sample order
    wf, _ = s.render(256, 6, seed=3, mode="wavefront")
    assert np.array_equal(wf.cpu().numpy(), one.cpu().numpy())
