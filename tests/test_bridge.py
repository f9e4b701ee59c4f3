"""include/prr_bridge.hpp: a scene built with the reference renderer's own
classes (MeshTriangle, Sphere, the four materials, EnvMap, Camera) is handed to
libprr and renders exactly as the same scene built through the Python API.

The reference objects come from the oracle build (oracle/_ref/
libprr_ref_bridge.so: the reference sources, the harness that assembles
reference scenes, and oracle/ref/bridge.cpp which calls prr_bridge::render)."""
import numpy as np
import pytest

from oracle import loader

pytestmark = pytest.mark.skipif(not loader.reference_available(bridge=True),
                                reason="oracle/_ref/libprr_ref_bridge.so not built")


@pytest.fixture(scope="module")
def bridge_ref(lib):
    return loader.ReferenceOracle(bridge=True)


def test_bridge_library_exports_entry_point(bridge_ref):
    assert hasattr(bridge_ref.L, "prr_ref_bridge_render")


def _scenes():
    from photorealisticrender4610_b200 import scenes
    yield "cornell", scenes.cornell_box(64, 64), 5
    yield "museum", scenes.museum_like(96, 64, level=3, env_size=(256, 128)), 8
    yield "textured", scenes.textured_showcase(96, 72), 8


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["plain", "wavefront"])
def test_bridge_render_matches_api(bridge_ref, cuda, mode):
    import photorealisticrender4610_b200 as prr
    from photorealisticrender4610_b200.api import RENDER_MODES
    for name, desc, depth in _scenes():
        rs = bridge_ref.scene(desc)
        rgb, spp, u8, rep = rs.bridge_render(depth, 8, 8, seed=3, mode=RENDER_MODES[mode],
                                             mapper=2, exposure=0.18)
        n_mesh = sum(o.kind == "mesh" for o in desc.objects)
        assert rep["meshes"] == n_mesh and rep["skipped_objects"] == 0, (name, rep)
        assert rep["spheres"] == len(desc.objects) - n_mesh and rep["dropped"] == 0
        assert rep["attributed_meshes"] == sum(o.kind == "mesh" and o.has_attributes()
                                               for o in desc.objects)
        assert rep["textures"] == sum(t is not None for m in desc.materials
                                      for t in m.texture_list())
        s = prr.Scene.from_desc(desc)
        want, cnt = s.render(8, depth, seed=3, mode=mode)
        assert np.array_equal(rgb.view(np.uint32), want.cpu().numpy().view(np.uint32)), name
        assert (spp == 8).all() and (cnt.cpu().numpy() == 8).all()
        _, want_u8 = prr.tonemap(want, "agx", 0.18)
        assert np.array_equal(u8, want_u8.cpu().numpy()), name


@pytest.mark.gpu
def test_bridge_adaptive_render_matches_api(bridge_ref, cuda):
    import photorealisticrender4610_b200 as prr
    from photorealisticrender4610_b200 import scenes
    desc = scenes.cornell_box(48, 48)
    rgb, spp, _, _ = bridge_ref.scene(desc).bridge_render(5, 4, 64, threshold=0.05, seed=2,
                                                          mode=0)
    want, cnt = prr.Scene.from_desc(desc).render(64, 5, seed=2, min_spp=4, threshold=0.05)
    assert np.array_equal(spp, cnt.cpu().numpy())
    assert np.array_equal(rgb.view(np.uint32), want.cpu().numpy().view(np.uint32))
    assert spp.min() >= 4 and spp.max() <= 64 and spp.min() < spp.max()
