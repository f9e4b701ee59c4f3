"""Seeded random scenes -- spheres and meshes of every material kind (GGX
diffuse/metallic, mirror, glass, emissive), area lights and/or an HDR sky --
rendered on the GPU: the wavefront integrator equals the plain one bit for bit
(fixed and adaptive spp), and both agree with the reference renderer on the
same RNG streams (relative MSE <= 1e-3, as the other image tests)."""
import numpy as np
import pytest

import photorealisticrender4610_b200 as prr
from photorealisticrender4610_b200 import scenes

pytestmark = pytest.mark.gpu

SEEDS = [11, 12, 13, 14, 15, 16]
REL_MSE_TOL = 1e-3


def rel_mse(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-30))


def random_scene(seed: int, w: int = 48, h: int = 40) -> scenes.SceneDesc:
    rng = np.random.default_rng(seed)
    d = scenes.SceneDesc(width=w, height=h, name=f"fuzz{seed}")

    def material():
        k = rng.choice([scenes.DIFFUSE, scenes.DIFFUSE, scenes.MIRROR, scenes.GLASS])
        base = tuple(rng.uniform(0.1, 0.95, 3))
        if k == scenes.DIFFUSE:
            return d.add_material(scenes.Material(scenes.DIFFUSE, base, float(rng.uniform(0.05, 1.0)),
                                                  float(rng.random() < 0.4)))
        if k == scenes.GLASS:
            return d.add_material(scenes.Material(scenes.GLASS, (1.0, 1.0, 1.0), 0.0, 0.0,
                                                  float(rng.uniform(1.2, 1.8))))
        return d.add_material(scenes.Material(scenes.MIRROR, base))

    ground = d.add_material(scenes.Material(scenes.DIFFUSE, (0.6, 0.6, 0.6), 0.8, 0.0))
    d.objects.append(scenes.MeshObject(scenes.quad((-4, 0, 4), (4, 0, 4), (4, 0, -4), (-4, 0, -4)),
                                       ground))
    for _ in range(int(rng.integers(2, 5))):
        r = float(rng.uniform(0.15, 0.5))
        c = (float(rng.uniform(-1.5, 1.5)), r, float(rng.uniform(-1.5, 1.0)))
        d.objects.append(scenes.SphereObject(c, r, material()))
    for k in range(int(rng.integers(1, 4))):
        level = int(rng.integers(1, 3))
        c = (float(rng.uniform(-1.5, 1.5)), 0.45, float(rng.uniform(-1.5, 1.0)))
        v = scenes.displaced_icosphere(level, c, 0.4, 0.05, seed * 10 + k)
        d.objects.append(scenes.MeshObject(v, material()))
    lights = int(rng.integers(0, 3))
    if lights == 0 or rng.random() < 0.5:
        d.env = scenes.rgbe_quantize(scenes.procedural_sky(128, 64))
    for k in range(lights):
        le = float(rng.uniform(5, 30))
        lm = d.add_material(scenes.Material(scenes.EMISSIVE, (0.8, 0.8, 0.8), emission=(le, le, le)))
        if k == 0:
            y = 2.5
            d.objects.append(scenes.MeshObject(
                scenes.quad((-0.5, y, -0.5), (0.5, y, -0.5), (0.5, y, 0.5), (-0.5, y, 0.5)), lm))
        else:
            d.objects.append(scenes.SphereObject((1.5, 2.0, -1.0), 0.2, lm))
    d.camera = scenes.Camera(eye=(0.0, 1.6, 4.0), target=(0.0, 0.4, 0.0), up=(0.0, 1.0, 0.0),
                             fovv=45.0, fovh=52.0)
    return d


@pytest.mark.parametrize("seed", SEEDS)
def test_wavefront_equals_plain(cuda, seed):
    s = prr.Scene.from_desc(random_scene(seed))
    a, _ = s.render(8, 6, seed=seed, slices=1)
    s.set_wavefront(paths_per_pass=48 * 40 * 2, block_size=64, stack_smem=4)
    b, _ = s.render(8, 6, seed=seed, mode="wavefront")
    assert np.array_equal(a.cpu().numpy().view(np.uint32), b.cpu().numpy().view(np.uint32))
    # adaptive: images and spp maps
    ia, sa = s.render(16, 6, seed=seed, min_spp=2, threshold=0.05)
    ib, sb = s.render(16, 6, seed=seed, min_spp=2, threshold=0.05, mode="wavefront")
    assert np.array_equal(sa.cpu().numpy(), sb.cpu().numpy())
    assert np.array_equal(ia.cpu().numpy().view(np.uint32), ib.cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("seed", SEEDS)
def test_matches_reference(ref, cuda, seed):
    desc = random_scene(seed)
    s = prr.Scene.from_desc(desc)
    img, _ = s.render(64, 6, seed=seed, mode="wavefront")
    rimg, _ = ref.scene(desc).render(6, 64, seed)
    err = rel_mse(img.cpu().numpy(), rimg)
    print(f"random scene {seed}: rMSE vs reference {err:.3e}")
    assert err < REL_MSE_TOL


def test_server_mix_of_random_scenes(cuda):
    """All six scenes resident in one server, requests of mixed size, window,
    depth and spp submitted together: every served image equals a render of
    that request alone (wavefront steps share ray queues across scenes with
    and without sky, lights and glass)."""
    import dataclasses
    descs = [random_scene(seed) for seed in SEEDS]
    scene_objs = [prr.Scene.from_desc(d) for d in descs]
    srv = prr.Server(paths_per_launch=1 << 16)
    for s in scene_objs:
        srv.add_scene(s)
    rng = np.random.default_rng(5)
    jobs = []
    for k in range(14):
        sc = int(rng.integers(0, len(SEEDS)))
        W, H = [(48, 40), (64, 48), (32, 24)][int(rng.integers(0, 3))]
        x0, y0 = int(rng.integers(0, W // 2)), int(rng.integers(0, H // 2))
        win = (x0, y0, int(rng.integers(x0 + 1, W + 1)), int(rng.integers(y0 + 1, H + 1)))
        spp, depth = int(rng.integers(1, 24)), int(rng.integers(1, 8))
        rid = srv.submit(sc, spp, depth, seed=100 + k, window=win, size=(W, H))
        jobs.append((rid, sc, W, H, win, spp, depth, 100 + k))
    for rid, sc, W, H, win, spp, depth, seed in jobs:
        assert srv.wait(rid)["status"] == "done"
        alone = prr.Scene.from_desc(dataclasses.replace(descs[sc], width=W, height=H))
        want, _ = alone.render(spp, depth, seed=seed, window=win, slices=1)
        got = srv.result(rid)
        assert np.array_equal(got.view(np.uint32), want.cpu().numpy().view(np.uint32)), rid
    srv.close()
