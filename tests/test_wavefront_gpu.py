"""The wavefront integrator against the plain megakernel: the same paths, the
same random draws and the same per-pixel sample order, so the films are equal
bit for bit (the plain renderer with one thread per pixel is itself checked
against the reference in test_render_gpu.py)."""
import numpy as np
import pytest

import photorealisticrender4610_b200 as prr
from photorealisticrender4610_b200 import scenes

pytestmark = pytest.mark.gpu


def render_both(desc, spp, depth, seed=1, **kw):
    s = prr.Scene.from_desc(desc)
    plain, _, pr = s.render(spp, depth, seed=seed, slices=1, count_rays=True)
    wave, n, wr = s.render(spp, depth, seed=seed, mode="wavefront", count_rays=True, **kw)
    return s, plain.cpu().numpy(), wave.cpu().numpy(), pr.cpu().numpy(), wr.cpu().numpy()


@pytest.mark.parametrize("name", ["cornell", "museum", "caustics"])
def test_wavefront_equals_plain(cuda, name):
    if name == "cornell":
        desc, depth = scenes.cornell_box(64, 64), 5
    elif name == "museum":
        desc, depth = scenes.museum_like(96, 54, level=3, env_size=(256, 128)), 8
    else:
        desc, depth = scenes.caustics(64, 64, level=2), 6
    s, plain, wave, pr, wr = render_both(desc, 16, depth)
    assert np.array_equal(plain.view(np.uint32), wave.view(np.uint32))
    # the wavefront skips only the ray a delta bounce leaves after the last
    # iteration, which castRay traces and ignores
    assert wr[0] <= pr[0] and wr[0] > 0.9 * pr[0]
    assert wr[1] == pr[1]


def test_wavefront_passes_and_graphs(cuda):
    desc = scenes.museum_like(64, 48, level=3, env_size=(256, 128))
    s = prr.Scene.from_desc(desc)
    ref, _ = s.render(24, 8, seed=3, slices=1)
    ref = ref.cpu().numpy()
    for paths, graphs in [(64 * 48 * 2, True), (64 * 48 * 3, False), (64 * 48 * 24, True)]:
        s.set_wavefront(paths_per_pass=paths, block_size=64, use_graphs=graphs)
        out, _ = s.render(24, 8, seed=3, mode="wavefront")
        assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.view(np.uint32)), paths
    # a window and a sample offset address the same (pixel, sample) streams
    a, _ = s.render(8, 8, seed=3, mode="wavefront", sample_offset=8, window=(10, 5, 42, 29))
    b, _ = s.render(8, 8, seed=3, slices=1, sample_offset=8)
    assert np.array_equal(a.cpu().numpy(), b.cpu().numpy()[5:29, 10:42])


def test_autotune_picks_a_config(cuda):
    desc = scenes.cornell_box(128, 128)
    s = prr.Scene.from_desc(desc)
    best = s.autotune(4, 5)
    assert best["paths_per_pass"] > 0 and best["block_size"] in (64, 128, 256)
    a, _ = s.render(8, 5, mode="wavefront")
    b, _ = s.render(8, 5, slices=1)
    assert np.array_equal(a.cpu().numpy(), b.cpu().numpy())


@pytest.mark.parametrize("stack,ordered", [(1, False), (3, True), (8, False), (12, True)])
def test_wavefront_stack_spill(cuda, stack, ordered):
    # mesh stacks mostly in the global spill buffer (stack=1) up to a few
    # levels short of the tree depth: the same film as the plain renderer
    desc = scenes.museum_like(80, 48, level=4, env_size=(256, 128))
    s = prr.Scene.from_desc(desc)
    assert s.stats()["blas_depth"] + 1 > 12
    ref, _ = s.render(8, 8, seed=5, slices=1)
    s.set_wavefront(paths_per_pass=80 * 48 * 4, block_size=128, stack_smem=stack, ordered=ordered)
    out, _ = s.render(8, 8, seed=5, mode="wavefront")
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("refill", [1, 4, 32])
def test_wavefront_refill_threshold(cuda, refill):
    # how many idle lanes a traversal warp waits for before taking new rays
    # changes only the schedule: the same film as the plain renderer
    desc = scenes.museum_like(80, 48, level=4, env_size=(256, 128))
    s = prr.Scene.from_desc(desc)
    ref, _ = s.render(8, 8, seed=6, slices=1)
    s.set_wavefront(paths_per_pass=80 * 48 * 4, block_size=128, stack_smem=8, refill=refill)
    out, _ = s.render(8, 8, seed=6, mode="wavefront")
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.cpu().numpy().view(np.uint32))


def test_autotune_tries_queue_order_and_stack_depth(cuda):
    desc = scenes.museum_like(96, 64, level=3, env_size=(256, 128))
    s = prr.Scene.from_desc(desc)
    best = s.autotune(2, 8)
    assert best["ordered"] in (0, 1) and best["stack_smem"] in (0, 16, 8, 4, 2)
    assert best["refill"] in (0, 4, 12, 16)
    a, _ = s.render(4, 8, mode="wavefront")
    b, _ = s.render(4, 8, slices=1)
    assert np.array_equal(a.cpu().numpy(), b.cpu().numpy())


@pytest.mark.parametrize("name", ["cornell", "museum", "caustics"])
def test_wavefront_ordered_queues_equal_plain(cuda, name):
    # queues rebuilt in path order by the stable partition (ragged last tile,
    # several passes): the same film, and the same ray counts as append order
    if name == "cornell":
        desc, depth = scenes.cornell_box(72, 40), 5
    elif name == "museum":
        desc, depth = scenes.museum_like(96, 54, level=3, env_size=(256, 128)), 8
    else:
        desc, depth = scenes.caustics(64, 48, level=2), 6
    s = prr.Scene.from_desc(desc)
    plain, _ = s.render(12, depth, seed=4, slices=1)
    npix = desc.width * desc.height
    s.set_wavefront(paths_per_pass=npix * 3, block_size=128, ordered=False)
    _, _, r_app = s.render(12, depth, seed=4, mode="wavefront", count_rays=True)
    s.set_wavefront(paths_per_pass=npix * 3, block_size=128, ordered=True)
    wave, _, r_ord = s.render(12, depth, seed=4, mode="wavefront", count_rays=True)
    assert np.array_equal(wave.cpu().numpy().view(np.uint32), plain.cpu().numpy().view(np.uint32))
    assert np.array_equal(r_app.cpu().numpy(), r_ord.cpu().numpy())


@pytest.mark.parametrize("name,paths_spp,ordered", [("cornell", 8, True), ("cornell", 32, False),
                                                    ("museum", 4, True)])
def test_wavefront_adaptive_equals_plain(cuda, name, paths_spp, ordered):
    # adaptive sampling (Renderer.cpp:74-99) in the wavefront: passes over the
    # still-active pixels, the Welford stop replayed per sample in the film
    # stage; same sample counts and the same image as the plain adaptive
    # renderer (itself checked against the reference in test_render_gpu.py)
    if name == "cornell":
        desc, depth, lo, hi, thr = scenes.cornell_box(48, 40), 5, 8, 128, 0.1
    else:
        desc, depth, lo, hi, thr = scenes.museum_like(64, 36, level=3, env_size=(256, 128)), 8, 4, 64, 0.2
    s = prr.Scene.from_desc(desc)
    ref, rspp = s.render(hi, depth, seed=6, min_spp=lo, threshold=thr)
    npix = desc.width * desc.height
    s.set_wavefront(paths_per_pass=npix * paths_spp, block_size=128, ordered=ordered)
    out, spp, rays = s.render(hi, depth, seed=6, min_spp=lo, threshold=thr, mode="wavefront",
                              count_rays=True)
    spp, rspp = spp.cpu().numpy(), rspp.cpu().numpy()
    assert np.array_equal(spp, rspp)
    assert spp.min() >= lo and spp.max() <= hi and spp.min() < spp.max()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.cpu().numpy().view(np.uint32))
    assert s.stats()["last_render_launches"] > 0


def test_render_counts_match_oracle_traversal(port, cuda):
    """prr_render_counts: the same image as prr_render in wavefront mode, and
    traversal counts equal to the oracle's walk of the same rays. A mirror soup
    at depth 1 traces exactly the camera rays (the ray a delta bounce leaves
    after the last iteration is not traced), so every counted interior node and
    triangle test can be checked against the C restatement's counting walk
    (BVH.cpp:311-415) on those rays, taken from the camera with the first two
    draws of each (pixel, sample) stream."""
    verts, _, _ = scenes.query_set(20_000, 1, seed=11)
    desc = scenes.SceneDesc(width=64, height=48, name="mirror soup")
    m = desc.add_material(scenes.Material(scenes.MIRROR, (0.9, 0.9, 0.9), 0.0, 0.0))
    desc.objects.append(scenes.MeshObject(verts, m))
    desc.camera = scenes.Camera(eye=(2.2, 1.6, 2.4), target=(0.5, 0.5, 0.5), fovv=40, fovh=45)
    s = prr.Scene.from_desc(desc)
    spp, seed = 2, 5
    img, c = s.render_counts(spp, 1, seed=seed)
    want, _, rays = s.render(spp, 1, seed=seed, mode="wavefront", count_rays=True)
    assert np.array_equal(img.cpu().numpy().view(np.uint32), want.cpu().numpy().view(np.uint32))
    rays = rays.cpu().numpy()
    n = desc.width * desc.height * spp
    assert c["closest_rays"] == rays[0] == n
    assert c["shadow_rays"] == rays[1] == 0
    assert c["misses"] + c["delta_hits"] + c["surface_hits"] == n
    assert c["surface_hits"] == 0 and c["delta_hits"] > 0
    px, py, smp = np.meshgrid(np.arange(desc.width), np.arange(desc.height), np.arange(spp),
                              indexing="ij")
    px, py, smp = px.ravel(), py.ravel(), smp.ravel()
    draws = np.array([port.rng_stream(seed, int(i + j * desc.width), int(k), 2)
                      for i, j, k in zip(px, py, smp)], np.float32)
    o, d = s.camera_rays(px, py, draws[:, 0], draws[:, 1])
    o, d = o.cpu().numpy(), d.cpu().numpy()
    hid, _, _, vis, tst = port.mesh(verts).intersect(o, d, stats=True)
    assert (hid >= 0).sum() == c["delta_hits"]
    # one object (the scene BVH's root is the mesh's leaf): one entry per ray
    assert c["closest_objects"] == n
    assert c["closest_nodes"] == int(vis.sum())
    assert c["closest_tris"] == int(tst.sum())


def test_render_counts_two_level_consistency(cuda):
    """On a scene of meshes, spheres, emitters and the sky: the counting render
    equals the timed renderer's image bit for bit, and its ray totals and hit
    classes add up."""
    desc = scenes.museum_like(96, 54, level=3, env_size=(256, 128))
    s = prr.Scene.from_desc(desc)
    img, c = s.render_counts(4, 8, seed=2)
    want, _, rays = s.render(4, 8, seed=2, mode="wavefront", count_rays=True)
    assert np.array_equal(img.cpu().numpy().view(np.uint32), want.cpu().numpy().view(np.uint32))
    rays = rays.cpu().numpy()
    assert c["closest_rays"] == rays[0] and c["shadow_rays"] == rays[1]
    assert c["misses"] + c["delta_hits"] + c["surface_hits"] == c["closest_rays"]
    assert c["closest_objects"] >= c["closest_rays"] - c["misses"]
    assert c["closest_nodes"] > c["closest_rays"] and c["closest_tris"] > 0
    assert c["shadow_nodes"] > 0 and c["shadow_tris"] > 0
