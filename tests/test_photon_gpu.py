"""Caustic photons on the GPU against the reference's Photon.cpp: the grid
and fixed-radius estimate bit for bit on a given photon array, the traced
photon set against the reference's trace under the same per-photon streams,
and the resulting irradiance within rMSE 1e-3."""
import numpy as np
import pytest
import torch

import photorealisticrender4610_b200 as prr
from photorealisticrender4610_b200 import scenes

pytestmark = pytest.mark.gpu


def rel_mse(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-30))


def random_photons(n, seed):
    rng = np.random.default_rng(seed)
    rec = np.zeros((n, 9), np.float32)
    rec[:, :3] = rng.uniform(-1, 1, (n, 3)) * np.array([1, 0.05, 1])
    rec[:, 3:6] = rng.normal(size=(n, 3))
    rec[:, 6:] = rng.uniform(0, 1e-3, (n, 3))
    q = (rng.uniform(-1, 1, (4000, 3)) * np.array([1, 0.05, 1])).astype(np.float32)
    return rec, q


@pytest.mark.parametrize("radius", [0.02, 0.05, 0.3])
def test_grid_and_estimate_bit_exact(ref, port, cuda, radius):
    rec, q = random_photons(30000, 4)
    pm = prr.PhotonMap().set(rec).build(radius)
    got = pm.gather(q).cpu().numpy()
    want, res = ref.photon_estimate(rec, radius, q)
    assert pm.info()[1] == res
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    again, _ = port.photon_estimate(rec, radius, q)
    assert np.array_equal(again.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("k", [1, 8, 64])
def test_knn_cap_matches_oracle(ref, port, cuda, k):
    """The k-nearest-capped gather against the oracle's brute-force k nearest
    (over the reference's own grid query) bit for bit, including queries with
    ties at the k-th distance: every photon is stored twice at the same spot,
    so the tie rule (lower photon index kept) decides which copy counts."""
    rec, q = random_photons(30000, 5)
    rec = np.concatenate([rec, rec])            # photon i and i + 30000 coincide
    rec[30000:, 6:] *= 1.5                       # ... with different powers
    pm = prr.PhotonMap().set(rec).build(0.05)
    got = pm.gather(q, k_nearest=k).cpu().numpy()
    want, inside = ref.photon_estimate_knn(rec, 0.05, q, k)
    assert (inside > k).sum() > 500
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    again, inside2 = port.photon_estimate_knn(rec, 0.05, q, k)
    assert np.array_equal(inside, inside2)
    assert np.array_equal(again.view(np.uint32), want.view(np.uint32))
    # at most k inside: the fixed-radius estimate itself
    full = pm.gather(q).cpu().numpy()
    few = inside <= k
    assert np.array_equal(got[few].view(np.uint32), full[few].view(np.uint32))


@pytest.fixture(scope="module")
def config4(cuda):
    """Config 4 at its size: 2,000,000 photons emitted on the GPU into the
    caustics scene (glass sphere r=1 over a plane, a level-3 emissive icosphere
    standing in for the point light), radius 0.02."""
    desc = scenes.caustics(1024, 1024)
    s = prr.Scene.from_desc(desc)
    pm = prr.PhotonMap().emit(s, 2_000_000, seed=3)
    rec, owner = pm.export()
    pm.build(0.02)
    return desc, s, pm, rec, owner


def config4_queries(rec, seed=0):
    """10,000 points on a grid over the floor around the caustic and 10,000
    next to stored photons (dense where the caustic is)."""
    rng = np.random.default_rng(seed)
    g = np.linspace(-1.5, 1.5, 100, dtype=np.float32)
    gx, gz = np.meshgrid(g, g)
    grid = np.stack([gx.ravel(), np.zeros(gx.size, np.float32), gz.ravel()], 1)
    near = rec[rng.choice(len(rec), 10_000, replace=False), :3].astype(np.float64)
    near[:, [0, 2]] += rng.normal(0, 0.005, (10_000, 2))
    return np.concatenate([grid, near]).astype(np.float32)


def test_config4_gather_matches_oracle(ref, config4):
    """k = 64 gather at 2M photons / r = 0.02 bit for bit against the oracle's
    k nearest, on 20,000 queries of which well over 1,000 hold more than 64
    photons; k = 0 bit for bit against estimateIrradiance."""
    desc, s, pm, rec, _ = config4
    q = config4_queries(rec)
    got = pm.gather(q, k_nearest=64).cpu().numpy()
    want, inside = ref.photon_estimate_knn(rec, 0.02, q, 64)
    assert len(q) >= 10_000 and (inside > 64).sum() >= 1_000
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    fixed = pm.gather(q).cpu().numpy()
    want0, res = ref.photon_estimate(rec, 0.02, q)
    assert pm.info()[1] == res
    assert np.array_equal(fixed.view(np.uint32), want0.view(np.uint32))


def test_config4_emit_matches_reference_trace(ref, config4):
    """The photon set traced on the GPU against the reference's own trace
    (Photon.cpp:96-188, same per-photon streams) at 2,000,000 photons: the
    irradiance of both sets through the reference estimator at r = 0.02 within
    rMSE 1e-3."""
    desc, s, pm, rec, owner = config4
    rrec, rowner = ref.scene(desc).photon_emit(2_000_000, 3)
    assert len(rec) > 20_000
    assert abs(len(rec) - len(rrec)) <= 0.01 * len(rrec)
    assert (np.diff(owner) >= 0).all()
    q = config4_queries(rrec, seed=1)
    e_gpu, _ = ref.photon_estimate(rec, 0.02, q)
    e_ref, _ = ref.photon_estimate(rrec, 0.02, q)
    assert e_ref.max() > 0
    assert rel_mse(e_gpu, e_ref) < 1e-3


@pytest.mark.parametrize("k,window", [(0, (384, 512, 640, 768)), (64, (448, 560, 576, 688))])
def test_config4_caustic_render_matches_oracle(ref, config4, k, window):
    """The caustic render (1024 x 1024, 32 spp) of a crop over the caustic
    against the oracle's restatement on the reference's own scene, materials
    and estimator (camera ray through castRay's delta chain to the first
    diffuse hit, baseColor / pi * E there) on the same photon array and the same
    per-sample streams: rMSE <= 1e-3."""
    desc, s, pm, rec, _ = config4
    got = pm.render_caustics(s, 32, k_nearest=k, window=window).cpu().numpy()
    want = ref.scene(desc).caustic_render(rec, 0.02, 32, k_nearest=k, window=window)
    assert want.max() > 0
    assert rel_mse(got, want) < 1e-3
    # most pixels agree to the bit (the rest differ through CUDA's own
    # transcendentals in the camera and glass sampling)
    same = (got.view(np.uint32) == want.view(np.uint32)).all(axis=2).mean()
    assert same > 0.9, same


def test_emit_matches_reference_trace(ref, cuda):
    desc = scenes.caustics(64, 64, level=2)
    s = prr.Scene.from_desc(desc)
    n = 200_000
    pm = prr.PhotonMap().emit(s, n, seed=3)
    rec, owner = pm.export()
    rrec, rowner = ref.scene(desc).photon_emit(n, 3)
    assert len(rec) > 1000
    assert abs(len(rec) - len(rrec)) <= 0.01 * len(rrec)
    # the canonical order: photon index ascending
    assert (np.diff(owner) >= 0).all()
    # photons whose record lists agree in length agree record by record
    common = np.intersect1d(owner, rowner)
    assert len(common) > 0.97 * len(np.unique(rowner))
    a = {k: rec[owner == k] for k in common[:2000]}
    b = {k: rrec[rowner == k] for k in common[:2000]}
    same = [k for k in a if len(a[k]) == len(b[k])]
    assert len(same) > 0.97 * len(a)
    close = np.mean([np.allclose(a[k], b[k], rtol=1e-3, atol=1e-5) for k in same])
    assert close > 0.97
    # irradiance on the floor around the caustic, reference estimator on both sets
    g = np.linspace(-1.5, 1.5, 60, dtype=np.float32)
    gx, gz = np.meshgrid(g, g)
    q = np.stack([gx.ravel(), np.zeros(gx.size, np.float32), gz.ravel()], 1).astype(np.float32)
    e_gpu, _ = ref.photon_estimate(rec, 0.1, q)
    e_ref, _ = ref.photon_estimate(rrec, 0.1, q)
    assert rel_mse(e_gpu, e_ref) < 1e-3
    # and the GPU gather on the GPU set equals the reference estimator on it
    pm.build(0.1)
    assert np.array_equal(pm.gather(q).cpu().numpy().view(np.uint32), e_gpu.view(np.uint32))


def test_caustic_render(cuda):
    desc = scenes.caustics(64, 64, level=2)
    s = prr.Scene.from_desc(desc)
    pm = prr.PhotonMap().emit(s, 100_000, seed=1).build(0.05)
    img = pm.render_caustics(s, 4, k_nearest=0).cpu().numpy()
    assert np.isfinite(img).all() and img.max() > 0
    img64 = pm.render_caustics(s, 4, k_nearest=64).cpu().numpy()
    assert np.isfinite(img64).all()


def test_caustic_render_regression_fixture(cuda):
    """The caustic render's images at fixed seeds, bit for bit against the
    fixture written by tests/golden/make_caustics_fixture.py: every pixel is
    the sum of its samples in sample order, however the work is scheduled."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    import make_caustics_fixture as F
    want = np.load(Path(__file__).resolve().parent / "golden" / "caustics_render.npz")
    got = F.render_cases()
    assert got["photons"][0] == want["photons"][0]
    for name, _, _, _ in F.CASES:
        assert np.array_equal(got[name].view(np.uint32), want[name].view(np.uint32)), name


def test_caustic_render_in_chunks(cuda):
    """A render of more (pixel, sample) contributions than one call holds at
    once (1024 x 1024 x 520 > 2^28) runs in chunks of whole samples; its
    pixels equal those of a window small enough for one chunk."""
    desc = scenes.caustics(1024, 1024, level=2)
    s = prr.Scene.from_desc(desc)
    pm = prr.PhotonMap().emit(s, 100_000, seed=2).build(0.05)
    full = pm.render_caustics(s, 520, max_depth=8, seed=4, k_nearest=16).cpu().numpy()
    part = pm.render_caustics(s, 520, max_depth=8, seed=4, k_nearest=16,
                              window=(300, 400, 700, 460)).cpu().numpy()
    assert part.max() > 0
    assert np.array_equal(full[400:460, 300:700].view(np.uint32), part.view(np.uint32))


def test_caustic_render_counts(cuda):
    """The counting caustic render gives the same image bit for bit; its
    counts add up (a gather per diffuse camera hit at most one per sample,
    photons inside the radius among those tested)."""
    desc = scenes.caustics(64, 64, level=2)
    s = prr.Scene.from_desc(desc)
    pm = prr.PhotonMap().emit(s, 100_000, seed=1).build(0.05)
    for k in (0, 16):
        img = pm.render_caustics(s, 4, k_nearest=k).cpu().numpy()
        img2, c = pm.render_caustics_counts(s, 4, k_nearest=k)
        assert np.array_equal(img2.cpu().numpy().view(np.uint32), img.view(np.uint32))
        assert 0 < c["gathers"] <= 64 * 64 * 4 and c["gathers"] <= c["hits"]
        assert 0 < c["photons_inside"] <= c["photons_tested"]
        assert c["dense_gathers"] <= c["gathers"] and (k > 0 or c["dense_gathers"] == 0)


def test_caustic_dense_queue_and_in_place_agree(ref, cuda):
    """Gathers with more than k photons inside are selected by a second kernel
    (a warp per gather) from a queue with room for an eighth of a launch's
    items, at least 1024; beyond that they select in place (one thread each).
    A 16x16 window over the caustic at 16 spp (4,096 items, most of them dense
    gathers) overflows the queue; one-row windows of it fit: the pixels agree
    bit for bit. Both paths against the oracle's render pass on the same
    photons: rMSE <= 1e-3 and most pixels equal to the bit."""
    desc = scenes.caustics(64, 64, level=2)
    s = prr.Scene.from_desc(desc)
    pm = prr.PhotonMap().emit(s, 100_000, seed=1).build(0.5)
    # the 16x16 window of the brightest caustic
    lum = pm.render_caustics(s, 2, k_nearest=0).cpu().numpy().sum(axis=2)
    sums = [(lum[y:y + 16, x:x + 16].sum(), x, y) for y in range(0, 49, 4) for x in range(0, 49, 4)]
    _, x0, y0 = max(sums)
    win = (x0, y0, x0 + 16, y0 + 16)
    full, c = pm.render_caustics_counts(s, 16, k_nearest=4, window=win)
    full = full.cpu().numpy()
    assert c["dense_gathers"] > max(1024, 16 * 16 * 16 // 8), c  # more than the queue holds
    for y in range(y0, y0 + 16, 5):
        row = pm.render_caustics(s, 16, k_nearest=4, window=(x0, y, x0 + 16, y + 1)).cpu().numpy()
        assert np.array_equal(row.view(np.uint32), full[y - y0:y - y0 + 1].view(np.uint32)), y
    rec, _ = pm.export()
    want = ref.scene(desc).caustic_render(rec, 0.5, 16, k_nearest=4, window=win)
    assert want.max() > 0
    assert rel_mse(full, want) < 1e-3
    assert (full.view(np.uint32) == want.view(np.uint32)).all(axis=2).mean() > 0.9


@pytest.mark.parametrize("case", ["doubled", "pile"])
def test_caustic_dense_selection_paths(ref, cuda, case):
    """The dense-gather kernel selects among the photons it collects into
    shared memory within a threshold distance, and walks the whole query box
    instead when no threshold leaves between k and its capacity (512)
    photons. Two photon arrays made from an emitted map: every photon doubled
    (ties at the k-th distance, settled by the photon index, in shared
    memory), and a pile of 3,000 coincident photons at the caustic's densest
    spot (more than the capacity at every threshold that reaches the pile, so
    gathers near it take the box walk, with ties among the pile). Pixels
    against the in-place selection (a window whose dense gathers overflow the
    queue against one-row windows that fit) bit for bit, and against the
    oracle's render pass."""
    desc = scenes.caustics(64, 64, level=2)
    s = prr.Scene.from_desc(desc)
    rec, _ = prr.PhotonMap().emit(s, 100_000, seed=1).build(0.05).export()
    radius, k, spp = 0.3, 16, 16
    if case == "doubled":
        rec = np.concatenate([rec, rec])
        rec[len(rec) // 2:, 6:] *= 1.5
    else:
        p = rec[:, :3].astype(np.float64)
        d2 = ((p[:, None, :] - p[None, ::4, :]) ** 2).sum(axis=2)
        focus = int(np.argmax((d2 < 0.05 ** 2).sum(axis=0))) * 4
        pile = np.repeat(rec[focus:focus + 1], 3000, axis=0)
        pile[:, 6:] *= np.linspace(0.5, 1.5, 3000, dtype=np.float32)[:, None]
        rec = np.concatenate([rec[:focus], pile, rec[focus:]])
    pm = prr.PhotonMap().set(rec).build(radius)
    lum = pm.render_caustics(s, 2, k_nearest=0).cpu().numpy().sum(axis=2)
    sums = [(lum[y:y + 16, x:x + 16].sum(), x, y) for y in range(0, 49, 4) for x in range(0, 49, 4)]
    _, x0, y0 = max(sums)
    win = (x0, y0, x0 + 16, y0 + 16)
    full, c = pm.render_caustics_counts(s, spp, k_nearest=k, window=win)
    full = full.cpu().numpy()
    assert c["dense_gathers"] > max(1024, 16 * 16 * spp // 8), c
    for y in range(y0, y0 + 16, 3):
        row = pm.render_caustics(s, spp, k_nearest=k, window=(x0, y, x0 + 16, y + 1)).cpu().numpy()
        assert np.array_equal(row.view(np.uint32), full[y - y0:y - y0 + 1].view(np.uint32)), y
    want = ref.scene(desc).caustic_render(rec, radius, spp, k_nearest=k, window=win)
    assert want.max() > 0
    assert rel_mse(full, want) < 1e-3
    assert (full.view(np.uint32) == want.view(np.uint32)).all(axis=2).mean() > 0.9


def test_photon_map_counts_its_launches(cuda):
    """prr_photon_launches counts the kernels of every call on the map: a
    one-chunk caustic render launches the sample kernel and the film, plus
    the dense-gather kernel when k > 0."""
    desc = scenes.caustics(64, 64, level=2)
    s = prr.Scene.from_desc(desc)
    pm = prr.PhotonMap()
    assert pm.launches() == 0
    pm.emit(s, 100_000, seed=1)
    n0 = pm.launches()
    assert n0 >= 2
    pm.build(0.05)
    n1 = pm.launches()
    assert n1 >= n0 + 5
    pm.render_caustics(s, 4, k_nearest=0)
    assert pm.launches() == n1 + 2
    pm.render_caustics(s, 4, k_nearest=16)
    assert pm.launches() == n1 + 5
    pm.gather(np.zeros((8, 3), np.float32))
    assert pm.launches() == n1 + 6


def test_gather_radius_boundary_bit_exact(ref, port, cuda):
    """The fixed-radius test decides sqrtf(d.d) <= r on d.d against the
    largest float whose square root is at most r. Photons on rings whose
    radii step through r by a tenth of an ulp at a time (so the computed
    distance falls on either side of r, and on it), around several query
    points: the sums equal the reference estimator's bit for bit, with and
    without the k-nearest cap."""
    rng = np.random.default_rng(11)
    r = np.float32(0.05)
    q = rng.uniform(-1, 1, (8, 3)).astype(np.float32) * np.float32([1, 0.05, 1])
    recs = []
    for j in range(len(q)):
        u = rng.normal(size=(300, 3))
        u = (u / np.linalg.norm(u, axis=1, keepdims=True)).astype(np.float32)
        s = (r * (1 + (np.arange(300, dtype=np.float32) - 150) * np.float32(1e-8))).astype(np.float32)
        rec = np.zeros((300, 9), np.float32)
        rec[:, :3] = q[j] + u * s[:, None]
        rec[:, 6:] = rng.uniform(0, 1e-3, (300, 3))
        recs.append(rec)
    rec = np.concatenate(recs + [random_photons(5000, 12)[0]])
    d = (rec[None, :, :3] - q[:, None, :]).astype(np.float32)
    dist = np.sqrt((d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2])
    assert ((dist == r).sum() > 0) and ((np.abs(dist - r) <= 4e-9).sum() > 100)
    pm = prr.PhotonMap().set(rec).build(float(r))
    want, _ = ref.photon_estimate(rec, float(r), q)
    got = pm.gather(q).cpu().numpy()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    want16, inside = ref.photon_estimate_knn(rec, float(r), q, 16)
    assert (inside > 16).all()
    got16 = pm.gather(q, k_nearest=16).cpu().numpy()
    assert np.array_equal(got16.view(np.uint32), want16.view(np.uint32))


def test_grid_large_map_sorted_in_stages(ref, cuda):
    """A photon map whose sort needs more blocks of 2,048 keys than the
    device holds at once (700,000 photons: 1,048,576 keys, 512 blocks) is
    sorted a launch per stage instead of in one cooperative launch; the
    gathers still equal the reference estimator bit for bit."""
    rec, q = random_photons(700_000, 21)
    pm = prr.PhotonMap().set(rec)
    n0 = pm.launches()
    pm.build(0.02)
    assert pm.launches() - n0 > 20  # the staged sort, not the single launch
    got = pm.gather(q).cpu().numpy()
    want, res = ref.photon_estimate(rec, 0.02, q)
    assert pm.info()[1] == res
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    small = prr.PhotonMap().set(rec[:30_000])
    n1 = small.launches()
    small.build(0.02)
    assert small.launches() - n1 <= 12  # one sort launch among the build's kernels
