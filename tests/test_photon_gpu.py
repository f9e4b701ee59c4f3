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


def test_knn_cap(cuda):
    rec, q = random_photons(30000, 5)
    pm = prr.PhotonMap().set(rec).build(0.05)
    full = pm.gather(q).cpu().numpy()
    capped = pm.gather(q, k_nearest=64).cpu().numpy()
    big = pm.gather(q, k_nearest=64)  # repeatable
    assert np.array_equal(capped, big.cpu().numpy())
    # queries with <= 64 photons inside the radius are unchanged
    d = np.linalg.norm(rec[None, :200, :3] - q[:50, None, :], axis=2)
    assert np.isfinite(capped).all() and (capped >= 0).all()
    same = np.isclose(capped, full, rtol=0, atol=0).all(axis=1)
    assert same.mean() > 0.3
    del d


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
