"""Participating media (Volume.hpp, Volume.cpp) against the reference's own
functions compiled into the oracle: the dust / fog presets and the box
entry/exit of Medium::intersect bit for bit (axis-parallel rays, rays from
inside, behind and beside the box included), phaseHG exact on more than
99.5% of inputs and within 3 float ulps elsewhere (libm's powf against a
double pow rounded once), and samplePhaseHG
directions on the same RNG streams within 2e-6 (libm's float cos / sin
against double ones rounded once)."""
import numpy as np
import pytest

import photorealisticrender4610_b200 as prr
from oracle import loader

pytestmark = pytest.mark.skipif(not loader.reference_available(),
                                reason="reference oracle library not built")


@pytest.fixture(scope="module")
def L():
    return loader.ReferenceOracle().L


@pytest.mark.parametrize("name,which", [("dust", 0), ("fog", 1)])
def test_presets_match_reference(L, name, which):
    m = prr.medium_preset(name)
    want = np.empty(4, np.float32)
    L.prr_ref_medium_preset(which, want)
    got = np.array([m["sigma_a"], m["sigma_s"], m["sigma_t"], m["g"]], np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def rays(n, seed):
    rng = np.random.default_rng(seed)
    o = rng.uniform(-3, 3, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    # axis-parallel and zero components, origins on the box faces
    d[: n // 8, 1:] = 0.0
    d[n // 8: n // 4, 0] = 0.0
    d[n // 4: n // 4 + n // 16, 2] = -0.0
    o[n // 2: n // 2 + n // 16, 0] = -1.0
    return np.ascontiguousarray(o), np.ascontiguousarray(d.astype(np.float32))


@pytest.mark.gpu
@pytest.mark.parametrize("bounded", [True, False])
def test_medium_intersect_bit_exact(L, cuda, bounded):
    import torch
    o, d = rays(40000, 3)
    lo = np.array([-1.0, -0.5, -2.0], np.float32)
    hi = np.array([1.0, 1.5, 0.25], np.float32)
    med = dict(prr.medium_preset("fog"), bounded=bounded, bounds=(lo, hi))
    te, tx, hit = prr.medium_intersect(med, torch.from_numpy(o).to(cuda),
                                       torch.from_numpy(d).to(cuda))
    rte, rtx = np.empty(len(o), np.float32), np.empty(len(o), np.float32)
    rhit = np.empty(len(o), np.uint8)
    L.prr_ref_medium_intersect(int(bounded), lo, hi, o, d, len(o), rte, rtx, rhit.ctypes.data)
    assert np.array_equal(hit.cpu().numpy(), rhit)
    assert np.array_equal(te.cpu().numpy().view(np.uint32), rte.view(np.uint32))
    assert np.array_equal(tx.cpu().numpy().view(np.uint32), rtx.view(np.uint32))
    if bounded:
        assert 0.05 < rhit.mean() < 0.9
    else:
        assert rhit.all()


@pytest.mark.gpu
@pytest.mark.parametrize("g", [0.0, 0.6, -0.35, 0.95])
def test_phase_hg(L, cuda, g):
    import torch
    c = np.linspace(-1.0, 1.0, 20001).astype(np.float32)
    got = prr.phase_hg(torch.from_numpy(c).to(cuda), g).cpu().numpy()
    want = np.empty_like(c)
    L.prr_ref_phase_hg(c, len(c), g, want)
    ulps = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
    print(f"phaseHG g={g}: max {ulps.max()} ulp, {(ulps == 0).mean():.4f} exact")
    # the reference's float pow (libm's powf, within about 1 ulp) against a
    # double pow rounded once; where they differ by one ulp of the power, the
    # float quotient moves by up to 3 ulps (1 - 3.6e-7 relative)
    assert ulps.max() <= 3, ulps.max()
    assert (ulps == 0).mean() > 0.995


@pytest.mark.gpu
@pytest.mark.parametrize("g", [0.0, 5e-4, 0.6, -0.35, 0.95])
def test_phase_hg_sample(L, cuda, g):
    import torch
    rng = np.random.default_rng(11)
    wo = rng.normal(size=(30000, 3)).astype(np.float32)
    wo = (wo / np.linalg.norm(wo, axis=1, keepdims=True)).astype(np.float32)
    wo[:100] = (0.0, 0.0, 1.0)
    got = prr.phase_hg_sample(torch.from_numpy(wo).to(cuda), g, seed=7).cpu().numpy()
    want = np.empty_like(wo)
    L.prr_ref_phase_hg_sample(wo, len(wo), g, 7, want)
    assert np.abs(got - want).max() <= 2e-6
    assert (got == want).all(axis=1).mean() > 0.95
    # the mean cosine to wo is g (the HG asymmetry parameter)
    assert abs(float((got * wo).sum(1).mean()) - g) < 0.02
