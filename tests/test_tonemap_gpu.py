"""Display transform on the GPU against the reference's ToneMapping.hpp and
Renderer's exposure / 8-bit quantisation (golden fixtures recorded from the
reference), and the new ACES operator against the oracle's restatement."""
import numpy as np
import pytest
import torch

import photorealisticrender4610_b200 as prr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mapper", [0, 1, 2, 3])
def test_tonemap_matches_reference(golden, cuda, mapper):
    g = golden("tonemap")
    x = torch.from_numpy(g["in"]).to(cuda)
    out, u8 = prr.tonemap(x, mapper)
    out, u8 = out.cpu().numpy(), u8.cpu().numpy()
    want, want8 = g[f"out{mapper}"], g[f"u8_{mapper}"]
    if mapper == 0:  # no transcendental: bit-exact
        assert np.array_equal(out.view(np.uint32), want.view(np.uint32))
    # powf may differ from libm in the last ulp; AgX's outset matrix can cancel
    # O(1) terms, so the bound is absolute: 5e-6 is 1/800 of an 8-bit step
    assert np.allclose(out, want, rtol=1e-5, atol=5e-6)
    diff = np.abs(u8.astype(int) - want8.astype(int))
    assert diff.max() <= 1 and (diff > 0).mean() < 1e-3


def test_tonemap_exposure(golden, cuda):
    g = golden("tonemap")
    out, _ = prr.tonemap(torch.from_numpy(g["in"]).to(cuda), "agx", exposure=0.18)
    assert np.allclose(out.cpu().numpy(), g["out2_exp"], rtol=1e-5, atol=5e-6)


def test_aces_against_oracle(port, cuda):
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.uniform(0, 2, (5000, 3)), rng.uniform(0, 200, (5000, 3))]).astype(
        np.float32)
    out, u8 = prr.tonemap(torch.from_numpy(x).to(cuda), "aces")
    want, want8 = port.tonemap(4, x)
    assert np.allclose(out.cpu().numpy(), want, rtol=1e-5, atol=5e-6)
    assert np.abs(u8.cpu().numpy().astype(int) - want8.astype(int)).max() <= 1
