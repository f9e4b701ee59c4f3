"""Writes tests/golden/caustics_render.npz: caustic renders (prr_render_caustics)
of the small caustics scene at fixed seeds, as a bit-for-bit regression
fixture for changes to how the caustic render kernel schedules its work (the
image is defined by per-pixel sums of the samples in sample order, whatever
the schedule). Generated on a GPU (last when the k-nearest estimate came to add
its kept photons in the grid query's order):

    python tests/golden/make_caustics_fixture.py [out.npz]

The reference renderer has no caustic render (its castRay never gathers from
the photon map), so the photon map itself is checked against the reference
elsewhere (tests/test_photon_gpu.py); this fixture pins the render on top.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import photorealisticrender4610_b200 as prr  # noqa: E402
from photorealisticrender4610_b200 import scenes  # noqa: E402

CASES = [  # (name, spp, k_nearest, window)
    ("k0", 8, 0, None),
    ("k64", 8, 64, None),
    ("k8_window", 5, 8, (9, 14, 51, 47)),
]


def render_cases():
    desc = scenes.caustics(64, 64, level=2)
    s = prr.Scene.from_desc(desc)
    pm = prr.PhotonMap().emit(s, 100_000, seed=1).build(0.05)
    out = {}
    for name, spp, k, win in CASES:
        out[name] = pm.render_caustics(s, spp, max_depth=8, seed=7, k_nearest=k,
                                       window=win).cpu().numpy()
    out["photons"] = np.array([pm.info()[0]], np.int64)
    return out


if __name__ == "__main__":
    dst = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).with_name("caustics_render.npz")
    np.savez_compressed(dst, **render_cases())
    print("wrote", dst)
