"""Regenerates the golden fixtures in tests/golden/ by running the reference
renderer's own code (oracle/_ref/libprr_ref.so: the reference sources compiled
in place with IEEE flags and the counter-keyed RNG injected).

    python tests/golden/make_golden.py

Needs the reference tree on this host (oracle/Makefile builds the library).
The fixtures are small; the GPU parity tests check larger cases against the
oracle directly.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.loader import ReferenceOracle, build_reference  # noqa: E402
from photorealisticrender4610_b200 import scenes  # noqa: E402

OUT = Path(__file__).resolve().parent


def mesh_cases():
    """(name, verts, o, d) cases for the mesh micro-path."""
    cases = []
    for ntri, nray, seed in [(1, 512, 11), (3, 512, 12), (4, 512, 13), (5, 512, 14),
                             (17, 1024, 15), (3000, 8192, 7)]:
        v, o, d = scenes.query_set(ntri, nray, seed=seed, jitter=0.05 if ntri < 20 else 0.005)
        cases.append((f"q{ntri}", v, o, d))
    # all centroids coincide: median splits without reordering
    v = np.tile(np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]], np.float32), (37, 1))
    rng = np.random.default_rng(3)
    o = np.column_stack([rng.uniform(-0.2, 1.2, 512), rng.uniform(-0.2, 1.2, 512),
                         np.full(512, 2.0)]).astype(np.float32)
    d = np.tile(np.array([[0, 0, -1]], np.float32), (512, 1))
    cases.append(("degenerate", v, o, d))
    # axis-aligned rays (zero direction components -> infinite inverse) into a grid
    v, _, _ = scenes.query_set(500, 1, seed=21)
    g = np.linspace(0.0, 1.0, 16, dtype=np.float32)
    gx, gy = np.meshgrid(g, g)
    o = np.column_stack([gx.ravel(), gy.ravel(), np.full(gx.size, -1.0, np.float32)])
    d = np.tile(np.array([[0, 0, 1]], np.float32), (gx.size, 1))
    o2 = np.column_stack([np.full(gx.size, -1.0, np.float32), gx.ravel(), gy.ravel()])
    d2 = np.tile(np.array([[1, 0, 0]], np.float32), (gx.size, 1))
    cases.append(("axis", v, np.vstack([o, o2]).astype(np.float32),
                  np.vstack([d, d2]).astype(np.float32)))
    return cases


def main():
    build_reference()
    ref = ReferenceOracle()
    data = {}

    # RNG streams
    keys = np.array([[1, 0, 0], [1, 5, 7], [123456789, 4000000, 3], [2**63 + 5, 77, 0xFFFFFFFF]],
                    np.uint64)
    data["rng_keys"] = keys
    data["rng_draws"] = np.stack([ref.rng_stream(int(k[0]), int(k[1]), int(k[2]), 64)
                                  for k in keys])

    # mesh micro-path (BVHAccel(., 4) + Intersect / IntersectP)
    for name, v, o, d in mesh_cases():
        m = ref.mesh(v)
        nodes = m.nodes()
        hid, t = m.intersect(o, d)
        tmax = np.random.default_rng(len(v)).uniform(0.3, 4.0, len(o)).astype(np.float32)
        occ = m.occluded(o, d, tmax)
        area, bvh_area = m.areas()
        data[f"mesh_{name}_verts"] = v
        data[f"mesh_{name}_o"] = o
        data[f"mesh_{name}_d"] = d
        data[f"mesh_{name}_tmax"] = tmax
        data[f"mesh_{name}_id"] = hid
        data[f"mesh_{name}_t"] = t
        data[f"mesh_{name}_occ"] = occ
        data[f"mesh_{name}_area"] = np.array([area, bvh_area], np.float32)
        for k, a in nodes.items():
            data[f"mesh_{name}_{k}"] = a
    np.savez_compressed(OUT / "mesh.npz", **data)
    print("mesh.npz", sum(a.nbytes for a in data.values()))

    # Cornell box: scene BVH, two-level closest/any hit, light sampling
    data = {}
    desc = scenes.cornell_box(64, 64)
    rs = ref.scene(desc)
    tl = rs.nodes(-1)
    for k, a in tl.items():
        data[f"tlas_{k}"] = a
    rng = np.random.default_rng(5)
    n = 4096
    o = rng.uniform(-0.95, 0.95, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    px = rng.integers(0, 64, n).astype(np.int32)
    py = rng.integers(0, 64, n).astype(np.int32)
    xo = rng.random(n).astype(np.float32)
    yo = rng.random(n).astype(np.float32)
    co, cd = rs.camera_rays(px, py, xo, yo)
    O = np.vstack([o, co])
    D = np.vstack([d, cd])
    obj, prim, t, geo = rs.intersect(O, D, geo=True)
    tmax = rng.uniform(0.2, 3.0, len(O)).astype(np.float32)
    occ = rs.occluded(O, D, tmax)
    lp, ln, lpdf = rs.sample_light(9, 2048)
    data.update(o=O, d=D, obj=obj, prim=prim, t=t, geo=geo, tmax=tmax, occ=occ,
                cam_px=px, cam_py=py, cam_xo=xo, cam_yo=yo, cam_o=co, cam_d=cd,
                light_pos=lp, light_nrm=ln, light_pdf=lpdf,
                emit_area=np.array([rs.emit_area()], np.float32))
    for k in range(len(desc.objects)):
        if desc.objects[k].kind == "mesh":
            for kk, a in rs.nodes(k).items():
                data[f"obj{k}_{kk}"] = a
    # per-sample radiance in lockstep (same RNG stream per (pixel, sample))
    sx = rng.integers(0, 64, 2048).astype(np.int32)
    sy = rng.integers(0, 64, 2048).astype(np.int32)
    ss = rng.integers(0, 64, 2048).astype(np.int32)
    rad, draws = rs.cast_samples(5, 1, sx, sy, ss)
    data.update(samp_px=sx, samp_py=sy, samp_s=ss, samp_rgb=rad, samp_draws=draws)
    img, cnt = rs.render(5, 16, 1)
    data["render16"] = img
    np.savez_compressed(OUT / "cornell.npz", **data)
    print("cornell.npz", sum(a.nbytes for a in data.values()))

    # tone mapping
    data = {}
    g = np.concatenate([np.linspace(0, 1.5, 200), np.geomspace(1.5, 200, 100),
                        [0.0, 1e-6, 0.0031308, 0.18, 1.0, np.inf, -1.0, np.nan]])
    rgb = np.stack(np.meshgrid(g[::13], g[::17], g[::19]), -1).reshape(-1, 3).astype(np.float32)
    rgb = np.vstack([rgb, np.repeat(g[:, None], 3, 1)]).astype(np.float32)
    data["in"] = rgb
    for mapper in range(4):
        out, u8 = ref.tonemap(mapper, rgb, exposure=1.0)
        data[f"out{mapper}"] = out
        data[f"u8_{mapper}"] = u8
    out, u8 = ref.tonemap(2, rgb, exposure=0.18)
    data["out2_exp"] = out
    np.savez_compressed(OUT / "tonemap.npz", **data)

    # environment map: load via .hdr, CDF, lookups, importance samples
    data = {}
    desc = scenes.cornell_box(32, 32)
    desc.env = scenes.procedural_sky(128, 64)
    rs = ref.scene(desc)
    px, cdf, marg, tot = rs.env_export()
    data.update(env=desc.env, pixels=px, cdf=cdf, marginal=marg, total=np.array([tot]))
    dirs = np.random.default_rng(8).normal(size=(2048, 3))
    dirs = (dirs / np.linalg.norm(dirs, axis=1, keepdims=True)).astype(np.float32)
    rgb, pdf = rs.env_eval(dirs)
    sd, spdf = rs.env_importance(17, 2048)
    data.update(dirs=dirs, eval_rgb=rgb, eval_pdf=pdf, is_dirs=sd, is_pdf=spdf)
    np.savez_compressed(OUT / "env.npz", **data)
    print("done")


if __name__ == "__main__":
    main()
