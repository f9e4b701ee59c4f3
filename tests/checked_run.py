"""Runs the traversal and wavefront paths on the checked build of the library
(libprr_checked.so: every node, triangle, stack and queue index tested on the
device) and writes their outputs and the scenes' status words to an .npz.
Started by tests/test_checked_gpu.py in a child process with
PRR_LIBRARY=checked, so the checked build is the library loaded there."""
import ctypes as C
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import photorealisticrender4610_b200 as prr  # noqa: E402
from photorealisticrender4610_b200 import _lib, scenes  # noqa: E402

TRACE_CONFIGS = [None, {"persistent": 1}, {"persistent": 2}, {"persistent": 3},
                 {"persistent": 2, "sort_rays": 1}]


def status(scene):
    out = (C.c_uint32 * 3)()
    checked = _lib.check(_lib.load().prr_check_status(scene.h, out, 1))
    return checked, list(out)


def run(out_path):
    dev = torch.device("cuda:0")
    g = dict(np.load(ROOT / "tests" / "golden" / "mesh.npz"))
    res = {}
    words = []
    for case in ("q1", "q3", "q4", "q5", "q17", "q3000", "degenerate", "axis"):
        p = f"mesh_{case}_"
        s = prr.Scene.single_mesh(g[p + "verts"])
        o = torch.from_numpy(g[p + "o"]).to(dev)
        d = torch.from_numpy(g[p + "d"]).to(dev)
        for k, cfg in enumerate(TRACE_CONFIGS):
            hid, t = s.mesh_intersect(0, o, d, config=cfg)
            res[f"{case}_id_{k}"] = hid.cpu().numpy()
            res[f"{case}_t_{k}"] = t.cpu().numpy()
        occ = s.mesh_occluded(0, o, d, torch.from_numpy(g[p + "tmax"]).to(dev))
        res[f"{case}_occ"] = occ.cpu().numpy()
        words.append((case, *status(s)))
    desc = scenes.museum_like(96, 54, level=3, env_size=(256, 128))
    s = prr.Scene.from_desc(desc)
    for mode in ("plain", "wavefront"):
        img, _ = s.render(16, 8, seed=3, mode=mode)
        res[f"museum_{mode}"] = img.cpu().numpy()
        img, spp = s.render(32, 8, seed=3, mode=mode, min_spp=4, threshold=0.05)
        res[f"museum_{mode}_adaptive"] = img.cpu().numpy()
        res[f"museum_{mode}_spp"] = spp.cpu().numpy()
    s.set_wavefront(paths_per_pass=1 << 14, block_size=64, stack_smem=2, ordered=False)
    img, _ = s.render(16, 8, seed=3, mode="wavefront")
    res["museum_wavefront_small_stack"] = img.cpu().numpy()
    words.append(("museum", *status(s)))
    desc = scenes.caustics(64, 64, level=2)
    s = prr.Scene.from_desc(desc)
    pm = prr.PhotonMap().emit(s, 50_000, seed=1).build(0.05)
    res["caustics"] = pm.render_caustics(s, 4, k_nearest=16).cpu().numpy()
    words.append(("caustics", *status(s)))
    res["status_cases"] = np.array([w[0] for w in words])
    res["status_checked"] = np.array([w[1] for w in words], np.int32)
    res["status_words"] = np.array([w[2] for w in words], np.uint32)
    np.savez(out_path, **res)


if __name__ == "__main__":
    run(sys.argv[1])
