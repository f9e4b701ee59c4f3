"""The checked build (libprr_checked.so, compiled with -DPRR_CHECKED): every
node and triangle fetch of the traversal kernels tested against its array,
every stack push against its column's depth, every wavefront queue length and
append against the queue's capacity, failures recorded in the scene's status
words instead of trapping. Run in a child process (PRR_LIBRARY=checked) over
the golden meshes (closest and any hit, every launch shape), a museum-like
level-3 scene (plain and wavefront, fixed and adaptive, a 2-entry shared
stack that spills) and a caustic render: every status word stays 0, and every
output equals the normal build's bit for bit."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import photorealisticrender4610_b200 as prr  # noqa: F401

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def test_checked_build_reports_nothing_and_matches(cuda, tmp_path):
    lib = ROOT / "photorealisticrender4610_b200" / "libprr_checked.so"
    assert lib.exists(), "build the checked library (build.py --checked)"
    env = dict(os.environ, PRR_LIBRARY="checked")
    out_checked = tmp_path / "checked.npz"
    r = subprocess.run([sys.executable, str(ROOT / "tests" / "checked_run.py"), str(out_checked)],
                       env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    sys.path.insert(0, str(ROOT / "tests"))
    import checked_run
    out_plain = tmp_path / "plain.npz"
    checked_run.run(out_plain)  # this process loaded the normal build
    a, b = dict(np.load(out_checked)), dict(np.load(out_plain))
    assert (a["status_checked"] == 1).all() and (b["status_checked"] == 0).all()
    assert not a["status_words"].any(), dict(zip(a["status_cases"], a["status_words"].tolist()))
    assert not b["status_words"].any()
    for k in a:
        if k.startswith("status"):
            continue
        assert np.array_equal(a[k].view(np.uint8), b[k].view(np.uint8)), k
    g = np.load(ROOT / "tests" / "golden" / "mesh.npz")
    for case in ("q1", "q17", "q3000", "degenerate", "axis"):
        for cfg in range(len(checked_run.TRACE_CONFIGS)):
            assert np.array_equal(a[f"{case}_id_{cfg}"], g[f"mesh_{case}_id"]), (case, cfg)
        assert np.array_equal(a[f"{case}_occ"], g[f"mesh_{case}_occ"]), case
