"""prr_render_noalloc: the allocation-free render entry point, for callers that
cannot call cudaMalloc while they render (their device memory belongs to
another allocator, or their frame loop must stay out of the CUDA allocator).
Its scratch is a fixed array inside the library instead of cudaMalloc'd
memory. Checked through the C ABI against prr_render (the entry point that
allocates its scratch) on two calls in a row, which also shows that a call
does not depend on what the previous one left in the shared array.

This file sorts last so that a run stopping at its first failure has already
run every other test."""
import ctypes as C

import numpy as np
import pytest
import torch

import photorealisticrender4610_b200 as prr
from photorealisticrender4610_b200 import _lib, scenes
from photorealisticrender4610_b200.api import _ptr, _stream

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("slices", [4, 16])
def test_render_noalloc_matches_render(cuda, slices):
    """With the same settings and the same explicit slice count (which fixes
    the order in which each pixel's samples are summed), the image equals
    prr_render's bit for bit, on two calls in a row."""
    lib = _lib.load()
    desc = scenes.cornell_box(96, 64)
    s = prr.Scene.from_desc(desc)
    for window in [None, (8, 4, 72, 52)]:
        # the allocating entry point, plain mode, same window and slices
        want, _ = s.render(16, 5, seed=1, window=window, slices=slices)
        ref = want.cpu().numpy()
        rs = s._settings(16, 5, 1, None, 0.05, "plain", window, 10.0, 0, slices)
        x0, y0, x1, y1 = window or (0, 0, desc.width, desc.height)
        for call in range(2):
            out = torch.full(((y1 - y0), (x1 - x0), 3), float("nan"), dtype=torch.float32,
                             device=cuda)
            rays = torch.zeros(2, dtype=torch.int64, device=cuda)
            rc = lib.prr_render_noalloc(s.h, C.byref(rs), _ptr(out), _ptr(rays), _stream(None))
            assert rc == 0, _lib.last_error()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert got.shape == ref.shape
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (window, call)
            assert int(rays[0].item()) > 0


def test_render_noalloc_rejects_oversized_windows(cuda):
    lib = _lib.load()
    desc = scenes.cornell_box(1500, 1500)  # 2,250,000 pixels > 2,097,152
    s = prr.Scene.from_desc(desc)
    rs = s._settings(1, 1, 1, None, 0.05, "plain", None, 10.0, 0, 0)
    out = torch.empty((1500, 1500, 3), dtype=torch.float32, device=cuda)
    rc = lib.prr_render_noalloc(s.h, C.byref(rs), _ptr(out), None, _stream(None))
    assert rc == _lib.PRR_OK - 1  # PRR_ERR_INVALID_ARGUMENT
    assert "exceeds" in _lib.last_error()
    rs2 = s._settings(4, 5, 1, 2, 0.05, "plain", (0, 0, 32, 32), 10.0, 0, 0)
    assert lib.prr_render_noalloc(s.h, C.byref(rs2), _ptr(out), None, _stream(None)) == -5
    # an explicit slice count is never cut silently: 1,000,000 pixels x 4 slices
    # do not fit in the 2,097,152 partial sums
    rs3 = s._settings(8, 5, 1, None, 0.05, "plain", (0, 0, 1000, 1000), 10.0, 0, 4)
    rc = lib.prr_render_noalloc(s.h, C.byref(rs3), _ptr(out), None, _stream(None))
    assert rc == _lib.PRR_OK - 1, _lib.last_error()
    assert "slices" in _lib.last_error()
