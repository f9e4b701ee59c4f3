"""The render server: continuous batching over resident scenes, on both step
integrators. Each request's image is the same alone as in a mix (bit for
bit); on wavefront steps (all running requests' paths in one set of ordered
ray queues) it equals the plain renderer bit for bit, on megakernel steps
within float-summation tolerance (chunk sums); admission respects the device
budget; injected allocation failures, cancellations and timeouts are made on
the host and leave the server serving."""
import dataclasses

import numpy as np
import pytest
import torch

import photorealisticrender4610_b200 as prr
from photorealisticrender4610_b200 import scenes

pytestmark = pytest.mark.gpu

JOBS = [  # (scene, spp, depth, seed, window)
    (0, 16, 5, 1, None),
    (1, 32, 8, 2, None),
    (2, 8, 6, 3, (8, 8, 40, 40)),
    (1, 5, 8, 4, (0, 0, 48, 30)),
    (0, 64, 5, 5, None),
    (2, 12, 6, 6, None),
]


@pytest.fixture(scope="module")
def scene_set(cuda):
    descs = [scenes.cornell_box(64, 64), scenes.museum_like(96, 54, level=3, env_size=(256, 128)),
             scenes.caustics(64, 64, level=2)]
    return [prr.Scene.from_desc(d) for d in descs]


def make_server(scene_set, **kw):
    srv = prr.Server(samples_per_step=kw.pop("samples_per_step", 8192), **kw)
    for s in scene_set:
        srv.add_scene(s)
    return srv


@pytest.mark.parametrize("integrator,paths_per_launch", [
    ("wavefront", 0), ("wavefront", 40000), ("megakernel", 0)])
def test_same_alone_and_in_mix(scene_set, integrator, paths_per_launch):
    kw = dict(integrator=integrator, paths_per_launch=paths_per_launch)
    alone, alone_rays = [], []
    for sc, spp, depth, seed, win in JOBS:
        srv = make_server(scene_set, **kw)
        rid = srv.submit(sc, spp, depth, seed=seed, window=win)
        info = srv.wait(rid)
        assert info["status"] == "done"
        alone.append(srv.result(rid).copy())
        alone_rays.append(info["rays"])
        srv.close()
    srv = make_server(scene_set, **kw)
    rids = []
    for k, (sc, spp, depth, seed, win) in enumerate(JOBS):
        if k % 2 == 0:  # half of them into device memory
            W, H = scene_set[sc].desc.width, scene_set[sc].desc.height
            x0, y0, x1, y1 = win or (0, 0, W, H)
            out = torch.empty((y1 - y0, x1 - x0, 3), dtype=torch.float32, device="cuda")
            rids.append(srv.submit(sc, spp, depth, seed=seed, window=win, out=out))
        else:
            rids.append(srv.submit(sc, spp, depth, seed=seed, window=win))
    infos = [srv.wait(r) for r in rids]
    assert all(i["status"] == "done" for i in infos)
    # requests overlapped on the device: all of them where steps are small;
    # with 16M-path steps the first one may finish before the last arrives
    if integrator == "megakernel" or paths_per_launch:
        assert max(i["admit_s"] for i in infos) < min(i["done_s"] for i in infos)
    else:
        assert any(a["admit_s"] < b["done_s"] and b["admit_s"] < a["done_s"]
                   for k, a in enumerate(infos) for b in infos[k + 1:])
    for k, rid in enumerate(rids):
        got = srv.result(rid)
        got = got.cpu().numpy() if hasattr(got, "cpu") else got
        assert np.array_equal(got.view(np.uint32), alone[k].view(np.uint32)), k
        assert infos[k]["rays"] == alone_rays[k] > 0, k
    st = srv.stats()
    assert st["completed"] == len(JOBS) and st["failed"] == 0 and st["steps"] > 0
    assert st["rays"] == sum(alone_rays)
    # at least one kernel per step and one resolve per finished request
    assert st["launches"] >= st["steps"] + len(JOBS)
    srv.close()
    # and each equals the plain renderer: bit for bit where samples are added
    # one by one (wavefront), up to how the sums are grouped otherwise
    for k, (sc, spp, depth, seed, win) in enumerate(JOBS):
        ref, _ = scene_set[sc].render(spp, depth, seed=seed, window=win, slices=1)
        ref = ref.cpu().numpy()
        if integrator == "wavefront":
            assert np.array_equal(alone[k].view(np.uint32), ref.view(np.uint32)), k
        else:
            assert np.allclose(alone[k], ref, rtol=1e-5, atol=1e-6), k


@pytest.mark.parametrize("integrator", ["wavefront", "megakernel"])
def test_budget_faults_cancel_timeout(scene_set, integrator):
    scene_bytes = sum(s.stats()["device_bytes"] for s in scene_set)
    # room for one 64x64 request at a time (film + host staging = 24 bytes/pixel)
    srv = make_server(scene_set, budget_bytes=scene_bytes + 64 * 64 * 24 + 100,
                      fail_every_nth_admission=3, integrator=integrator)
    rids = [srv.submit(0, 8, 5, seed=k) for k in range(6)]
    infos = [srv.wait(r) for r in rids]
    st = [i["status"] for i in infos]
    assert st == ["done", "done", "failed", "done", "done", "failed"], st
    assert infos[2]["error"] == -3  # PRR_ERR_OUT_OF_MEMORY, injected on the host
    done = [i for i in infos if i["status"] == "done"]
    for a, b in zip(done, done[1:]):  # the budget admits one at a time
        assert b["admit_s"] >= a["done_s"]
    with pytest.raises(prr.PrrError, match="BUDGET"):
        srv.submit(1, 4, 8)  # 96x54 never fits
    # cancel a queued request, time out on a long one
    long_id = srv.submit(0, 1 << 16, 5, seed=9)  # 16 or more steps
    queued = srv.submit(0, 8, 5, seed=10)
    srv.cancel(queued)
    assert srv.wait(queued)["status"] == "cancelled"
    with pytest.raises(prr.PrrError, match="TIMEOUT"):
        srv.wait(long_id, timeout=0.0)
    srv.cancel(long_id)
    assert srv.wait(long_id)["status"] == "cancelled"
    ok = srv.submit(0, 8, 5, seed=0)
    assert srv.wait(ok)["status"] == "done"
    assert np.array_equal(srv.result(ok), srv.result(rids[0]))
    srv.close()


def test_other_resolution(scene_set):
    """A request at another resolution of the scene's camera equals the
    renderer's output for the same camera at that resolution."""
    srv = make_server(scene_set)
    rid = srv.submit(1, 12, 8, seed=7, size=(120, 70), window=(10, 5, 90, 61))
    assert srv.wait(rid)["status"] == "done"
    got = srv.result(rid)
    srv.close()
    s = prr.Scene.from_desc(dataclasses.replace(scene_set[1].desc, width=120, height=70))
    ref, _ = s.render(12, 8, seed=7, window=(10, 5, 90, 61), slices=1)
    assert np.array_equal(got.view(np.uint32), ref.cpu().numpy().view(np.uint32))


def test_unknown_integrator_rejected():
    with pytest.raises(ValueError):
        prr.Server(integrator="rasterizer")


def test_short_request_overtakes_long_one(scene_set):
    """Wavefront steps split their paths among the running requests, most of
    them to the requests with the least work left: a short request submitted
    after a long one finishes first, and both images equal the renderer's."""
    srv = make_server(scene_set, paths_per_launch=1 << 16)
    big = srv.submit(0, 256, 5, seed=3)  # 64x64x256 = 1M paths: 16+ steps
    small = srv.submit(0, 16, 5, seed=4, window=(0, 0, 16, 16))
    ib, is_ = srv.wait(big), srv.wait(small)
    assert ib["status"] == is_["status"] == "done"
    assert is_["done_s"] < ib["done_s"]
    for rid, (spp, seed, win) in ((big, (256, 3, None)), (small, (16, 4, (0, 0, 16, 16)))):
        ref, _ = scene_set[0].render(spp, 5, seed=seed, window=win, slices=1)
        assert np.array_equal(srv.result(rid).view(np.uint32), ref.cpu().numpy().view(np.uint32))
    assert srv.stats()["steps"] >= 16
    srv.close()
