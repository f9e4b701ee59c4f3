"""GPU parity of the traversal kernels through the C ABI: closest hit and any
hit on one mesh (BVHAccel::Intersect / IntersectP) and on a two-level scene
(Scene::intersect / intersectP), bit-exact against fixtures recorded from the
reference and against the C restatement at the full query-set size."""
import numpy as np
import pytest
import torch

import photorealisticrender4610_b200 as prr
from photorealisticrender4610_b200 import scenes

from test_oracle import MESH_CASES, NODE_KEYS

pytestmark = pytest.mark.gpu


def dev(a, cuda):
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


@pytest.mark.parametrize("case", MESH_CASES)
@pytest.mark.parametrize("config", [None, {"persistent": 1}, {"block_size": 64},
                                    {"persistent": 2}, {"persistent": 2, "batch": 1},
                                    {"persistent": 2, "batch": 32, "block_size": 64},
                                    {"persistent": 3}, {"persistent": 3, "leaf_batch": 1},
                                    {"persistent": 3, "leaf_batch": 32, "batch": 4},
                                    {"persistent": 3, "leaf_batch": 8, "block_size": 256},
                                    {"persistent": 2, "sort_rays": 1},
                                    {"persistent": 2, "batch": 12, "sort_rays": 2},
                                    {"persistent": 1, "sort_rays": 3},
                                    {"persistent": 2, "sort_rays": 4},
                                    {"persistent": 2, "sort_rays": 5},
                                    {"sort_rays": 1}, {"persistent": 3, "sort_rays": 1}])
def test_mesh_intersect_bit_exact(golden, cuda, case, config):
    g = golden("mesh")
    p = f"mesh_{case}_"
    s = prr.Scene.single_mesh(g[p + "verts"])
    nodes = s.export_nodes(0)
    for k in NODE_KEYS:
        assert np.array_equal(nodes[k], g[p + k]), k
    hid, t = s.mesh_intersect(0, dev(g[p + "o"], cuda), dev(g[p + "d"], cuda), config=config)
    torch.cuda.synchronize()
    assert np.array_equal(hid.cpu().numpy(), g[p + "id"])
    assert np.array_equal(t.cpu().numpy().view(np.uint32), g[p + "t"].view(np.uint32))


@pytest.mark.parametrize("case", MESH_CASES)
def test_mesh_occluded_bit_exact(golden, cuda, case):
    g = golden("mesh")
    p = f"mesh_{case}_"
    s = prr.Scene.single_mesh(g[p + "verts"])
    occ = s.mesh_occluded(0, dev(g[p + "o"], cuda), dev(g[p + "d"], cuda),
                          dev(g[p + "tmax"], cuda))
    assert np.array_equal(occ.cpu().numpy(), g[p + "occ"])


@pytest.mark.parametrize("config", [None, {"persistent": 2}, {"persistent": 3},
                                    {"persistent": 2, "batch": 12, "sort_rays": 1}])
def test_mesh_intersect_host_buffers(golden, cuda, config):
    g = golden("mesh")
    p = "mesh_q3000_"
    s = prr.Scene.single_mesh(g[p + "verts"])
    hid, t = s.mesh_intersect_host(0, g[p + "o"], g[p + "d"], config=config)
    assert np.array_equal(hid, g[p + "id"])
    assert np.array_equal(t.view(np.uint32), g[p + "t"].view(np.uint32))
    # several chunks over the pipeline's streams (1,200,000 rays: 512k, 176k,
    # 512k), pinned buffers, against the device-array call
    v, o, d = scenes.query_set(20_000, 1_200_000, seed=5)
    s2 = prr.Scene.single_mesh(v)
    import torch
    ho = torch.from_numpy(o).pin_memory().numpy()
    hd = torch.from_numpy(d).pin_memory().numpy()
    hid2, t2 = s2.mesh_intersect_host(0, ho, hd, config=config)
    did, dt = s2.mesh_intersect(0, dev(o, cuda), dev(d, cuda))
    assert np.array_equal(hid2, did.cpu().numpy())
    assert np.array_equal(t2.view(np.uint32), dt.cpu().numpy().view(np.uint32))


def test_query_set_full_size_against_restatement(port, cuda):
    """1M triangles x 4,194,304 rays: hit IDs and t bit-exact against the C
    restatement (itself pinned to the reference), the fp64 re-solve equal to
    the restatement's fp64 MT, and within 1e-6 relative of it by construction."""
    v, o, d = scenes.query_set(1_000_000, 4_194_304, seed=1)
    s = prr.Scene.single_mesh(v)
    st = s.stats()
    assert st["n_triangles"] == 1_000_000
    hid, t, t64 = s.mesh_intersect(0, dev(o, cuda), dev(d, cuda), t64=True)
    hid, t, t64 = hid.cpu().numpy(), t.cpu().numpy(), t64.cpu().numpy()
    m = port.mesh(v)
    rh, rt, rt64 = m.intersect(o, d)
    assert np.array_equal(hid, rh)
    assert np.array_equal(t.view(np.uint32), rt.view(np.uint32))
    hit = hid >= 0
    assert hit.mean() > 0.99
    assert np.array_equal(t64[hit], rt64[hit])
    assert np.isnan(t64[~hit]).all()
    # the persistent launch shapes give the same answer
    for cfg in ({"persistent": 1}, {"persistent": 2}, {"persistent": 2, "batch": 16},
                {"persistent": 3}, {"persistent": 3, "leaf_batch": 24},
                {"persistent": 2, "batch": 12, "sort_rays": 1},
                {"persistent": 2, "batch": 12, "sort_rays": 2},
                {"persistent": 2, "batch": 12, "sort_rays": 3},
                {"persistent": 2, "batch": 8, "sort_rays": 4},
                {"persistent": 2, "batch": 8, "sort_rays": 5}):
        hid2, t2, t642 = s.mesh_intersect(0, dev(o, cuda), dev(d, cuda), t64=True, config=cfg)
        assert np.array_equal(hid2.cpu().numpy(), rh)
        assert np.array_equal(t2.cpu().numpy().view(np.uint32), rt.view(np.uint32))
        assert np.array_equal(t642.cpu().numpy()[hit], rt64[hit])
    # any hit agrees with closest hit at tmax just beyond / before the hit
    tm = np.where(hit, rt * np.float32(1.0001), np.float32(10.0)).astype(np.float32)
    occ = s.mesh_occluded(0, dev(o, cuda), dev(d, cuda), dev(tm, cuda)).cpu().numpy()
    assert np.array_equal(occ, m.occluded(o, d, tm))
    assert occ[hit].mean() > 0.999


def test_scene_intersect_cornell(golden, cuda):
    g = golden("cornell")
    desc = scenes.cornell_box(64, 64)
    s = prr.Scene.from_desc(desc)
    tl = s.export_nodes(-1)
    for k in NODE_KEYS:
        assert np.array_equal(tl[k], g["tlas_" + k]), k
    obj, prim, t, geo = s.intersect(dev(g["o"], cuda), dev(g["d"], cuda), geo=True)
    obj, prim, t, geo = obj.cpu().numpy(), prim.cpu().numpy(), t.cpu().numpy(), geo.cpu().numpy()
    assert np.array_equal(obj, g["obj"])
    assert np.array_equal(prim, g["prim"])
    assert np.array_equal(t.view(np.uint32), g["t"].view(np.uint32))
    h = obj >= 0
    assert np.array_equal(geo[h].view(np.uint32), g["geo"][h].view(np.uint32))
    occ = s.intersectP(dev(g["o"], cuda), dev(g["d"], cuda), dev(g["tmax"], cuda))
    assert np.array_equal(occ.cpu().numpy(), g["occ"])
    assert abs(s.stats()["total_emit_area"] - float(g["emit_area"][0])) == 0


def test_scene_intersect_many_objects_against_reference(ref, cuda):
    """Random meshes and spheres (scene BVH of 40 objects) against the
    reference's Scene::intersect / intersectP."""
    rng = np.random.default_rng(2)
    desc = scenes.SceneDesc()
    m = desc.add_material(scenes.Material())
    for k in range(40):
        if k % 3 == 0:
            desc.objects.append(scenes.SphereObject(tuple(rng.uniform(-3, 3, 3)),
                                                    float(rng.uniform(0.1, 0.6)), m))
        else:
            v, _, _ = scenes.query_set(int(rng.integers(1, 400)), 1, seed=100 + k, jitter=0.05)
            v = (v.reshape(-1, 3) * rng.uniform(0.5, 2) + rng.uniform(-3, 3, 3)).reshape(-1, 9)
            desc.objects.append(scenes.MeshObject(v.astype(np.float32), m))
    o = rng.uniform(-4, 4, (20000, 3)).astype(np.float32)
    d = rng.normal(size=(20000, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    tm = rng.uniform(0.5, 6, 20000).astype(np.float32)
    rs = ref.scene(desc)
    ro, rp, rt = rs.intersect(o, d)
    rocc = rs.occluded(o, d, tm)
    s = prr.Scene.from_desc(desc)
    so, sp, st = s.intersect(dev(o, cuda), dev(d, cuda))
    assert np.array_equal(so.cpu().numpy(), ro)
    assert np.array_equal(sp.cpu().numpy(), rp)
    assert np.array_equal(st.cpu().numpy().view(np.uint32), rt.view(np.uint32))
    socc = s.intersectP(dev(o, cuda), dev(d, cuda), dev(tm, cuda))
    assert np.array_equal(socc.cpu().numpy(), rocc)


def test_edge_and_vertex_ties_all_launch_shapes(port, cuda):
    # rays aimed at the shared edges and vertices of a tessellated grid and of
    # an icosphere: many hits at equal (or one-ulp apart) distances in
    # neighbouring leaves, where only the reference's leaf order and culling
    # decide the winner
    n = 48
    g = np.linspace(-1.0, 1.0, n + 1, dtype=np.float32)
    tris = []
    for i in range(n):
        for j in range(n):
            a = (g[i], g[j], 0.5)
            b = (g[i + 1], g[j], 0.5)
            c = (g[i + 1], g[j + 1], 0.5)
            d = (g[i], g[j + 1], 0.5)
            tris += [a + b + c, a + c + d]
    grid = np.array(tris, np.float32)
    ico = scenes.icosphere(4) * np.float32(0.4)
    v = np.vstack([grid, ico.reshape(-1, 9)]).astype(np.float32)
    rng = np.random.default_rng(9)
    tv = grid.reshape(-1, 3)
    targets = np.vstack([tv, (grid[:, 0:3] + grid[:, 3:6]) * np.float32(0.5),
                         ico.reshape(-1, 3)]).astype(np.float32)
    targets = targets[rng.permutation(len(targets))[:60000]]
    o = np.column_stack([rng.uniform(-1.5, 1.5, len(targets)), rng.uniform(-1.5, 1.5, len(targets)),
                         rng.uniform(1.5, 3.0, len(targets))]).astype(np.float32)
    d = (targets - o).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True).astype(np.float32)
    d = d.astype(np.float32)
    s = prr.Scene.single_mesh(v)
    rh, rt, _ = port.mesh(v).intersect(o, d)
    for cfg in (None, {"persistent": 2}, {"persistent": 3}, {"persistent": 3, "leaf_batch": 1},
                {"persistent": 3, "leaf_batch": 32}, {"persistent": 2, "sort_rays": 1}):
        hid, t = s.mesh_intersect(0, dev(o, cuda), dev(d, cuda), config=cfg)
        assert np.array_equal(hid.cpu().numpy(), rh), cfg
        assert np.array_equal(t.cpu().numpy().view(np.uint32), rt.view(np.uint32)), cfg
