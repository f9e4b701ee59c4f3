"""C ABI checks that need no GPU: the library loads, exports every symbol the
headers declare, reports errors, and its host SAH builder reproduces the
reference's trees node for node."""
import ctypes as C

import numpy as np
import pytest

import photorealisticrender4610_b200 as prr
from photorealisticrender4610_b200 import _lib, scenes

from test_oracle import MESH_CASES, NODE_KEYS


def test_exports_every_declared_symbol(lib):
    names = prr.header_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.prr_abi_version() == 1


def test_checked_build_exports_every_declared_symbol():
    """The checked build (device-side bounds tests) is the same ABI."""
    import ctypes
    from photorealisticrender4610_b200 import build
    if not build.LIB_CHECKED.exists():
        pytest.skip("checked library not built")
    lib = ctypes.CDLL(str(build.LIB_CHECKED))
    missing = [n for n in prr.header_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.prr_abi_version() == 1


def test_error_paths(lib):
    s = prr.Scene()
    with pytest.raises(prr.PrrError, match="NOT_BUILT"):
        s.stats()
    with pytest.raises(prr.PrrError, match="INVALID_ARGUMENT"):
        s.add_mesh(np.zeros((1, 9), np.float32), 0)  # no material yet
    m = s.add_material(0, [0.8] * 3 + [0.5, 0.0, 1.5, 0, 0, 0])
    with pytest.raises(prr.PrrError, match="INVALID_ARGUMENT"):
        s.add_sphere((0, 0, 0), -1.0, m)
    with pytest.raises(prr.PrrError, match="INVALID_ARGUMENT"):
        s.add_material(9, [0] * 9)
    assert lib.prr_scene_build(None, None) == -1
    assert "NULL" in _lib.last_error()
    assert lib.prr_mesh_intersect(None, 0, None, None, 0, None, None, None, None, None) == -1


def bvh_build(prim_bounds, prim_areas, max_prims):
    lib = prr.load()
    n = len(prim_areas)
    pb = np.ascontiguousarray(prim_bounds, np.float32)
    pa = np.ascontiguousarray(prim_areas, np.float32)
    m = max(1, 2 * n - 1)
    b = np.empty((m, 6), np.float32)
    fc = np.empty(m, np.uint32)
    meta = np.empty(m, np.uint32)
    ar = np.empty(m, np.float32)
    od = np.empty(n, np.int32)
    md = C.c_int32()
    nn = _lib.check(lib.prr_bvh_build(pb.ctypes.data, pa.ctypes.data, n, max_prims,
                                      b.ctypes.data, fc.ctypes.data, meta.ctypes.data,
                                      ar.ctypes.data, od.ctypes.data, C.byref(md)))
    return dict(bounds=b[:nn], first_child=fc[:nn], meta=meta[:nn], area=ar[:nn],
                ordered=od), md.value


@pytest.mark.parametrize("case", MESH_CASES)
def test_host_sah_builder_matches_reference(golden, port, case):
    g = golden("mesh")
    p = f"mesh_{case}_"
    v = g[p + "verts"]
    pb = np.empty((len(v), 6), np.float32)
    pa = np.empty(len(v), np.float32)
    port.L.prr_oracle_triangle_prims(np.ascontiguousarray(v), len(v), pb, pa)
    nodes, depth = bvh_build(pb, pa, 4)
    for k in NODE_KEYS:
        assert np.array_equal(nodes[k], g[p + k]), k
    assert depth >= 0


def test_host_sah_builder_scene_level(golden):
    """The scene BVH over objects (maxPrimsInNode 1, nth_element for 2..4
    objects) of the Cornell box."""
    g = golden("cornell")
    desc = scenes.cornell_box(64, 64)
    pb, pa = [], []
    for o in desc.objects:
        if o.kind == "mesh":
            v = o.verts.reshape(-1, 3)
            pb.append(np.concatenate([v.min(0), v.max(0)]))
            e1 = o.verts[:, 3:6] - o.verts[:, 0:3]
            e2 = o.verts[:, 6:9] - o.verts[:, 0:3]
            c = np.cross(e1, e2).astype(np.float32)
            a = (np.sqrt((c * c).sum(1, dtype=np.float32)) * np.float32(0.5)).astype(np.float32)
            s = np.float32(0)
            for x in a:
                s = np.float32(s + x)
            pa.append(s)
        else:
            r = np.float32(o.radius)
            c = np.asarray(o.center, np.float32)
            pb.append(np.concatenate([c - r, c + r]))
            pa.append(np.float32(np.float32(np.float32(4) * np.float32(3.141592653589793)) * r) * r)
    nodes, _ = bvh_build(np.array(pb, np.float32), np.array(pa, np.float32), 1)
    for k in NODE_KEYS:
        assert np.array_equal(nodes[k], g["tlas_" + k]), k


def test_host_sah_builder_random_object_sets(port):
    """Scene-level builds over 2..40 random boxes against the C restatement
    (covers the nth_element restatement at 2, 3 and 4 objects)."""
    rng = np.random.default_rng(0)
    for n in list(range(2, 12)) + [17, 40]:
        for trial in range(20):
            c = rng.uniform(-5, 5, (n, 3)).astype(np.float32)
            if trial % 3 == 0:
                c[:, rng.integers(0, 3)] = 1.0  # ties on one axis
            h = rng.uniform(0.1, 1, (n, 3)).astype(np.float32)
            pb = np.hstack([c - h, c + h]).astype(np.float32)
            pa = rng.uniform(0.1, 2, n).astype(np.float32)
            ours, _ = bvh_build(pb, pa, 1)
            nb = np.empty((2 * n, 6), np.float32)
            fc = np.empty(2 * n, np.uint32)
            meta = np.empty(2 * n, np.uint32)
            ar = np.empty(2 * n, np.float32)
            od = np.empty(n, np.int32)
            nn = port.L.prr_oracle_bvh_build(pb, pa, n, 1, nb, fc, meta, ar, od)
            assert np.array_equal(ours["bounds"], nb[:nn])
            assert np.array_equal(ours["first_child"], fc[:nn])
            assert np.array_equal(ours["meta"], meta[:nn])
            assert np.array_equal(ours["ordered"], od)


def test_scene_level_builder_against_reference_nth_element(ref):
    """Scene BVHs over 2..9 random spheres (the sizes where the reference calls
    std::nth_element) built by the reference and by the host builder."""
    rng = np.random.default_rng(1)
    for n in range(2, 10):
        for trial in range(15):
            desc = scenes.SceneDesc()
            m = desc.add_material(scenes.Material())
            c = rng.uniform(-3, 3, (n, 3)).astype(np.float32)
            if trial % 4 == 0:
                c[:, rng.integers(0, 3)] = 0.5
            r = rng.uniform(0.05, 0.5, n).astype(np.float32)
            for k in range(n):
                desc.objects.append(scenes.SphereObject(tuple(c[k]), float(r[k]), m))
            rs = ref.scene(desc)
            want = rs.nodes(-1)
            pb = np.hstack([c - r[:, None], c + r[:, None]]).astype(np.float32)
            pa = np.array([np.float32(np.float32(np.float32(4) * np.float32(3.141592653589793))
                                      * x) * x for x in r], np.float32)
            got, _ = bvh_build(pb, pa, 1)
            for k in NODE_KEYS:
                assert np.array_equal(got[k], want[k]), (n, trial, k)


@pytest.mark.parametrize("kw", [dict(paths_per_pass=(1 << 30) + 1), dict(paths_per_pass=-1),
                                dict(block_size=48), dict(block_size=1024),
                                dict(stack_smem=-2), dict(refill=33)])
def test_wavefront_config_rejected(lib, kw):
    """prr_scene_set_wavefront refuses launch shapes it cannot run (a pass of
    more than 2^30 paths would also overflow its path indices)."""
    import photorealisticrender4610_b200 as prr
    s = prr.Scene()
    with pytest.raises(prr.PrrError, match="wavefront config"):
        s.set_wavefront(**kw)
    s.set_wavefront(paths_per_pass=1 << 30, block_size=128, stack_smem=8)


def test_host_sah_builder_large_mesh(port):
    """A 400,000-triangle soup (the query set's generator), its subtrees built
    on several host threads: the tree equals the C restatement's node for
    node, areas and prim order included."""
    verts, _, _ = scenes.query_set(400_000, 1, seed=5)
    v = np.ascontiguousarray(verts, np.float32)
    n = len(v)
    pb = np.empty((n, 6), np.float32)
    pa = np.empty(n, np.float32)
    port.L.prr_oracle_triangle_prims(v, n, pb, pa)
    ours, _ = bvh_build(pb, pa, 4)
    m = 2 * n
    nb = np.empty((m, 6), np.float32)
    fc = np.empty(m, np.uint32)
    meta = np.empty(m, np.uint32)
    ar = np.empty(m, np.float32)
    od = np.empty(n, np.int32)
    nn = port.L.prr_oracle_bvh_build(pb, pa, n, 4, nb, fc, meta, ar, od)
    assert np.array_equal(ours["bounds"], nb[:nn])
    assert np.array_equal(ours["first_child"], fc[:nn])
    assert np.array_equal(ours["meta"], meta[:nn])
    assert np.array_equal(ours["area"].view(np.uint32), ar[:nn].view(np.uint32))
    assert np.array_equal(ours["ordered"], od)
