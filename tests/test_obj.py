"""OBJ ingest (prr_scene_add_obj / prr_obj_read) against the reference's own
MeshTriangle(filename, offset, m) (Triangle.cpp:4-32 over its bundled
OBJ_Loader.hpp, compiled into the oracle): the same triangles bit for bit for
every face-corner form, negative indices, CRLF lines, polygons (whose corners
the reference takes three at a time across faces), faces before the first
group line and offsets; files the reference cannot take (more than one mesh,
a corner count that is not a multiple of three, bad indices or numbers) are
errors."""
import numpy as np
import pytest

import photorealisticrender4610_b200 as prr
from oracle import loader

needs_ref = pytest.mark.skipif(not loader.reference_available(),
                               reason="reference oracle library not built")


@pytest.fixture(scope="module")
def ref_oracle():
    return loader.ReferenceOracle()


def write(tmp_path, name, text, crlf=False):
    p = tmp_path / name
    data = text.replace("\n", "\r\n") if crlf else text
    p.write_bytes(data.encode())
    return p


def grid_obj(n=6, seed=0, forms=("p", "pt", "pn", "ptn"), negative=False):
    """An n x n height-field as an OBJ text: v / vt / vn lines and two
    triangles per cell, cycling through the corner forms."""
    rng = np.random.default_rng(seed)
    lines = ["# test grid", "mtllib none.mtl", "o grid"]
    for j in range(n):
        for i in range(n):
            lines.append(f"v {i / (n - 1):.6f} {rng.normal(0, 0.05):.7g} {j / (n - 1):.6f}")
            lines.append(f"vt {i / (n - 1):.4f} {j / (n - 1):.4f}")
            lines.append("vn 0 1 0")
    nv = n * n
    k = 0
    for j in range(n - 1):
        for i in range(n - 1):
            a, b, c, d = j * n + i + 1, j * n + i + 2, (j + 1) * n + i + 2, (j + 1) * n + i + 1
            for tri in ((a, b, c), (a, c, d)):
                form = forms[k % len(forms)]
                k += 1
                idx = [x - nv - 1 if negative and k % 3 == 0 else x for x in tri]
                corner = {"p": "{0}", "pt": "{0}/{0}", "pn": "{0}//{0}", "ptn": "{0}/{0}/{0}"}[form]
                lines.append("f " + " ".join(corner.format(x) for x in idx))
    return "\n".join(lines) + "\n"


def compare(ref_oracle, path, offset=(0.0, 0.0, 0.0)):
    ours = prr.read_obj(path, offset)
    rm = loader.RefGltf.obj(ref_oracle, path, offset).mesh(0)
    assert ours.shape == rm["verts"].shape
    assert np.array_equal(ours.view(np.uint32), rm["verts"].view(np.uint32))
    return ours


@needs_ref
@pytest.mark.parametrize("crlf", [False, True])
@pytest.mark.parametrize("negative", [False, True])
def test_grid_matches_reference(tmp_path, ref_oracle, crlf, negative):
    p = write(tmp_path, "grid.obj", grid_obj(7, seed=3, negative=negative), crlf)
    v = compare(ref_oracle, p, (0.25, -1.5, 3.0))
    assert len(v) == 2 * 6 * 6
    s = prr.Scene()
    m = s.add_material(0, [0.8, 0.8, 0.8, 0.5, 0.0, 1.5, 0.0, 0.0, 0.0])
    obj = s.add_obj(p, m, (0.25, -1.5, 3.0))
    assert np.array_equal(s.export_mesh(obj)["verts"].view(np.uint32), v.view(np.uint32))


@needs_ref
def test_polygons_faces_before_group_and_usemtl(tmp_path, ref_oracle):
    """Quads and a pentagon append all their corners (taken three at a time
    across faces, as the reference does); faces before the first "o" line and
    an "usemtl" before any face stay in the one mesh."""
    text = "\n".join([
        "v 0 0 0", "v 1 0 0", "v 1 1 0", "v 0 1 0", "v 0.5 1.5 0", "v 2 2 2",
        "usemtl first",
        "f 1 2 3 4",
        "o thing",
        "f 1 2 3 5 4",  # a convex pentagon
        "f 2 3 6",
        "f 1 3 6",
        "   f   4 5 6",  # leading blanks before the token
    ]) + "\n"
    p = write(tmp_path, "poly.obj", text)
    v = compare(ref_oracle, p)
    assert len(v) == (4 + 5 + 3 + 3 + 3) // 3


@pytest.mark.parametrize("text,match", [
    ("o a\nv 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\no b\nf 3 2 1\n", "exactly one mesh"),
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\nusemtl x\nf 3 2 1\n", "exactly one mesh"),
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nf 1 2 3 4\nf 4 3 2 1\n", "multiple of three"),
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n", "position index"),
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 0 1 2\n", "position index"),
    ("v 0 0\nf 1 1 1\n", "vertex position"),
    ("v 0  0 0\nf 1 1 1\n", "vertex position"),
    ("v 0 0 0\nv 1 0 0\n", "exactly one mesh"),
])
def test_files_the_reference_cannot_take(tmp_path, text, match):
    p = write(tmp_path, "bad.obj", text)
    with pytest.raises(prr.PrrError, match=match):
        prr.read_obj(p)


def test_name_and_missing_file(tmp_path):
    p = write(tmp_path, "mesh.txt", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    with pytest.raises(prr.PrrError, match=r"\.obj"):
        prr.read_obj(p)
    with pytest.raises(prr.PrrError, match="cannot open"):
        prr.read_obj(tmp_path / "missing.obj")


def test_c_abi_capacity_and_null_offset(tmp_path):
    """prr_obj_read through the C ABI: the count query, a too-small output
    (rejected) and a NULL offset (no shift)."""
    import ctypes as C
    from photorealisticrender4610_b200 import _lib
    lib = _lib.load()
    p = write(tmp_path, "tri.obj", "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nf 1 2 3\nf 2 4 3\n")
    n = C.c_int64()
    assert lib.prr_obj_read(str(p).encode(), None, None, 0, C.byref(n)) == 0
    assert n.value == 2
    out = np.zeros((2, 9), np.float32)
    assert lib.prr_obj_read(str(p).encode(), None, C.c_void_p(out.ctypes.data), 1,
                            C.byref(n)) < 0
    assert lib.prr_obj_read(str(p).encode(), None, C.c_void_p(out.ctypes.data), 2,
                            C.byref(n)) == 0
    assert np.array_equal(out, np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0],
                                         [1, 0, 0, 1, 1, 0, 0, 1, 0]], np.float32))
