"""Test infrastructure only: ctypes bindings to the oracle libraries.

Two oracles live here:

* ``ReferenceOracle`` -- the reference renderer's own C++ sources compiled in
  place by ``oracle/Makefile`` into ``oracle/_ref/libprr_ref.so`` (IEEE flags,
  the parity oracle) and ``libprr_ref_fast.so`` (the reference's shipped
  ``-O3 -ffast-math`` flags, the timed CPU baseline), driven through
  ``oracle/ref/harness.cpp``.
* ``PortOracle`` -- the plain-C restatement ``oracle/prr_oracle.c``.

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
this module, always as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
# The one setting that locates the reference source tree on the build host
# (compiled in place by oracle/Makefile; read by tests for its .glb assets).
REFERENCE_ROOT = Path(os.environ.get("PRR_REFERENCE_ROOT", "/root/reference"))
PORT_LIB = HERE / "libprr_oracle.so"

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def build_port() -> Path:
    """Compile the C restatement (gcc only; works on any host with the image)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "port"], check=True)
    return PORT_LIB


def build_reference(ref_root: str | None = None) -> bool:
    """Compile the reference sources in place into oracle/_ref/ (needs the
    reference tree, which exists only on the build host). The bridge library
    also needs the package's libprr.so, so it is built only when that exists."""
    root = str(ref_root or REFERENCE_ROOT)
    if not Path(root, "BVH.cpp").exists():
        return False
    targets = ["ref"]
    if (HERE.parent / "photorealisticrender4610_b200" / "libprr.so").exists():
        targets.append("bridge")
    subprocess.run(["make", "-s", "-j8", "-C", str(HERE), *targets, f"REF={root}"], check=True)
    return True


def _ref_lib(fast: bool = False, bridge: bool = False) -> Path:
    if bridge:
        return REF_DIR / "libprr_ref_bridge.so"
    return REF_DIR / ("libprr_ref_fast.so" if fast else "libprr_ref.so")


def reference_available(fast: bool = False, bridge: bool = False) -> bool:
    return _ref_lib(fast, bridge).exists()


class PortOracle:
    """The C restatement (oracle/prr_oracle.c)."""

    def __init__(self):
        if not PORT_LIB.exists():
            build_port()
        L = C.CDLL(str(PORT_LIB))
        L.prr_oracle_rng_stream.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_int, _f32p]
        L.prr_oracle_bvh_build.restype = C.c_int64
        L.prr_oracle_bvh_build.argtypes = [_f32p, _f32p, C.c_int64, C.c_int, _f32p, _u32p, _u32p,
                                           _f32p, _i32p]
        L.prr_oracle_triangle_prims.argtypes = [_f32p, C.c_int64, _f32p, _f32p]
        L.prr_oracle_mesh_new.restype = C.c_void_p
        L.prr_oracle_mesh_new.argtypes = [_f32p, C.c_int64]
        L.prr_oracle_mesh_free.argtypes = [C.c_void_p]
        L.prr_oracle_mesh_nodes.restype = C.c_int64
        L.prr_oracle_mesh_nodes.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p]
        L.prr_oracle_mesh_intersect.argtypes = [C.c_void_p, _f32p, _f32p, C.c_int64, _i32p, _f32p,
                                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.prr_oracle_mesh_occluded.argtypes = [C.c_void_p, _f32p, _f32p, _f32p, C.c_int64, _u8p,
                                               C.c_int]
        L.prr_oracle_tonemap.argtypes = [C.c_int, C.c_float, _f32p, C.c_int64, _f32p, _u8p]
        L.prr_oracle_env_cdf.argtypes = [_f32p, C.c_int, C.c_int, _f32p, _f32p,
                                         C.POINTER(C.c_float)]
        L.prr_oracle_photon_estimate.argtypes = [_f32p, C.c_int64, C.c_float, _f32p, C.c_int64,
                                                 _f32p, C.POINTER(C.c_int32)]
        L.prr_oracle_photon_estimate_knn.argtypes = [_f32p, C.c_int64, C.c_float, C.c_int, _f32p,
                                                     C.c_int64, _f32p, _i32p,
                                                     C.POINTER(C.c_int32)]
        self.L = L

    def rng_stream(self, seed, stream, index, n):
        out = np.empty(n, np.float32)
        self.L.prr_oracle_rng_stream(seed, stream, index, n, out)
        return out

    def mesh(self, verts):
        return PortMesh(self, _c(verts, np.float32).reshape(-1, 9))

    def tonemap(self, mapper, rgb, exposure=1.0):
        rgb = _c(rgb, np.float32).reshape(-1, 3)
        out = np.empty_like(rgb)
        u8 = np.empty(rgb.shape, np.uint8)
        self.L.prr_oracle_tonemap(mapper, exposure, rgb, len(rgb), out, u8)
        return out, u8

    def env_cdf(self, rgb):
        rgb = _c(rgb, np.float32)
        h, w = rgb.shape[:2]
        cdf = np.empty(h * w, np.float32)
        marg = np.empty(h, np.float32)
        tot = C.c_float()
        self.L.prr_oracle_env_cdf(rgb.reshape(-1), w, h, cdf, marg, C.byref(tot))
        return cdf, marg, tot.value

    def photon_estimate(self, rec, radius, q):
        rec = _c(rec, np.float32).reshape(-1, 9)
        q = _c(q, np.float32).reshape(-1, 3)
        out = np.empty((len(q), 3), np.float32)
        res = C.c_int32()
        self.L.prr_oracle_photon_estimate(rec, len(rec), radius, q, len(q), out, C.byref(res))
        return out, res.value

    def photon_estimate_knn(self, rec, radius, q, k):
        """Irradiance capped at the k nearest photons (k = 0: fixed radius),
        and the number of photons inside the radius of each query."""
        rec = _c(rec, np.float32).reshape(-1, 9)
        q = _c(q, np.float32).reshape(-1, 3)
        out = np.empty((len(q), 3), np.float32)
        inside = np.empty(len(q), np.int32)
        res = C.c_int32()
        self.L.prr_oracle_photon_estimate_knn(rec, len(rec), radius, k, q, len(q), out, inside,
                                              C.byref(res))
        return out, inside


class PortMesh:
    def __init__(self, port: PortOracle, verts):
        self.port = port
        self.n = len(verts)
        self.h = port.L.prr_oracle_mesh_new(verts, self.n)

    def __del__(self):
        if getattr(self, "h", None):
            self.port.L.prr_oracle_mesh_free(self.h)
            self.h = None

    def nodes(self):
        L = self.port.L
        nn = L.prr_oracle_mesh_nodes(self.h, None, None, None, None, None)
        b = np.empty((nn, 6), np.float32)
        fc = np.empty(nn, np.uint32)
        meta = np.empty(nn, np.uint32)
        area = np.empty(nn, np.float32)
        order = np.empty(self.n, np.int32)
        L.prr_oracle_mesh_nodes(self.h, b.ctypes.data, fc.ctypes.data, meta.ctypes.data,
                                area.ctypes.data, order.ctypes.data)
        return dict(bounds=b, first_child=fc, meta=meta, area=area, ordered=order)

    def intersect(self, o, d, threads=0, stats=False):
        o = _c(o, np.float32).reshape(-1, 3)
        d = _c(d, np.float32).reshape(-1, 3)
        n = len(o)
        hid = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        t64 = np.empty(n, np.float64)
        vis = np.empty(n, np.int32) if stats else None
        tst = np.empty(n, np.int32) if stats else None
        self.port.L.prr_oracle_mesh_intersect(
            self.h, o, d, n, hid, t, t64.ctypes.data,
            vis.ctypes.data if stats else None, tst.ctypes.data if stats else None,
            threads or os.cpu_count())
        if stats:
            return hid, t, t64, vis, tst
        return hid, t, t64

    def occluded(self, o, d, tmax, threads=0):
        o = _c(o, np.float32).reshape(-1, 3)
        d = _c(d, np.float32).reshape(-1, 3)
        tmax = _c(tmax, np.float32).reshape(-1)
        out = np.empty(len(o), np.uint8)
        self.port.L.prr_oracle_mesh_occluded(self.h, o, d, tmax, len(o), out,
                                             threads or os.cpu_count())
        return out


class ReferenceOracle:
    """The reference's own code (oracle/_ref/libprr_ref*.so via harness.cpp).
    bridge=True loads the parity build that also carries the prr_bridge.hpp
    test entry point (RefScene.bridge_render)."""

    def __init__(self, fast: bool = False, bridge: bool = False):
        path = _ref_lib(fast, bridge)
        self.bridge = bridge
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (oracle/Makefile ref)")
        L = C.CDLL(str(path))
        vp = C.c_void_p
        L.prr_ref_rng_stream.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_int, _f32p]
        L.prr_ref_max_threads.restype = C.c_int
        L.prr_ref_mesh_new.restype = vp
        L.prr_ref_mesh_new.argtypes = [_f32p, C.c_int64]
        L.prr_ref_mesh_free.argtypes = [vp]
        L.prr_ref_mesh_nodes.restype = C.c_int64
        L.prr_ref_mesh_nodes.argtypes = [vp, vp, vp, vp, vp, vp]
        L.prr_ref_mesh_area.restype = C.c_float
        L.prr_ref_mesh_area.argtypes = [vp, C.POINTER(C.c_float)]
        L.prr_ref_mesh_intersect.argtypes = [vp, _f32p, _f32p, C.c_int64, _i32p, _f32p, vp, vp,
                                             C.c_int]
        L.prr_ref_mesh_occluded.argtypes = [vp, _f32p, _f32p, _f32p, C.c_int64, _u8p, C.c_int]
        L.prr_ref_scene_new.restype = vp
        L.prr_ref_scene_free.argtypes = [vp]
        L.prr_ref_scene_add_material.restype = C.c_int
        L.prr_ref_scene_add_material.argtypes = [vp, C.c_int, _f32p]
        L.prr_ref_scene_add_mesh.restype = C.c_int
        L.prr_ref_scene_add_mesh.argtypes = [vp, _f32p, C.c_int64, C.c_int]
        L.prr_ref_scene_add_gltf.restype = C.c_int
        L.prr_ref_scene_add_gltf.argtypes = [vp, C.c_char_p, C.c_int]
        L.prr_ref_scene_add_obj.restype = C.c_int
        L.prr_ref_scene_add_obj.argtypes = [vp, C.c_char_p, _f32p, C.c_int]
        L.prr_ref_medium_preset.restype = None
        L.prr_ref_medium_preset.argtypes = [C.c_int, _f32p]
        L.prr_ref_medium_intersect.restype = None
        L.prr_ref_medium_intersect.argtypes = [C.c_int, _f32p, _f32p, _f32p, _f32p, C.c_int64,
                                               _f32p, _f32p, vp]
        L.prr_ref_phase_hg.restype = None
        L.prr_ref_phase_hg.argtypes = [_f32p, C.c_int64, C.c_float, _f32p]
        L.prr_ref_phase_hg_sample.restype = None
        L.prr_ref_phase_hg_sample.argtypes = [_f32p, C.c_int64, C.c_float, C.c_uint64, _f32p]
        L.prr_ref_scene_export_mesh.restype = C.c_int64
        L.prr_ref_scene_export_mesh.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp]
        L.prr_ref_scene_export_material.restype = C.c_int
        L.prr_ref_scene_export_material.argtypes = [vp, C.c_int, vp, vp, vp]
        L.prr_ref_scene_export_texture.restype = C.c_int
        L.prr_ref_scene_export_texture.argtypes = [vp, C.c_int, C.c_int, vp]
        L.prr_ref_scene_add_mesh_attr.restype = C.c_int
        L.prr_ref_scene_add_mesh_attr.argtypes = [vp, _f32p, vp, vp, vp, C.c_int64, C.c_int]
        L.prr_ref_scene_set_texture.restype = C.c_int
        L.prr_ref_scene_set_texture.argtypes = [vp, C.c_int, C.c_int, _u8p, C.c_int, C.c_int,
                                                C.c_int]
        L.prr_ref_scene_add_sphere.restype = C.c_int
        L.prr_ref_scene_add_sphere.argtypes = [vp, _f32p, C.c_float, C.c_int]
        L.prr_ref_scene_set_background.argtypes = [vp, _f32p]
        L.prr_ref_scene_set_env.restype = C.c_int
        L.prr_ref_scene_set_env.argtypes = [vp, _f32p, C.c_int, C.c_int, C.c_char_p]
        L.prr_ref_scene_env_export.restype = C.c_int
        L.prr_ref_scene_env_export.argtypes = [vp, vp, vp, vp, vp]
        L.prr_ref_env_eval.argtypes = [vp, _f32p, C.c_int64, _f32p, _f32p]
        L.prr_ref_env_importance.argtypes = [vp, C.c_uint64, C.c_int64, _f32p, _f32p]
        L.prr_ref_scene_set_camera.argtypes = [vp, _f32p, _f32p, _f32p, C.c_float, C.c_float,
                                               C.c_float, C.c_float, C.c_int, C.c_int]
        L.prr_ref_scene_build.argtypes = [vp]
        L.prr_ref_scene_tlas_nodes.restype = C.c_int64
        L.prr_ref_scene_tlas_nodes.argtypes = [vp, vp, vp, vp, vp, vp]
        L.prr_ref_scene_object_nodes.restype = C.c_int64
        L.prr_ref_scene_object_nodes.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp]
        L.prr_ref_scene_emit_area.restype = C.c_float
        L.prr_ref_scene_emit_area.argtypes = [vp]
        L.prr_ref_scene_intersect.argtypes = [vp, _f32p, _f32p, C.c_int64, _i32p, _i32p, _f32p,
                                              vp, C.c_int]
        L.prr_ref_scene_occluded.argtypes = [vp, _f32p, _f32p, _f32p, C.c_int64, _u8p, C.c_int]
        L.prr_ref_scene_sample_light.argtypes = [vp, C.c_uint64, C.c_int64, _f32p, _f32p, _f32p]
        L.prr_ref_render.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_uint64,
                                     C.c_int, C.c_int, C.c_int, C.c_int, _f32p, vp, C.c_int]
        L.prr_ref_cast_samples.argtypes = [vp, C.c_int, C.c_uint64, _i32p, _i32p, _i32p,
                                           C.c_int64, _f32p, vp, C.c_int]
        L.prr_ref_camera_rays.argtypes = [vp, _i32p, _i32p, _f32p, _f32p, C.c_int64, _f32p, _f32p]
        L.prr_ref_tonemap.argtypes = [C.c_int, C.c_float, _f32p, C.c_int64, _f32p, _u8p]
        L.prr_ref_photon_emit.restype = vp
        L.prr_ref_photon_emit.argtypes = [vp, C.c_int64, C.c_uint64, C.c_int, C.c_int]
        L.prr_ref_photon_export.restype = C.c_int64
        L.prr_ref_photon_export.argtypes = [vp, vp, vp]
        L.prr_ref_photon_free.argtypes = [vp]
        if bridge:
            L.prr_ref_bridge_render.restype = C.c_int
            L.prr_ref_bridge_render.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_float,
                                                C.c_uint64, C.c_int, C.c_int, C.c_float, _f32p,
                                                _i32p, _u8p, vp]
        L.prr_ref_photon_estimate.argtypes = [_f32p, C.c_int64, C.c_float, _f32p, C.c_int64,
                                              _f32p, C.POINTER(C.c_int32), C.c_int]
        L.prr_ref_photon_estimate_knn.argtypes = [_f32p, C.c_int64, C.c_float, C.c_int, _f32p,
                                                  C.c_int64, _f32p, _i32p, C.c_int]
        L.prr_ref_caustic_render.argtypes = [vp, _f32p, C.c_int64, C.c_float, C.c_int, C.c_int,
                                             C.c_int, C.c_uint64, C.c_int, C.c_int, C.c_int,
                                             C.c_int, C.c_int, _f32p, C.c_int]
        self.L = L
        self.fast = fast

    def max_threads(self):
        return self.L.prr_ref_max_threads()

    def rng_stream(self, seed, stream, index, n):
        out = np.empty(n, np.float32)
        self.L.prr_ref_rng_stream(seed, stream, index, n, out)
        return out

    def mesh(self, verts):
        return RefMesh(self, _c(verts, np.float32).reshape(-1, 9))

    def scene(self, desc):
        return RefScene(self, desc)

    def tonemap(self, mapper, rgb, exposure=1.0):
        rgb = _c(rgb, np.float32).reshape(-1, 3)
        out = np.empty_like(rgb)
        u8 = np.empty(rgb.shape, np.uint8)
        self.L.prr_ref_tonemap(mapper, exposure, rgb, len(rgb), out, u8)
        return out, u8

    def photon_estimate(self, rec, radius, q, threads=0):
        rec = _c(rec, np.float32).reshape(-1, 9)
        q = _c(q, np.float32).reshape(-1, 3)
        out = np.empty((len(q), 3), np.float32)
        res = C.c_int32()
        self.L.prr_ref_photon_estimate(rec, len(rec), radius, q, len(q), out, C.byref(res),
                                       threads)
        return out, res.value

    def photon_estimate_knn(self, rec, radius, q, k, threads=0):
        """The k-nearest-capped estimate over the reference's own grid query
        (k = 0 or at most k photons inside: estimateIrradiance itself), and the
        number of photons inside the radius of each query."""
        rec = _c(rec, np.float32).reshape(-1, 9)
        q = _c(q, np.float32).reshape(-1, 3)
        out = np.empty((len(q), 3), np.float32)
        inside = np.empty(len(q), np.int32)
        self.L.prr_ref_photon_estimate_knn(rec, len(rec), radius, k, q, len(q), out, inside,
                                           threads)
        return out, inside


class RefMesh:
    def __init__(self, ref: ReferenceOracle, verts):
        self.ref = ref
        self.n = len(verts)
        self.h = ref.L.prr_ref_mesh_new(verts, self.n)

    def __del__(self):
        if getattr(self, "h", None):
            self.ref.L.prr_ref_mesh_free(self.h)
            self.h = None

    def nodes(self):
        L = self.ref.L
        nn = L.prr_ref_mesh_nodes(self.h, None, None, None, None, None)
        b = np.empty((nn, 6), np.float32)
        fc = np.empty(nn, np.uint32)
        meta = np.empty(nn, np.uint32)
        area = np.empty(nn, np.float32)
        order = np.empty(self.n, np.int32)
        L.prr_ref_mesh_nodes(self.h, b.ctypes.data, fc.ctypes.data, meta.ctypes.data,
                             area.ctypes.data, order.ctypes.data)
        return dict(bounds=b, first_child=fc, meta=meta, area=area, ordered=order)

    def areas(self):
        tot = C.c_float()
        a = self.ref.L.prr_ref_mesh_area(self.h, C.byref(tot))
        return a, tot.value

    def intersect(self, o, d, threads=0, uv=False):
        o = _c(o, np.float32).reshape(-1, 3)
        d = _c(d, np.float32).reshape(-1, 3)
        n = len(o)
        hid = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        u = np.empty(n, np.float32) if uv else None
        v = np.empty(n, np.float32) if uv else None
        self.ref.L.prr_ref_mesh_intersect(self.h, o, d, n, hid, t,
                                          u.ctypes.data if uv else None,
                                          v.ctypes.data if uv else None, threads)
        return (hid, t, u, v) if uv else (hid, t)

    def occluded(self, o, d, tmax, threads=0):
        o = _c(o, np.float32).reshape(-1, 3)
        d = _c(d, np.float32).reshape(-1, 3)
        tmax = _c(tmax, np.float32).reshape(-1)
        out = np.empty(len(o), np.uint8)
        self.ref.L.prr_ref_mesh_occluded(self.h, o, d, tmax, len(o), out, threads)
        return out


class RefScene:
    """A reference Scene built from a photorealisticrender4610_b200 SceneDesc."""

    def __init__(self, ref: ReferenceOracle, desc, env_tmp: str | None = None):
        L = ref.L
        self.ref = ref
        self.desc = desc
        self.h = L.prr_ref_scene_new()
        for m in desc.materials:
            mid = L.prr_ref_scene_add_material(self.h, int(m.kind), _c(m.params(), np.float32))
            for slot, t in enumerate(m.texture_list()):
                if t is not None:
                    t = _c(t, np.uint8)
                    L.prr_ref_scene_set_texture(self.h, mid, slot, t.reshape(-1), t.shape[1],
                                                t.shape[0], t.shape[2])
        keep = []
        for obj in desc.objects:
            if obj.kind == "mesh" and obj.has_attributes():
                v = _c(obj.verts, np.float32).reshape(-1, 9)
                ptrs = []
                for a, k in ((obj.normals, 9), (obj.uvs, 6), (obj.tangents, 12)):
                    if a is None:
                        ptrs.append(None)
                    else:
                        a = _c(a, np.float32).reshape(-1, k)
                        keep.append(a)
                        ptrs.append(a.ctypes.data)
                L.prr_ref_scene_add_mesh_attr(self.h, v, *ptrs, len(v), obj.material)
            elif obj.kind == "mesh":
                v = _c(obj.verts, np.float32).reshape(-1, 9)
                L.prr_ref_scene_add_mesh(self.h, v, len(v), obj.material)
            else:
                L.prr_ref_scene_add_sphere(self.h, _c(obj.center, np.float32), float(obj.radius),
                                           obj.material)
        L.prr_ref_scene_set_background(self.h, _c(desc.background, np.float32))
        if desc.env is not None:
            import tempfile
            fd, path = tempfile.mkstemp(suffix=".hdr")
            os.close(fd)
            try:
                env = _c(desc.env, np.float32)
                rc = L.prr_ref_scene_set_env(self.h, env.reshape(-1), env.shape[1], env.shape[0],
                                             path.encode())
                if rc != 0:
                    raise RuntimeError(f"reference EnvMap::load failed ({rc})")
            finally:
                os.unlink(path)
        cam = desc.camera
        L.prr_ref_scene_set_camera(self.h, _c(cam.eye, np.float32), _c(cam.target, np.float32),
                                   _c(cam.up, np.float32), cam.fovv, cam.fovh, cam.aperture,
                                   cam.focus_distance, desc.width, desc.height)
        L.prr_ref_scene_build(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.ref.L.prr_ref_scene_free(self.h)
            self.h = None

    def bridge_render(self, max_depth, min_spp, max_spp, threshold=0.05, seed=1, mode=1,
                      mapper=2, exposure=0.18):
        """This reference scene rendered by libprr through include/prr_bridge.hpp
        (needs ReferenceOracle(bridge=True) and a GPU). Returns (linear rgb,
        spp, 8-bit rgb, report dict)."""
        if not self.ref.bridge:
            raise RuntimeError("load ReferenceOracle(bridge=True) for the bridge entry point")
        W, H = self.desc.width, self.desc.height
        n = W * H
        rgb = np.empty(n * 3, np.float32)
        spp = np.empty(n, np.int32)
        u8 = np.empty(n * 3, np.uint8)
        rep = np.zeros(8, np.int64)
        rc = self.ref.L.prr_ref_bridge_render(self.h, max_depth, min_spp, max_spp, threshold,
                                              seed, mode, mapper, exposure, rgb, spp, u8,
                                              rep.ctypes.data)
        if rc != 0:
            raise RuntimeError("prr_ref_bridge_render failed (see stderr)")
        keys = ("meshes", "spheres", "triangles", "materials", "textures",
                "attributed_meshes", "skipped_objects", "dropped")
        shape = (H, W, 3)
        return (rgb.reshape(shape), spp.reshape(H, W), u8.reshape(shape),
                dict(zip(keys, rep.tolist())))

    def env_export(self):
        e = self.desc.env
        h, w = e.shape[:2]
        px = np.empty((h, w, 3), np.float32)
        cdf = np.empty(h * w, np.float32)
        marg = np.empty(h, np.float32)
        tot = np.empty(1, np.float32)
        self.ref.L.prr_ref_scene_env_export(self.h, px.ctypes.data, cdf.ctypes.data,
                                            marg.ctypes.data, tot.ctypes.data)
        return px, cdf, marg, float(tot[0])

    def env_eval(self, dirs):
        dirs = _c(dirs, np.float32).reshape(-1, 3)
        rgb = np.empty_like(dirs)
        pdf = np.empty(len(dirs), np.float32)
        self.ref.L.prr_ref_env_eval(self.h, dirs, len(dirs), rgb, pdf)
        return rgb, pdf

    def env_importance(self, seed, n):
        dirs = np.empty((n, 3), np.float32)
        pdf = np.empty(n, np.float32)
        self.ref.L.prr_ref_env_importance(self.h, seed, n, dirs, pdf)
        return dirs, pdf

    def nodes(self, obj=-1):
        L = self.ref.L
        if obj < 0:
            nn = L.prr_ref_scene_tlas_nodes(self.h, None, None, None, None, None)
            nprim = len(self.desc.objects)
        else:
            nn = L.prr_ref_scene_object_nodes(self.h, obj, None, None, None, None, None)
            nprim = len(self.desc.objects[obj].verts)
        b = np.empty((nn, 6), np.float32)
        fc = np.empty(nn, np.uint32)
        meta = np.empty(nn, np.uint32)
        area = np.empty(nn, np.float32)
        order = np.empty(nprim, np.int32)
        if obj < 0:
            L.prr_ref_scene_tlas_nodes(self.h, b.ctypes.data, fc.ctypes.data, meta.ctypes.data,
                                       area.ctypes.data, order.ctypes.data)
        else:
            L.prr_ref_scene_object_nodes(self.h, obj, b.ctypes.data, fc.ctypes.data,
                                         meta.ctypes.data, area.ctypes.data, order.ctypes.data)
        return dict(bounds=b, first_child=fc, meta=meta, area=area, ordered=order)

    def emit_area(self):
        return self.ref.L.prr_ref_scene_emit_area(self.h)

    def intersect(self, o, d, threads=0, geo=False):
        o = _c(o, np.float32).reshape(-1, 3)
        d = _c(d, np.float32).reshape(-1, 3)
        n = len(o)
        obj = np.empty(n, np.int32)
        prim = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        g = np.zeros((n, 6), np.float32) if geo else None
        self.ref.L.prr_ref_scene_intersect(self.h, o, d, n, obj, prim, t,
                                           g.ctypes.data if geo else None, threads)
        return (obj, prim, t, g) if geo else (obj, prim, t)

    def occluded(self, o, d, tmax, threads=0):
        o = _c(o, np.float32).reshape(-1, 3)
        d = _c(d, np.float32).reshape(-1, 3)
        tmax = _c(tmax, np.float32).reshape(-1)
        out = np.empty(len(o), np.uint8)
        self.ref.L.prr_ref_scene_occluded(self.h, o, d, tmax, len(o), out, threads)
        return out

    def sample_light(self, seed, n):
        pos = np.empty((n, 3), np.float32)
        nrm = np.empty((n, 3), np.float32)
        pdf = np.empty(n, np.float32)
        self.ref.L.prr_ref_scene_sample_light(self.h, seed, n, pos, nrm, pdf)
        return pos, nrm, pdf

    def render(self, max_depth, spp, seed, window=None, min_spp=None, threshold=0.05,
               threads=0):
        W, H = self.desc.width, self.desc.height
        x0, y0, x1, y1 = window or (0, 0, W, H)
        out = np.empty(((y1 - y0) * (x1 - x0), 3), np.float32)
        cnt = np.empty((y1 - y0) * (x1 - x0), np.int32)
        self.ref.L.prr_ref_render(self.h, max_depth, spp if min_spp is None else min_spp, spp,
                                  threshold, seed, x0, y0, x1, y1, out, cnt.ctypes.data, threads)
        return out.reshape(y1 - y0, x1 - x0, 3), cnt.reshape(y1 - y0, x1 - x0)

    def cast_samples(self, max_depth, seed, px, py, sample, threads=0):
        px = _c(px, np.int32)
        py = _c(py, np.int32)
        sample = _c(sample, np.int32)
        n = len(px)
        out = np.empty((n, 3), np.float32)
        draws = np.empty(n, np.int32)
        self.ref.L.prr_ref_cast_samples(self.h, max_depth, seed, px, py, sample, n, out,
                                        draws.ctypes.data, threads)
        return out, draws

    def camera_rays(self, px, py, xo, yo):
        px = _c(px, np.int32)
        py = _c(py, np.int32)
        xo = _c(xo, np.float32)
        yo = _c(yo, np.float32)
        n = len(px)
        o = np.empty((n, 3), np.float32)
        d = np.empty((n, 3), np.float32)
        self.ref.L.prr_ref_camera_rays(self.h, px, py, xo, yo, n, o, d)
        return o, d

    def caustic_render(self, rec, radius, spp, k_nearest=0, max_depth=8, seed=1,
                       sample_offset=0, window=None, threads=0):
        """The caustic image of a photon array: each camera sample follows
        castRay's delta chain to its first diffuse hit and takes
        baseColor / pi * the (k-capped) irradiance there."""
        rec = _c(rec, np.float32).reshape(-1, 9)
        W, H = self.desc.width, self.desc.height
        x0, y0, x1, y1 = window or (0, 0, W, H)
        out = np.empty(((y1 - y0) * (x1 - x0), 3), np.float32)
        self.ref.L.prr_ref_caustic_render(self.h, rec, len(rec), radius, k_nearest, max_depth,
                                          spp, seed, sample_offset, x0, y0, x1, y1, out, threads)
        return out.reshape(y1 - y0, x1 - x0, 3)

    def photon_emit(self, n_photons, seed, max_depth=30, threads=0):
        L = self.ref.L
        ph = L.prr_ref_photon_emit(self.h, n_photons, seed, max_depth, threads)
        try:
            n = L.prr_ref_photon_export(ph, None, None)
            rec = np.empty((n, 9), np.float32)
            owner = np.empty(n, np.int32)
            L.prr_ref_photon_export(ph, rec.ctypes.data, owner.ctypes.data)
        finally:
            L.prr_ref_photon_free(ph)
        return rec, owner


class RefGltf:
    """Meshes and materials as the reference's GLTFLoader::load builds them
    (oracle build), for comparing ingest field by field."""

    TYPES = {"diffuse": 0, "glass": 1, "mirror": 2, "emit": 3}

    def __init__(self, ref: ReferenceOracle, path, material_type="diffuse"):
        self.ref = ref
        self.h = ref.L.prr_ref_scene_new()
        self.count = ref.L.prr_ref_scene_add_gltf(self.h, str(path).encode(),
                                                  self.TYPES[material_type])

    @classmethod
    def obj(cls, ref: ReferenceOracle, path, offset=(0.0, 0.0, 0.0)):
        """MeshTriangle(filename, offset, m) of the reference on an OBJ file
        (object 0). The file must hold exactly one mesh: the reference
        asserts it and would end the process otherwise."""
        self = cls.__new__(cls)
        self.ref = ref
        self.h = ref.L.prr_ref_scene_new()
        m = ref.L.prr_ref_scene_add_material(self.h, 0, np.array(
            [0.8, 0.8, 0.8, 0.5, 0.0, 1.5, 0.0, 0.0, 0.0], np.float32))
        ref.L.prr_ref_scene_add_obj(self.h, str(path).encode(), np.ascontiguousarray(
            offset, np.float32), m)
        self.count = 1
        return self

    def __del__(self):
        if getattr(self, "h", None):
            self.ref.L.prr_ref_scene_free(self.h)
            self.h = None

    def mesh(self, k):
        L = self.ref.L
        attr = C.c_int()
        n = L.prr_ref_scene_export_mesh(self.h, k, C.byref(attr), None, None, None, None)
        out = {"verts": np.empty((n, 9), np.float32), "normals": np.empty((n, 9), np.float32),
               "uvs": np.empty((n, 6), np.float32), "tangents": np.empty((n, 12), np.float32)}
        L.prr_ref_scene_export_mesh(self.h, k, None, out["verts"].ctypes.data,
                                    out["normals"].ctypes.data, out["uvs"].ctypes.data,
                                    out["tangents"].ctypes.data)
        out["attr"] = attr.value
        return out

    def material(self, k):
        L = self.ref.L
        kind = C.c_int()
        p = np.empty(9, np.float32)
        dims = np.zeros(16, np.int32)
        L.prr_ref_scene_export_material(self.h, k, C.byref(kind), p.ctypes.data, dims.ctypes.data)
        tex = []
        for slot in range(4):
            w, h, c, nbytes = (int(x) for x in dims[slot * 4: slot * 4 + 4])
            if w == 0:
                tex.append(None)
                continue
            t = np.empty(nbytes, np.uint8)
            L.prr_ref_scene_export_texture(self.h, k, slot, t.ctypes.data)
            tex.append(t.reshape(h, w, -1) if nbytes % (w * h) == 0 else t)
        
        return {"kind": kind.value, "params": p, "textures": tex}
