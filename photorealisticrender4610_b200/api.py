"""Python mirror of the reference's host interface over libprr's C ABI.

``Scene`` follows Scene (Scene.hpp:15-41): ``add_material`` / ``add_mesh`` /
``add_sphere`` (MeshTriangle, Sphere + Scene::Add), ``set_env`` (EnvMap),
``set_camera`` (Camera::init), ``buildBVH`` (Scene::buildBVH), and the batch
forms of ``intersect`` / ``intersectP`` (Scene::intersect / intersectP) and of
the mesh-level ``BVHAccel::Intersect`` / ``IntersectP``. Device arrays are torch
CUDA tensors (torch supplies memory and streams only); ``*_host`` calls take
numpy arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import (check, prr_camera, prr_render_count, prr_render_settings, prr_request,
                   prr_request_info, prr_scene_stats, prr_server_config, prr_server_stats,
                   prr_trace_config, prr_wavefront_config)

RENDER_MODES = {"plain": 0, "wavefront": 1}
TONEMAPPERS = {"raw": 0, "standard": 1, "agx": 2, "pbrneutral": 3, "aces": 4}


def tonemap(rgb, mapper="agx", exposure: float = 1.0, stream=None):
    """Renderer's display transform on a CUDA tensor of linear RGB (..., 3):
    returns (mapped float32, uint8) tensors of the same shape."""
    import torch
    lib = _lib.load()
    x = rgb.to(torch.float32).contiguous()
    n = x.numel() // 3
    out = torch.empty_like(x)
    u8 = torch.empty(x.shape, dtype=torch.uint8, device=x.device)
    m = TONEMAPPERS[mapper] if isinstance(mapper, str) else int(mapper)
    check(lib.prr_tonemap(m, exposure, _ptr(x), n, _ptr(out), _ptr(u8), _stream(stream)))
    return out, u8


def write_image(path, rgb8) -> None:
    """The 8-bit output files of Renderer::Render: (h, w, 3) uint8 (numpy or a
    CUDA tensor) to a .png or .ppm file."""
    a = rgb8.cpu().numpy() if hasattr(rgb8, "cpu") else rgb8
    a = np.ascontiguousarray(a, np.uint8)
    h, w = a.shape[:2]
    check(_lib.load().prr_write_image(str(path).encode(), C.c_void_p(a.ctypes.data), w, h))


def sample_count_image(spp, max_spp: int) -> np.ndarray:
    """The adaptive-sampling visualisation (h, w, 3) uint8 of an spp map."""
    a = spp.cpu().numpy() if hasattr(spp, "cpu") else spp
    a = np.ascontiguousarray(a, np.int32)
    out = np.empty(a.shape + (3,), np.uint8)
    check(_lib.load().prr_sample_count_image(C.c_void_p(a.ctypes.data), a.size, max_spp,
                                              C.c_void_p(out.ctypes.data)))
    return out


def read_obj(path, offset=(0.0, 0.0, 0.0)) -> np.ndarray:
    """The (ntri, 9) float32 triangles MeshTriangle(filename, offset, m) makes
    of an OBJ file."""
    lib = _lib.load()
    nt = C.c_int64()
    off = _f3(offset)
    check(lib.prr_obj_read(str(path).encode(), off, None, 0, C.byref(nt)))
    out = np.empty((nt.value, 9), np.float32)
    check(lib.prr_obj_read(str(path).encode(), off, C.c_void_p(out.ctypes.data), nt.value,
                           C.byref(nt)))
    return out


MEDIUM_PRESETS = {"dust": 0, "fog": 1}


def medium_preset(name: str) -> dict:
    """Medium::dust() / Medium::fog() (Volume.hpp:47-63) as a dict."""
    m = _lib.prr_medium()
    check(_lib.load().prr_medium_preset(MEDIUM_PRESETS[name], C.byref(m)))
    return {"sigma_a": m.sigma_a, "sigma_s": m.sigma_s, "sigma_t": m.sigma_t, "g": m.g,
            "bounded": False}


def _medium(d: dict):
    m = _lib.prr_medium()
    for k in ("sigma_a", "sigma_s", "sigma_t", "g"):
        setattr(m, k, float(d.get(k, 0.0)))
    m.bounded = 1 if d.get("bounded") else 0
    lo, hi = d.get("bounds", ((0.0,) * 3, (0.0,) * 3))
    m.bounds_min = (C.c_float * 3)(*map(float, lo))
    m.bounds_max = (C.c_float * 3)(*map(float, hi))
    return m


def medium_intersect(medium: dict, o, d, stream=None):
    """Medium::intersect for (n, 3) float32 CUDA tensors: (t_enter, t_exit,
    hit) with zeros where a ray misses the medium's box."""
    import torch
    n = o.shape[0]
    te = torch.empty(n, dtype=torch.float32, device=o.device)
    tx = torch.empty_like(te)
    hit = torch.empty(n, dtype=torch.uint8, device=o.device)
    m = _medium(medium)
    check(_lib.load().prr_medium_intersect(C.byref(m), _ptr(o), _ptr(d), n, _ptr(te), _ptr(tx),
                                           _ptr(hit), _stream(stream)))
    return te, tx, hit


def phase_hg(cos_theta, g: float, stream=None):
    """phaseHG(cos_theta, g) (Volume.cpp:3-6) of a float32 CUDA tensor."""
    import torch
    out = torch.empty_like(cos_theta)
    check(_lib.load().prr_phase_hg(_ptr(cos_theta), cos_theta.numel(), float(g), _ptr(out),
                                   _stream(stream)))
    return out


def phase_hg_sample(wo, g: float, seed: int = 1, stream=None):
    """samplePhaseHG(wo[k], g) (Volume.cpp:8-28) for an (n, 3) float32 CUDA
    tensor; item k draws from stream (seed, k, 0)."""
    import torch
    out = torch.empty_like(wo)
    check(_lib.load().prr_phase_hg_sample(_ptr(wo), wo.shape[0], float(g), seed, _ptr(out),
                                          _stream(stream)))
    return out


def _normalize_rows(v: np.ndarray) -> np.ndarray:
    """normalize (Vector.hpp:103-111) row by row in float32: v * (1 / sqrt(|v|^2))."""
    x, y, z = v[:, 0], v[:, 1], v[:, 2]
    m2 = x * x + y * y + z * z
    with np.errstate(divide="ignore"):
        inv = np.float32(1) / np.sqrt(m2)
    out = v * inv[:, None]
    return np.where((m2 > 0)[:, None], out, v).astype(np.float32)


def _trace_config(config: dict | None):
    if not config:
        return None
    return prr_trace_config(config.get("block_size", 0), config.get("persistent", 0),
                            config.get("blocks_per_sm", 0), config.get("batch", 0),
                            config.get("leaf_batch", 0), config.get("sort_rays", 0))


def _ptr(t):
    return C.c_void_p(0 if t is None else t.data_ptr())


def _stream(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _f3(x):
    return (C.c_float * 3)(*[float(v) for v in x])


def _rays(o, d):
    import torch
    o = o.to(torch.float32).contiguous()
    d = d.to(torch.float32).contiguous()
    if not o.is_cuda or not d.is_cuda:
        raise ValueError("device calls take CUDA tensors; use the *_host forms for host arrays")
    if o.shape != d.shape or o.shape[-1] != 3:
        raise ValueError("rays must be (n, 3) origins and directions")
    return o.reshape(-1, 3), d.reshape(-1, 3)


class Scene:
    def __init__(self):
        self.lib = _lib.load()
        h = C.c_void_p()
        check(self.lib.prr_scene_create(C.byref(h)))
        self.h = h
        self.objects = []
        self.desc = None
        self.size = None  # (width, height) of the camera, set by set_camera

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.prr_scene_destroy(h)
            self.h = None

    # ---- construction ----
    def add_material(self, kind: int, params) -> int:
        p = (C.c_float * 9)(*[float(x) for x in params])
        out = C.c_int()
        check(self.lib.prr_scene_add_material(self.h, kind, p, C.byref(out)))
        return out.value

    def add_mesh(self, verts, material: int) -> int:
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 9)
        out = C.c_int()
        check(self.lib.prr_scene_add_mesh(self.h, C.c_void_p(v.ctypes.data), len(v), material,
                                          C.byref(out)))
        self.objects.append(("mesh", len(v)))
        return out.value

    def add_mesh_attr(self, verts, material: int, normals=None, uvs=None, tangents=None,
                      normalize: bool = True) -> int:
        """MeshTriangle with per-corner normals (n, 9), uvs (n, 6) and tangents
        (n, 12: xyz + handedness per corner), any of them None. With
        `normalize` the corner normals are normalized first, as the glTF
        loader does (GLTFLoader.cpp:237-239), in the same float steps."""
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 9)
        if normals is not None and normalize:
            normals = _normalize_rows(np.ascontiguousarray(normals, np.float32).reshape(-1, 3))
        arrs = []
        for a, k in ((normals, 9), (uvs, 6), (tangents, 12)):
            arrs.append(None if a is None else np.ascontiguousarray(a, np.float32).reshape(-1, k))
        for a in arrs:
            if a is not None and len(a) != len(v):
                raise ValueError("per-corner arrays need one row per triangle")
        ptr = [C.c_void_p(a.ctypes.data) if a is not None else None for a in arrs]
        out = C.c_int()
        check(self.lib.prr_scene_add_mesh_attr(self.h, C.c_void_p(v.ctypes.data), ptr[0], ptr[1],
                                               ptr[2], len(v), material, C.byref(out)))
        self.objects.append(("mesh", len(v)))
        return out.value

    def add_texture(self, texels) -> int:
        """An 8-bit texture, (h, w, 3 or 4) uint8."""
        t = np.ascontiguousarray(texels, np.uint8)
        h, w, c = t.shape
        out = C.c_int()
        check(self.lib.prr_scene_add_texture(self.h, C.c_void_p(t.ctypes.data), w, h, c,
                                             C.byref(out)))
        return out.value

    def set_material_textures(self, material: int, base_color: int = -1,
                              metallic_roughness: int = -1, normal: int = -1, emissive: int = -1):
        check(self.lib.prr_scene_set_material_textures(self.h, material, base_color,
                                                       metallic_roughness, normal, emissive))

    GLTF_TYPES = {"diffuse": 0, "glass": 1, "mirror": 2, "emit": 3}

    def add_gltf(self, path: str, material_type: str = "diffuse",
                 override_material: int = -1) -> dict:
        """GLTFLoader::load + Scene::Add for every primitive: returns the first
        object added, how many, and how many images could not be decoded."""
        first, count, und = C.c_int(), C.c_int(), C.c_int()
        check(self.lib.prr_scene_add_gltf(self.h, str(path).encode(),
                                          self.GLTF_TYPES[material_type], override_material,
                                          C.byref(first), C.byref(count), C.byref(und)))
        for k in range(count.value):
            nt = C.c_int64()
            check(self.lib.prr_scene_export_mesh(self.h, first.value + k, C.byref(nt), None,
                                                 None, None, None, None))
            self.objects.append(("mesh", nt.value))
        return {"first": first.value, "count": count.value, "undecoded_images": und.value}

    def add_obj(self, path: str, material: int, offset=(0.0, 0.0, 0.0)) -> int:
        """MeshTriangle(filename, offset, m) + Scene::Add: the OBJ file's one
        mesh as the reference reads it; returns the object id."""
        out = C.c_int()
        check(self.lib.prr_scene_add_obj(self.h, str(path).encode(), _f3(offset), material,
                                         C.byref(out)))
        nt = C.c_int64()
        check(self.lib.prr_scene_export_mesh(self.h, out.value, C.byref(nt), None, None, None,
                                             None, None))
        self.objects.append(("mesh", nt.value))
        return out.value

    def export_mesh(self, obj: int) -> dict:
        """The mesh as added (host side): triangles and per-corner data."""
        nt, attr = C.c_int64(), C.c_int()
        check(self.lib.prr_scene_export_mesh(self.h, obj, C.byref(nt), C.byref(attr), None, None,
                                             None, None))
        n = nt.value
        out = {"verts": np.empty((n, 9), np.float32)}
        if attr.value & 1:
            out["normals"] = np.empty((n, 9), np.float32)
        if attr.value & 2:
            out["uvs"] = np.empty((n, 6), np.float32)
        if attr.value & 4:
            out["tangents"] = np.empty((n, 12), np.float32)
        ptr = lambda k: C.c_void_p(out[k].ctypes.data) if k in out else None  # noqa: E731
        check(self.lib.prr_scene_export_mesh(self.h, obj, None, None, ptr("verts"),
                                             ptr("normals"), ptr("uvs"), ptr("tangents")))
        return out

    def export_material(self, material: int) -> dict:
        kind = C.c_int()
        p = np.empty(9, np.float32)
        tex = np.empty(4, np.int32)
        check(self.lib.prr_scene_export_material(self.h, material, C.byref(kind),
                                                 C.c_void_p(p.ctypes.data),
                                                 C.c_void_p(tex.ctypes.data)))
        return {"kind": kind.value, "params": p, "textures": tex}

    def export_texture(self, texture: int) -> np.ndarray:
        w, h, c = C.c_int(), C.c_int(), C.c_int()
        check(self.lib.prr_scene_export_texture(self.h, texture, C.byref(w), C.byref(h),
                                                C.byref(c), None))
        t = np.empty((h.value, w.value, c.value), np.uint8)
        check(self.lib.prr_scene_export_texture(self.h, texture, None, None, None,
                                                C.c_void_p(t.ctypes.data)))
        return t

    def add_sphere(self, center, radius: float, material: int) -> int:
        out = C.c_int()
        check(self.lib.prr_scene_add_sphere(self.h, _f3(center), float(radius), material,
                                            C.byref(out)))
        self.objects.append(("sphere", 1))
        return out.value

    def set_background(self, rgb):
        check(self.lib.prr_scene_set_background(self.h, _f3(rgb)))

    def set_env(self, rgb):
        e = np.ascontiguousarray(rgb, np.float32)
        h, w = e.shape[:2]
        check(self.lib.prr_scene_set_env(self.h, C.c_void_p(e.ctypes.data), w, h))

    def set_camera(self, cam, width: int, height: int):
        c = prr_camera()
        c.eye[:] = list(map(float, cam.eye))
        c.target[:] = list(map(float, cam.target))
        c.up[:] = list(map(float, cam.up))
        c.fovv = cam.fovv
        c.fovh = cam.fovh
        c.aperture = cam.aperture
        c.focus_distance = cam.focus_distance
        check(self.lib.prr_scene_set_camera(self.h, C.byref(c), width, height))
        self.size = (int(width), int(height))

    def buildBVH(self, stream=None):
        check(self.lib.prr_scene_build(self.h, _stream(stream)))
        return self

    @classmethod
    def from_desc(cls, desc, build: bool = True) -> "Scene":
        s = cls()
        s.desc = desc
        for m in desc.materials:
            mid = s.add_material(int(m.kind), m.params())
            tex = [s.add_texture(t) if t is not None else -1 for t in m.texture_list()]
            if any(t >= 0 for t in tex):
                s.set_material_textures(mid, *tex)
        for o in desc.objects:
            if o.kind == "mesh" and o.has_attributes():
                s.add_mesh_attr(o.verts, o.material, o.normals, o.uvs, o.tangents)
            elif o.kind == "mesh":
                s.add_mesh(o.verts, o.material)
            else:
                s.add_sphere(o.center, o.radius, o.material)
        s.set_background(desc.background)
        if desc.env is not None:
            s.set_env(desc.env)
        s.set_camera(desc.camera, desc.width, desc.height)
        if build:
            s.buildBVH()
        return s

    @classmethod
    def single_mesh(cls, verts) -> "Scene":
        """One MeshTriangle (its own BVHAccel(ptrs, 4)) and nothing else."""
        s = cls()
        m = s.add_material(0, [0.8, 0.8, 0.8, 0.5, 0.0, 1.5, 0.0, 0.0, 0.0])
        s.add_mesh(verts, m)
        return s.buildBVH()

    # ---- inspection ----
    def stats(self) -> dict:
        st = prr_scene_stats()
        check(self.lib.prr_scene_stats_get(self.h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}

    def export_nodes(self, obj: int = -1) -> dict:
        n = check(self.lib.prr_scene_export_nodes(self.h, obj, None, None, None, None, None))
        nprim = len(self.objects) if obj < 0 else self.objects[obj][1]
        b = np.empty((n, 6), np.float32)
        fc = np.empty(n, np.uint32)
        meta = np.empty(n, np.uint32)
        area = np.empty(n, np.float32)
        order = np.empty(nprim, np.int32)
        check(self.lib.prr_scene_export_nodes(self.h, obj, b.ctypes.data, fc.ctypes.data,
                                              meta.ctypes.data, area.ctypes.data,
                                              order.ctypes.data))
        return dict(bounds=b, first_child=fc, meta=meta, area=area, ordered=order)

    # ---- batch queries (device) ----
    def mesh_intersect(self, obj: int, o, d, t64: bool = False, config: dict | None = None,
                       stream=None):
        """BVHAccel::Intersect on one mesh: (id int32, t float32[, t64 float64])."""
        import torch
        o, d = _rays(o, d)
        n = o.shape[0]
        hid = torch.empty(n, dtype=torch.int32, device=o.device)
        t = torch.empty(n, dtype=torch.float32, device=o.device)
        tt = torch.empty(n, dtype=torch.float64, device=o.device) if t64 else None
        cfg = None
        if config:
            cfg = _trace_config(config)
        check(self.lib.prr_mesh_intersect(self.h, obj, _ptr(o), _ptr(d), n, _ptr(hid), _ptr(t),
                                          _ptr(tt), C.byref(cfg) if cfg else None,
                                          _stream(stream)))
        return (hid, t, tt) if t64 else (hid, t)

    def mesh_intersect_host(self, obj: int, o, d, out_id=None, out_t=None,
                            config: dict | None = None, stream=None):
        o = np.ascontiguousarray(o, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(d, np.float32).reshape(-1, 3)
        n = len(o)
        hid = out_id if out_id is not None else np.empty(n, np.int32)
        t = out_t if out_t is not None else np.empty(n, np.float32)
        cfg = _trace_config(config)
        check(self.lib.prr_mesh_intersect_host(self.h, obj, C.c_void_p(o.ctypes.data),
                                               C.c_void_p(d.ctypes.data), n,
                                               C.c_void_p(hid.ctypes.data),
                                               C.c_void_p(t.ctypes.data),
                                               C.byref(cfg) if cfg is not None else None,
                                               _stream(stream)))
        return hid, t

    def mesh_occluded(self, obj: int, o, d, tmax, stream=None):
        import torch
        o, d = _rays(o, d)
        tmax = tmax.to(torch.float32).contiguous()
        out = torch.empty(o.shape[0], dtype=torch.uint8, device=o.device)
        check(self.lib.prr_mesh_occluded(self.h, obj, _ptr(o), _ptr(d), _ptr(tmax), o.shape[0],
                                         _ptr(out), _stream(stream)))
        return out

    def intersect(self, o, d, geo: bool = False, stream=None):
        """Scene::intersect: (obj, prim, t[, geo (n,6)])."""
        import torch
        o, d = _rays(o, d)
        n = o.shape[0]
        obj = torch.empty(n, dtype=torch.int32, device=o.device)
        prim = torch.empty(n, dtype=torch.int32, device=o.device)
        t = torch.empty(n, dtype=torch.float32, device=o.device)
        g = torch.empty((n, 6), dtype=torch.float32, device=o.device) if geo else None
        check(self.lib.prr_scene_intersect(self.h, _ptr(o), _ptr(d), n, _ptr(obj), _ptr(prim),
                                           _ptr(t), _ptr(g), _stream(stream)))
        return (obj, prim, t, g) if geo else (obj, prim, t)

    def intersectP(self, o, d, tmax, stream=None):
        """Scene::intersectP: uint8 per ray."""
        import torch
        o, d = _rays(o, d)
        tmax = tmax.to(torch.float32).contiguous()
        out = torch.empty(o.shape[0], dtype=torch.uint8, device=o.device)
        check(self.lib.prr_scene_occluded(self.h, _ptr(o), _ptr(d), _ptr(tmax), o.shape[0],
                                          _ptr(out), _stream(stream)))
        return out

    # ---- rendering (Renderer::Render up to the linear framebuffer) ----
    def _settings(self, spp, max_depth, seed, min_spp, threshold, mode, window, indirect_clamp,
                  sample_offset, slices):
        if self.size is None:
            raise ValueError("render needs a camera (set_camera or Scene.from_desc)")
        W, H = self.size
        x0, y0, x1, y1 = window or (0, 0, W, H)
        rs = prr_render_settings()
        rs.width, rs.height = W, H
        rs.min_spp = spp if min_spp is None else min_spp
        rs.max_spp = spp
        rs.max_depth = max_depth
        rs.variance_threshold = threshold
        rs.indirect_clamp = indirect_clamp
        rs.mode = RENDER_MODES[mode]
        rs.seed = seed
        rs.x0, rs.y0, rs.x1, rs.y1 = x0, y0, x1, y1
        rs.sample_offset = sample_offset
        rs.slices = slices
        return rs

    def set_wavefront(self, paths_per_pass: int = 0, block_size: int = 0, use_graphs: bool = True,
                      stack_smem: int = 0, ordered: bool = True, refill: int = 0):
        cfg = prr_wavefront_config(paths_per_pass, block_size, int(use_graphs), stack_smem,
                                   int(ordered), refill)
        check(self.lib.prr_scene_set_wavefront(self.h, C.byref(cfg)))

    def autotune(self, spp: int, max_depth: int, window=None, seed: int = 1, stream=None) -> dict:
        rs = self._settings(spp, max_depth, seed, None, 0.05, "wavefront", window, 10.0, 0, 0)
        best = prr_wavefront_config()
        check(self.lib.prr_autotune(self.h, C.byref(rs), C.byref(best), _stream(stream)))
        return {k: getattr(best, k) for k, _ in best._fields_}

    def render(self, spp: int, max_depth: int, seed: int = 1, min_spp: int | None = None,
               threshold: float = 0.05, mode: str = "plain", window=None,
               indirect_clamp: float = 10.0, sample_offset: int = 0, slices: int = 0,
               count_rays: bool = False, stream=None):
        """Mean radiance per pixel of the window: (h, w, 3) float32 CUDA tensor,
        plus samples per pixel and, with count_rays, (closest, shadow) rays."""
        import torch
        if self.size is None:
            raise ValueError("render needs a camera (set_camera or Scene.from_desc)")
        W, H = self.size
        x0, y0, x1, y1 = window or (0, 0, W, H)
        rs = prr_render_settings()
        rs.width, rs.height = W, H
        rs.min_spp = spp if min_spp is None else min_spp
        rs.max_spp = spp
        rs.max_depth = max_depth
        rs.variance_threshold = threshold
        rs.indirect_clamp = indirect_clamp
        rs.mode = RENDER_MODES[mode]
        rs.seed = seed
        rs.x0, rs.y0, rs.x1, rs.y1 = x0, y0, x1, y1
        rs.sample_offset = sample_offset
        rs.slices = slices
        dev = torch.device("cuda", torch.cuda.current_device())
        out = torch.empty(((y1 - y0), (x1 - x0), 3), dtype=torch.float32, device=dev)
        cnt = torch.empty(((y1 - y0), (x1 - x0)), dtype=torch.int32, device=dev)
        rays = torch.zeros(2, dtype=torch.int64, device=dev) if count_rays else None
        check(self.lib.prr_render(self.h, C.byref(rs), _ptr(out), _ptr(cnt), _ptr(rays),
                                  _stream(stream)))
        if count_rays:
            return out, cnt, rays
        return out, cnt

    def render_counts(self, spp: int, max_depth: int, seed: int = 1, min_spp: int | None = None,
                      threshold: float = 0.05, window=None, indirect_clamp: float = 10.0,
                      stream=None):
        """A wavefront render with counting traversal stages: (image, dict of
        rays, traversal steps and hit classes; see prr_render_count)."""
        import torch
        rs = self._settings(spp, max_depth, seed, min_spp, threshold, "wavefront", window,
                            indirect_clamp, 0, 0)
        x0, y0, x1, y1 = rs.x0, rs.y0, rs.x1, rs.y1
        dev = torch.device("cuda", torch.cuda.current_device())
        out = torch.empty(((y1 - y0), (x1 - x0), 3), dtype=torch.float32, device=dev)
        cnt = prr_render_count()
        check(self.lib.prr_render_counts(self.h, C.byref(rs), _ptr(out), C.byref(cnt),
                                         _stream(stream)))
        return out, {k: int(getattr(cnt, k)) for k, _ in cnt._fields_}

    # ---- per-call reference methods, batched ----
    def cast_samples(self, px, py, sample, max_depth: int, seed: int = 1,
                     indirect_clamp: float = 10.0, stream=None):
        """Integrator::castRay per (pixel, sample): (n, 3) radiance."""
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        px = torch.as_tensor(np.ascontiguousarray(px, np.int32)).to(dev)
        py = torch.as_tensor(np.ascontiguousarray(py, np.int32)).to(dev)
        sm = torch.as_tensor(np.ascontiguousarray(sample, np.int32)).to(dev)
        out = torch.empty((px.shape[0], 3), dtype=torch.float32, device=dev)
        check(self.lib.prr_cast_samples(self.h, _ptr(px), _ptr(py), _ptr(sm), px.shape[0], seed,
                                        max_depth, indirect_clamp, _ptr(out), _stream(stream)))
        return out

    def camera_rays(self, px, py, xo, yo, stream=None):
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        t = [torch.as_tensor(np.ascontiguousarray(a, dt)).to(dev)
             for a, dt in ((px, np.int32), (py, np.int32), (xo, np.float32), (yo, np.float32))]
        n = t[0].shape[0]
        o = torch.empty((n, 3), dtype=torch.float32, device=dev)
        d = torch.empty((n, 3), dtype=torch.float32, device=dev)
        check(self.lib.prr_camera_rays(self.h, *map(_ptr, t), n, _ptr(o), _ptr(d),
                                       _stream(stream)))
        return o, d

    def sample_light(self, seed: int, n: int, stream=None):
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        pos = torch.empty((n, 3), dtype=torch.float32, device=dev)
        nrm = torch.empty((n, 3), dtype=torch.float32, device=dev)
        pdf = torch.empty(n, dtype=torch.float32, device=dev)
        check(self.lib.prr_scene_sample_light(self.h, seed, n, _ptr(pos), _ptr(nrm), _ptr(pdf),
                                              _stream(stream)))
        return pos, nrm, pdf

    def env_eval(self, dirs, stream=None):
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        d = torch.as_tensor(np.ascontiguousarray(dirs, np.float32)).to(dev)
        rgb = torch.empty_like(d)
        pdf = torch.empty(d.shape[0], dtype=torch.float32, device=dev)
        check(self.lib.prr_env_eval(self.h, _ptr(d), d.shape[0], _ptr(rgb), _ptr(pdf),
                                    _stream(stream)))
        return rgb, pdf

    def env_importance_sample(self, seed: int, n: int, stream=None):
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        d = torch.empty((n, 3), dtype=torch.float32, device=dev)
        pdf = torch.empty(n, dtype=torch.float32, device=dev)
        check(self.lib.prr_env_importance_sample(self.h, seed, n, _ptr(d), _ptr(pdf),
                                                 _stream(stream)))
        return d, pdf

    def env_export(self):
        e = self.desc.env
        h, w = e.shape[:2]
        cdf = np.empty(h * w, np.float32)
        marg = np.empty(h, np.float32)
        tot = C.c_float()
        check(self.lib.prr_env_export(self.h, C.c_void_p(cdf.ctypes.data),
                                      C.c_void_p(marg.ctypes.data), C.byref(tot)))
        return cdf, marg, tot.value


class PhotonMap:
    """PhotonMap (Photon.hpp:32-45) on the device: emit/trace, grid build,
    irradiance gathers and the caustic image."""

    def __init__(self):
        self.lib = _lib.load()
        h = C.c_void_p()
        check(self.lib.prr_photon_map_create(C.byref(h)))
        self.h = h

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.prr_photon_map_destroy(h)
            self.h = None

    def emit(self, scene: Scene, num_photons: int, seed: int = 1, max_depth: int = 30,
             stream=None):
        check(self.lib.prr_photon_emit(self.h, scene.h, num_photons, seed, max_depth,
                                       _stream(stream)))
        return self

    def set(self, records, stream=None):
        r = np.ascontiguousarray(records, np.float32).reshape(-1, 9)
        check(self.lib.prr_photon_set(self.h, C.c_void_p(r.ctypes.data), len(r), _stream(stream)))
        return self

    def build(self, radius: float = 0.01, stream=None):
        check(self.lib.prr_photon_build(self.h, radius, _stream(stream)))
        return self

    def info(self):
        n = C.c_int64()
        res = C.c_int32()
        check(self.lib.prr_photon_info(self.h, C.byref(n), C.byref(res)))
        return n.value, res.value

    def launches(self) -> int:
        """Kernels launched so far by the calls on this photon map."""
        n = C.c_int64()
        check(self.lib.prr_photon_launches(self.h, C.byref(n)))
        return n.value

    def export(self):
        n, _ = self.info()
        rec = np.empty((n, 9), np.float32)
        owner = np.empty(n, np.int32)
        check(self.lib.prr_photon_export(self.h, C.c_void_p(rec.ctypes.data),
                                         C.c_void_p(owner.ctypes.data), _stream(None)))
        return rec, owner

    def gather(self, points, k_nearest: int = 0, stream=None):
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        q = torch.as_tensor(np.ascontiguousarray(points, np.float32)).to(dev).reshape(-1, 3)
        out = torch.empty_like(q)
        check(self.lib.prr_photon_gather(self.h, _ptr(q), q.shape[0], k_nearest, _ptr(out),
                                         _stream(stream)))
        return out

    def render_caustics(self, scene: Scene, spp: int, max_depth: int = 8, seed: int = 1,
                        k_nearest: int = 0, window=None, stream=None):
        import torch
        rs = scene._settings(spp, max_depth, seed, None, 0.05, "plain", window, 10.0, 0, 0)
        W, H = scene.size
        x0, y0, x1, y1 = window or (0, 0, W, H)
        dev = torch.device("cuda", torch.cuda.current_device())
        out = torch.empty(((y1 - y0), (x1 - x0), 3), dtype=torch.float32, device=dev)
        check(self.lib.prr_render_caustics(scene.h, self.h, C.byref(rs), k_nearest, _ptr(out),
                                           _stream(stream)))
        return out

    def render_caustics_counts(self, scene: Scene, spp: int, max_depth: int = 8, seed: int = 1,
                               k_nearest: int = 0, window=None, stream=None):
        """render_caustics with counting kernels: (image, dict of camera hits,
        gathers, photons tested and photons inside the radius)."""
        import torch
        rs = scene._settings(spp, max_depth, seed, None, 0.05, "plain", window, 10.0, 0, 0)
        W, H = scene.size
        x0, y0, x1, y1 = window or (0, 0, W, H)
        dev = torch.device("cuda", torch.cuda.current_device())
        out = torch.empty(((y1 - y0), (x1 - x0), 3), dtype=torch.float32, device=dev)
        cnt = (C.c_uint64 * 5)()
        check(self.lib.prr_render_caustics_counts(scene.h, self.h, C.byref(rs), k_nearest,
                                                  _ptr(out), cnt, _stream(stream)))
        keys = ("hits", "gathers", "photons_tested", "photons_inside", "dense_gathers")
        return out, dict(zip(keys, (int(x) for x in cnt)))


REQUEST_STATUS = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}


class Server:
    """The render server (continuous batching over resident scenes)."""

    def __init__(self, budget_bytes: int = 0, max_active: int = 0, samples_per_step: int = 0,
                 fail_every_nth_admission: int = 0, integrator: str = "wavefront",
                 paths_per_launch: int = 0):
        """`integrator`: "wavefront" (every running request's paths in one
        set of ordered ray queues per step) or "megakernel" (one launch over
        (request, tile) items per step)."""
        self.lib = _lib.load()
        kinds = {"wavefront": 0, "megakernel": 1}
        if integrator not in kinds:
            raise ValueError(f"integrator must be one of {sorted(kinds)}")
        cfg = prr_server_config(budget_bytes, max_active, samples_per_step,
                                fail_every_nth_admission, kinds[integrator], paths_per_launch)
        h = C.c_void_p()
        check(self.lib.prr_server_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self.scenes = []
        self._keep = {}

    def close(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.prr_server_destroy(h)
            self.h = None

    def __del__(self):
        self.close()

    def add_scene(self, scene: Scene) -> int:
        out = C.c_int()
        check(self.lib.prr_server_add_scene(self.h, scene.h, C.byref(out)))
        self.scenes.append(scene)
        return out.value

    def submit(self, scene_id: int, spp: int, max_depth: int, seed: int = 1, window=None,
               out=None, size=None) -> int:
        """Queue a render; `out` is a (h, w, 3) float32 CUDA tensor or a numpy
        array (pinned or pageable) that receives the image; `size` = (W, H)
        renders the scene's camera at another resolution."""
        sc = self.scenes[scene_id]
        rs = sc._settings(spp, max_depth, seed, None, 0.05, "plain", window, 10.0, 0, 0)
        W, H = size or sc.size
        rs.width, rs.height = W, H
        if window is None:
            rs.x0, rs.y0, rs.x1, rs.y1 = 0, 0, W, H
        x0, y0, x1, y1 = window or (0, 0, W, H)
        if out is None:
            out = np.empty((y1 - y0, x1 - x0, 3), np.float32)
        ptr = out.data_ptr() if hasattr(out, "data_ptr") else out.ctypes.data
        req = prr_request(scene_id, rs, C.c_void_p(ptr))
        rid = C.c_uint64()
        check(self.lib.prr_server_submit(self.h, C.byref(req), C.byref(rid)))
        self._keep[rid.value] = out
        return rid.value

    def result(self, rid: int):
        return self._keep[rid]

    def _info(self, info):
        d = {k: getattr(info, k) for k, _ in info._fields_}
        d["status"] = REQUEST_STATUS[d["status"]]
        return d

    def wait(self, rid: int, timeout: float = -1.0) -> dict:
        info = prr_request_info()
        check(self.lib.prr_server_wait(self.h, rid, timeout, C.byref(info)))
        return self._info(info)

    def poll(self, rid: int) -> dict:
        info = prr_request_info()
        check(self.lib.prr_server_poll(self.h, rid, C.byref(info)))
        return self._info(info)

    def cancel(self, rid: int):
        check(self.lib.prr_server_cancel(self.h, rid))

    def stats(self) -> dict:
        st = prr_server_stats()
        check(self.lib.prr_server_stats_get(self.h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}
