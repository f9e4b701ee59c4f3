"""Procedural scenes and query sets for the path-tracing hot path.

The reference renders hand-built museum scenes from .glb assets; none of those
assets ship with it, so every workload here is generated from a seed:

* ``query_set``      -- closest-hit query set: triangles with uniform centroids
                        in [0,1]^3 and N(0, 0.005^2) vertex jitter, rays from a
                        radius-2 sphere towards uniform points in the cube.
* ``cornell_box``    -- the plain-method Cornell box (10 wall/light triangles,
                        two r=0.3 spheres, a 2-triangle quad light of radiance 15).
* ``museum_like``    -- six displaced level-7 icospheres on a ground plane with
                        GGX materials, a glass sphere and a procedural HDR sky.
* ``caustics``       -- a glass sphere over a diffuse plane lit by a small
                        emissive sphere standing in for a point light.

All generators are deterministic numpy code; the GPU path and the oracle read
the same float32 arrays.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

# Material kinds (Material.hpp:120-183): DiffuseMaterial, EmissiveMaterial,
# MirrorMaterial, GlassMaterial.
DIFFUSE, EMISSIVE, MIRROR, GLASS = 0, 1, 2, 3

# Scene::backgroundColor default (Scene.hpp:17)
DEFAULT_BACKGROUND = (0.235294, 0.67451, 0.843137)


@dataclass
class Material:
    """Material fields as in Material.hpp:40-44 (defaults included)."""
    kind: int = DIFFUSE
    base_color: tuple = (0.8, 0.8, 0.8)
    roughness: float = 0.5
    metallic: float = 0.0
    ior: float = 1.5
    emission: tuple = (0.0, 0.0, 0.0)
    # textures, (h, w, 3 or 4) uint8 (Material.hpp:45-48)
    base_color_tex: Optional[np.ndarray] = None
    metallic_roughness_tex: Optional[np.ndarray] = None
    normal_tex: Optional[np.ndarray] = None
    emissive_tex: Optional[np.ndarray] = None

    def params(self) -> np.ndarray:
        return np.array([*self.base_color, self.roughness, self.metallic, self.ior,
                         *self.emission], np.float32)

    def texture_list(self) -> list:
        return [self.base_color_tex, self.metallic_roughness_tex, self.normal_tex,
                self.emissive_tex]


@dataclass
class MeshObject:
    verts: np.ndarray  # (n, 9) float32: v0, v1, v2 per triangle
    material: int
    kind: str = "mesh"
    # per-corner data (Triangle.hpp:17-23), None when absent
    normals: Optional[np.ndarray] = None   # (n, 9)
    uvs: Optional[np.ndarray] = None       # (n, 6)
    tangents: Optional[np.ndarray] = None  # (n, 12): xyz + handedness per corner

    def has_attributes(self) -> bool:
        return self.normals is not None or self.uvs is not None or self.tangents is not None


@dataclass
class SphereObject:
    center: tuple
    radius: float
    material: int
    kind: str = "sphere"


@dataclass
class Camera:
    """Camera.create fields (Camera.hpp:23-31); fovh alone sets the focal length."""
    eye: tuple = (0.0, 0.0, -1.0)
    target: tuple = (0.0, 0.0, 0.0)
    up: tuple = (0.0, 1.0, 0.0)
    fovv: float = 40.0
    fovh: float = 40.0
    aperture: float = 0.0
    focus_distance: float = -1.0


@dataclass
class SceneDesc:
    materials: List[Material] = field(default_factory=list)
    objects: list = field(default_factory=list)
    env: Optional[np.ndarray] = None  # (h, w, 3) float32, RGBE-exact values
    background: tuple = DEFAULT_BACKGROUND
    camera: Camera = field(default_factory=Camera)
    width: int = 256
    height: int = 256
    name: str = ""

    def add_material(self, m: Material) -> int:
        self.materials.append(m)
        return len(self.materials) - 1

    def n_triangles(self) -> int:
        return sum(len(o.verts) for o in self.objects if o.kind == "mesh")


# ---------------------------------------------------------------------------
# Closest-hit query set
# ---------------------------------------------------------------------------
def query_set(n_tris: int = 1_000_000, n_rays: int = 4_194_304, seed: int = 1,
              jitter: float = 0.005):
    """Triangles with centroids c ~ U[0,1]^3 and vertices c + N(0, jitter^2)^3;
    rays with origins uniform on the r=2 sphere (z ~ U[-1,1], phi ~ U[0,2pi))
    aimed at uniform points of the unit cube. Returns (verts (n,9), o, d)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    c = rng.random((n_tris, 1, 3))
    v = c + rng.normal(0.0, jitter, (n_tris, 3, 3))
    verts = v.reshape(n_tris, 9).astype(np.float32)
    z = rng.uniform(-1.0, 1.0, n_rays)
    phi = rng.uniform(0.0, 2.0 * math.pi, n_rays)
    s = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    o = 2.0 * np.stack([s * np.cos(phi), s * np.sin(phi), z], axis=1)
    tgt = rng.random((n_rays, 3))
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return verts, o.astype(np.float32), d.astype(np.float32)


# ---------------------------------------------------------------------------
# Geometry helpers
# ---------------------------------------------------------------------------
def quad(p0, p1, p2, p3) -> np.ndarray:
    """Two triangles (p0,p1,p2), (p0,p2,p3); normal = (p1-p0) x (p2-p0)."""
    p0, p1, p2, p3 = (np.asarray(p, np.float64) for p in (p0, p1, p2, p3))
    return np.stack([np.concatenate([p0, p1, p2]), np.concatenate([p0, p2, p3])]).astype(
        np.float32)


def icosphere(level: int) -> np.ndarray:
    """Unit icosphere as a triangle soup, float64 (20 * 4**level, 3, 3)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]],
                 np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9],
                  [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2],
                  [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
                  [8, 6, 7], [9, 8, 1]])
    tri = v[f]  # (20, 3, 3)
    for _ in range(level):
        a, b, c = tri[:, 0], tri[:, 1], tri[:, 2]
        # a+b is symmetric, so neighbouring triangles share bit-identical midpoints
        ab = a + b
        bc = b + c
        ca = c + a
        ab /= np.linalg.norm(ab, axis=1, keepdims=True)
        bc /= np.linalg.norm(bc, axis=1, keepdims=True)
        ca /= np.linalg.norm(ca, axis=1, keepdims=True)
        tri = np.concatenate([np.stack([a, ab, ca], 1), np.stack([ab, b, bc], 1),
                              np.stack([ca, bc, c], 1), np.stack([ab, bc, ca], 1)])
    return tri


def value_noise(p: np.ndarray, seed: int) -> np.ndarray:
    """Trilinear value noise in [-1,1] on the integer lattice, smoothstep fade."""
    i = np.floor(p).astype(np.int64)
    f = p - i
    u = f * f * (3.0 - 2.0 * f)

    def h(ix, iy, iz):
        k = (ix * 73856093) ^ (iy * 19349663) ^ (iz * 83492791) ^ (seed * 2654435761)
        k = k & 0xFFFFFFFF
        k = (k ^ (k >> 16)) * 0x45D9F3B & 0xFFFFFFFF
        k = (k ^ (k >> 16)) * 0x45D9F3B & 0xFFFFFFFF
        k = k ^ (k >> 16)
        return (k & 0xFFFFFF) / float(0xFFFFFF) * 2.0 - 1.0

    x, y, z = i[..., 0], i[..., 1], i[..., 2]
    out = 0.0
    for dx in (0, 1):
        wx = u[..., 0] if dx else 1.0 - u[..., 0]
        for dy in (0, 1):
            wy = u[..., 1] if dy else 1.0 - u[..., 1]
            for dz in (0, 1):
                wz = u[..., 2] if dz else 1.0 - u[..., 2]
                out = out + wx * wy * wz * h(x + dx, y + dy, z + dz)
    return out


def displaced_icosphere(level: int, center, radius: float, amplitude: float, seed: int,
                        octaves: int = 3) -> np.ndarray:
    """Icosphere with vertices moved along the normal by fractal value noise:
    r' = radius * (1 + amplitude * sum_o 0.5^o noise(4 * 2^o p))."""
    tri = icosphere(level)
    p = tri.reshape(-1, 3)
    disp = np.zeros(len(p))
    norm = 0.0
    for o in range(octaves):
        disp += 0.5 ** o * value_noise(p * (4.0 * 2 ** o), seed + o)
        norm += 0.5 ** o
    disp /= norm
    q = np.asarray(center, np.float64) + p * (radius * (1.0 + amplitude * disp))[:, None]
    return q.reshape(-1, 9).astype(np.float32)


# ---------------------------------------------------------------------------
# Environment map: procedural sky, quantised exactly as a Radiance .hdr stores it
# ---------------------------------------------------------------------------
def rgbe_quantize(rgb: np.ndarray) -> np.ndarray:
    """float RGB -> RGBE bytes -> float RGB, as stb_image_write v1.16's
    stbiw__linear_to_rgbe (stb_image_write.h:639-654) encodes and stb_image
    v2.28's stbi__hdr_convert (stb_image.h:7150-7175) decodes. The reference's
    EnvMap::load sees exactly these values, so both sides share them."""
    x = np.ascontiguousarray(rgb, np.float32).reshape(-1, 3)
    maxc = np.maximum(x[:, 0], np.maximum(x[:, 1], x[:, 2]))
    out = np.zeros_like(x)
    ok = maxc >= np.float32(1e-32)
    mant, ex = np.frexp(maxc[ok].astype(np.float64))
    normalize = (mant.astype(np.float32) * np.float32(256.0)) / maxc[ok]
    b = (x[ok] * normalize[:, None]).astype(np.float32)
    b = np.floor(b).astype(np.int32)  # (unsigned char) truncation of a non-negative value
    e = ex.astype(np.int32) + 128
    f1 = np.ldexp(np.float32(1.0), e - 136).astype(np.float32)
    out[ok] = b.astype(np.float32) * f1[:, None]
    return out.reshape(rgb.shape)


def uv_to_dir(u, v):
    """EnvMap::uvToDir (EnvMap.hpp:80-89), in float64."""
    phi = u * 2.0 * math.pi - math.pi
    theta = v * math.pi
    st = np.sin(theta)
    return np.stack([st * np.cos(phi), np.cos(theta), st * np.sin(phi)], -1)


def procedural_sky(width: int = 2048, height: int = 1024, sun_dir=(0.45, 0.55, -0.70),
                   dynamic_range: float = 1.0e4) -> np.ndarray:
    """Sky gradient plus a Gaussian sun lobe; peak / minimum luminance is about
    ``dynamic_range``. Returned RGBE-exact, (height, width, 3) float32."""
    u = (np.arange(width) + 0.5) / width
    v = (np.arange(height) + 0.5) / height
    uu, vv = np.meshgrid(u, v)
    d = uv_to_dir(uu, vv)
    y = d[..., 1]
    horizon = np.array([0.9, 0.85, 0.8])
    zenith = np.array([0.25, 0.45, 0.95])
    ground = np.array([0.12, 0.1, 0.08])
    t = np.clip(y, 0.0, 1.0)[..., None]
    sky = np.where(y[..., None] >= 0.0, horizon * (1 - t) + zenith * t, ground)
    sky = sky * 0.5
    s = np.asarray(sun_dir, np.float64)
    s /= np.linalg.norm(s)
    cosang = np.clip((d * s).sum(-1), -1.0, 1.0)
    ang = np.arccos(cosang)
    sigma = 0.03
    min_lum = float((sky @ np.array([0.2126, 0.7152, 0.0722])).min())
    peak = dynamic_range * min_lum
    sun = peak * np.exp(-0.5 * (ang / sigma) ** 2)
    rgb = sky + sun[..., None] * np.array([1.0, 0.95, 0.88])
    return rgbe_quantize(rgb.astype(np.float32))


# ---------------------------------------------------------------------------
# Scenes
# ---------------------------------------------------------------------------
def cornell_box(width: int = 256, height: int = 256) -> SceneDesc:
    """Room [-1,1]^3 open towards +z: floor, ceiling and back wall white 0.73,
    left wall red (0.65,0.05,0.05), right wall green (0.12,0.45,0.15), each a
    2-triangle mesh; a 0.5 x 0.5 quad light of radiance 15 just under the
    ceiling facing down; two diffuse spheres of radius 0.3. 'Lambertian' is the
    reference's DiffuseMaterial with metallic 0 and roughness 1, which still
    carries its 4% GGX lobe (Material.hpp:113-117)."""
    s = SceneDesc(width=width, height=height, name="cornell")
    white = s.add_material(Material(DIFFUSE, (0.73, 0.73, 0.73), 1.0, 0.0))
    red = s.add_material(Material(DIFFUSE, (0.65, 0.05, 0.05), 1.0, 0.0))
    green = s.add_material(Material(DIFFUSE, (0.12, 0.45, 0.15), 1.0, 0.0))
    light = s.add_material(Material(EMISSIVE, (0.8, 0.8, 0.8), 0.5, 0.0, 1.5, (15.0, 15.0, 15.0)))
    # floor (normal +y), ceiling (-y), back (+z), left (+x), right (-x)
    s.objects.append(MeshObject(quad((-1, -1, 1), (1, -1, 1), (1, -1, -1), (-1, -1, -1)), white))
    s.objects.append(MeshObject(quad((-1, 1, -1), (1, 1, -1), (1, 1, 1), (-1, 1, 1)), white))
    s.objects.append(MeshObject(quad((-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1)), white))
    s.objects.append(MeshObject(quad((-1, -1, 1), (-1, -1, -1), (-1, 1, -1), (-1, 1, 1)), red))
    s.objects.append(MeshObject(quad((1, -1, -1), (1, -1, 1), (1, 1, 1), (1, 1, -1)), green))
    y = 0.99
    s.objects.append(MeshObject(quad((-0.25, y, -0.25), (0.25, y, -0.25), (0.25, y, 0.25),
                                     (-0.25, y, 0.25)), light))
    s.objects.append(SphereObject((-0.4, -0.7, -0.3), 0.3, white))
    s.objects.append(SphereObject((0.45, -0.7, 0.3), 0.3, white))
    s.camera = Camera(eye=(0.0, 0.0, 3.5), target=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0),
                      fovv=40.0, fovh=40.0)
    return s


def checker_texture(n: int = 64, cells: int = 8, a=(220, 200, 160), b=(40, 60, 110),
                    channels: int = 3) -> np.ndarray:
    """An n x n sRGB checkerboard, (n, n, channels) uint8."""
    i = np.arange(n)
    mask = ((i[:, None] * cells // n + i[None, :] * cells // n) % 2).astype(bool)
    img = np.where(mask[..., None], np.array(a, np.uint8), np.array(b, np.uint8))
    if channels == 4:
        img = np.concatenate([img, np.full((n, n, 1), 255, np.uint8)], -1)
    return np.ascontiguousarray(img)


def bump_normal_map(n: int = 64, waves: float = 4.0, amp: float = 0.35) -> np.ndarray:
    """A tangent-space normal map of sine ripples, encoded (n*0.5+0.5)*255."""
    x = (np.arange(n) + 0.5) / n * 2 * math.pi * waves
    dx = amp * np.cos(x)[None, :].repeat(n, 0)
    dy = amp * np.cos(x)[:, None].repeat(n, 1)
    nrm = np.stack([-dx, -dy, np.ones_like(dx)], -1)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    return np.clip(np.round((nrm * 0.5 + 0.5) * 255), 0, 255).astype(np.uint8)


def metal_rough_map(n: int = 32) -> np.ndarray:
    """glTF metallic-roughness texels: G = roughness ramp, B = metallic stripes."""
    img = np.zeros((n, n, 4), np.uint8)
    img[..., 1] = np.linspace(20, 240, n, dtype=np.float64)[None, :].round().astype(np.uint8)
    img[..., 2] = np.where((np.arange(n) // 4) % 2 == 0, 230, 10)[:, None].astype(np.uint8)
    img[..., 3] = 255
    return img


def uv_sphere_attrs(tri: np.ndarray):
    """Per-corner normals, spherical uvs and tangents (d/dphi, w = +1) of a
    unit-sphere triangle soup (n, 3, 3)."""
    n = tri / np.linalg.norm(tri, axis=-1, keepdims=True)
    phi = np.arctan2(n[..., 2], n[..., 0])
    u = phi / (2 * math.pi) + 0.5
    v = np.arccos(np.clip(n[..., 1], -1, 1)) / math.pi
    # keep a triangle's u on one side of the seam
    span = u.max(1, keepdims=True) - u.min(1, keepdims=True)
    u = np.where((span > 0.5) & (u < 0.5), u + 1.0, u)
    tan = np.stack([-np.sin(phi), np.zeros_like(phi), np.cos(phi)], -1)
    tan = np.concatenate([tan, np.ones(phi.shape + (1,))], -1)
    return (n.reshape(-1, 9).astype(np.float32), np.stack([u, v], -1).reshape(-1, 6).astype(
        np.float32), tan.reshape(-1, 12).astype(np.float32))


def textured_showcase(width: int = 320, height: int = 240, env_size=(256, 128)) -> SceneDesc:
    """Per-corner data and textures on the path: a floor grid (uv tiling,
    tangents, base-colour checker, metallic-roughness map, ripple normal map),
    a smooth-shaded icosphere (interpolated normals, spherical uvs, tangents,
    checker and normal map), a glass sphere over it, a quad light and a sky."""
    s = SceneDesc(width=width, height=height, name="textured")
    floor_m = s.add_material(Material(DIFFUSE, (1.0, 1.0, 1.0), 0.6, 0.0,
                                      base_color_tex=checker_texture(64, 8),
                                      metallic_roughness_tex=metal_rough_map(32),
                                      normal_tex=bump_normal_map(64, 4.0)))
    ball_m = s.add_material(Material(DIFFUSE, (1.0, 1.0, 1.0), 0.35, 0.3,
                                     base_color_tex=checker_texture(
                                         32, 6, (200, 60, 50), (240, 230, 200), channels=4),
                                     normal_tex=bump_normal_map(32, 6.0, 0.25)))
    glass = s.add_material(Material(GLASS, (0.95, 1.0, 0.97), 0.0, 0.0, 1.5))
    le = 12.0
    light = s.add_material(Material(EMISSIVE, (0.8, 0.8, 0.8), 0.5, 0.0, 1.5, (le, le, le)))
    # floor: a 6 x 6 grid of quads on y = 0, uvs tiled 3x, tangent +x
    g = np.linspace(-3.0, 3.0, 7)
    tris, uvs = [], []
    for i in range(6):
        for j in range(6):
            a = (g[i], 0.0, g[j + 1])
            b = (g[i + 1], 0.0, g[j + 1])
            c = (g[i + 1], 0.0, g[j])
            d = (g[i], 0.0, g[j])
            ua = [(x + 3) / 2.0 for x in (a[0], a[2])]
            ub = [(x + 3) / 2.0 for x in (b[0], b[2])]
            uc = [(x + 3) / 2.0 for x in (c[0], c[2])]
            ud = [(x + 3) / 2.0 for x in (d[0], d[2])]
            tris += [a + b + c, a + c + d]
            uvs += [ua + ub + uc, ua + uc + ud]
    fv = np.array(tris, np.float32)
    nf = len(fv)
    s.objects.append(MeshObject(fv, floor_m,
                                normals=np.tile(np.array([0, 1, 0] * 3, np.float32), (nf, 1)),
                                uvs=np.array(uvs, np.float32),
                                tangents=np.tile(np.array([1, 0, 0, 1] * 3, np.float32),
                                                 (nf, 1))))
    ico = icosphere(3)
    nrm, uv, tan = uv_sphere_attrs(ico)
    center, r = np.array([-0.8, 0.9, 0.2]), 0.9
    s.objects.append(MeshObject((ico * r + center).reshape(-1, 9).astype(np.float32), ball_m,
                                normals=nrm, uvs=uv, tangents=tan))
    s.objects.append(SphereObject((1.1, 0.7, 0.6), 0.7, glass))
    y = 3.2
    s.objects.append(MeshObject(quad((-0.6, y, -0.6), (0.6, y, -0.6), (0.6, y, 0.6),
                                     (-0.6, y, 0.6)), light))
    s.env = procedural_sky(*env_size)
    s.camera = Camera(eye=(0.0, 2.2, 5.0), target=(0.0, 0.6, 0.0), up=(0.0, 1.0, 0.0),
                      fovv=45.0, fovh=50.0)
    return s


def museum_like(width: int = 1920, height: int = 1080, level: int = 7, seed: int = 1,
                env_size=(2048, 1024), amplitude: float = 0.05, spheres: int = 6) -> SceneDesc:
    """Six (or the first ``spheres``) displaced level-``level`` icospheres
    (20*4^level triangles each) in a 3x2 grid on a ground quad; GGX alpha ~
    U[0.05,0.8] (roughness = sqrt(alpha)), metallic ~ Bernoulli(0.5), base
    colour ~ U[0.2,0.9]^3; sphere 4 is glass (IOR 1.5); lit only by a
    procedural HDR sky."""
    rng = np.random.Generator(np.random.PCG64(seed))
    s = SceneDesc(width=width, height=height, name="museum_like")
    ground = s.add_material(Material(DIFFUSE, (0.5, 0.5, 0.5), 0.7, 0.0))
    s.objects.append(MeshObject(quad((-30, 0, 30), (30, 0, 30), (30, 0, -30), (-30, 0, -30)),
                                ground))
    r = 0.8
    for k in range(spheres):
        cx = (k % 3 - 1) * 2.2
        cz = (k // 3) * -2.2 + 1.0
        alpha = rng.uniform(0.05, 0.8)
        metallic = float(rng.random() < 0.5)
        base = tuple(rng.uniform(0.2, 0.9, 3))
        if k == 4:
            m = s.add_material(Material(GLASS, (1.0, 1.0, 1.0), 0.0, 0.0, 1.5))
        else:
            m = s.add_material(Material(DIFFUSE, base, math.sqrt(alpha), metallic))
        s.objects.append(MeshObject(displaced_icosphere(level, (cx, r, cz), r, amplitude,
                                                        seed * 100 + k), m))
    s.env = procedural_sky(*env_size)
    s.camera = Camera(eye=(0.0, 2.6, 6.5), target=(0.0, 0.6, -0.2), up=(0.0, 1.0, 0.0),
                      fovv=34.0, fovh=55.0)
    return s


def caustics(width: int = 1024, height: int = 1024, light_radius: float = 0.05,
             intensity: float = 100.0, level: int = 3) -> SceneDesc:
    """Glass sphere (r=1, IOR 1.5) resting over a diffuse plane, lit by an
    emissive icosphere of radius ``light_radius`` at (0,4,0) whose radiance
    L = I / (pi r^2) gives the power 4 pi I of a point light of intensity I.
    The reference has no point-light emission (PointLight.hpp is unused and
    Photon.cpp:168 samples area emitters only), hence the small sphere."""
    s = SceneDesc(width=width, height=height, name="caustics")
    floor = s.add_material(Material(DIFFUSE, (0.8, 0.8, 0.8), 1.0, 0.0))
    glass = s.add_material(Material(GLASS, (1.0, 1.0, 1.0), 0.0, 0.0, 1.5))
    le = intensity / (math.pi * light_radius ** 2)
    light = s.add_material(Material(EMISSIVE, (0.8, 0.8, 0.8), 0.5, 0.0, 1.5, (le, le, le)))
    s.objects.append(MeshObject(quad((-6, 0, 6), (6, 0, 6), (6, 0, -6), (-6, 0, -6)), floor))
    s.objects.append(SphereObject((0.0, 1.05, 0.0), 1.0, glass))
    tri = icosphere(level) * light_radius + np.array([0.0, 4.0, 0.0])
    s.objects.append(MeshObject(tri.reshape(-1, 9).astype(np.float32), light))
    s.camera = Camera(eye=(0.0, 3.5, 5.5), target=(0.0, 0.5, 0.0), up=(0.0, 1.0, 0.0),
                      fovv=45.0, fovh=45.0)
    return s
