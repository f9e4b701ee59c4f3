"""Test helper: writes small glTF 2.0 files (.glb, or .gltf with a base64
buffer and an external PNG) that exercise the ingest paths -- float and
normalized u8 / u16 texture coordinates, interleaved views with byteStride,
u8 / u16 / u32 / absent indices, materials with factors and PNG textures
(RGB, RGBA, grey, palette, 16-bit), several primitives per mesh."""
from __future__ import annotations

import base64
import io
import json
import struct

import numpy as np


def png_bytes(img: np.ndarray, mode: str | None = None) -> bytes:
    from PIL import Image
    im = Image.fromarray(img) if mode is None else Image.fromarray(img, mode)
    buf = io.BytesIO()
    im.save(buf, format="PNG")
    return buf.getvalue()


def png16_rgb(img16: np.ndarray) -> bytes:
    """A 16-bit RGB PNG written by hand (PIL has no 16-bit RGB writer)."""
    import zlib
    h, w, _ = img16.shape
    raw = b"".join(b"\x00" + img16[y].astype(">u2").tobytes() for y in range(h))

    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)
    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 16, 2, 0, 0, 0))
            + chunk(b"IDAT", zlib.compress(raw)) + chunk(b"IEND", b""))


class Builder:
    def __init__(self):
        self.bin = bytearray()
        self.doc = {"asset": {"version": "2.0"}, "buffers": [], "bufferViews": [],
                    "accessors": [], "meshes": [], "materials": [], "textures": [], "images": []}

    def _view(self, data: bytes, stride: int = 0) -> int:
        while len(self.bin) % 4:
            self.bin.append(0)
        v = {"buffer": 0, "byteOffset": len(self.bin), "byteLength": len(data)}
        if stride:
            v["byteStride"] = stride
        self.bin += data
        self.doc["bufferViews"].append(v)
        return len(self.doc["bufferViews"]) - 1

    def accessor(self, arr: np.ndarray, ctype: int, type_: str, view: int | None = None,
                 offset: int = 0, count: int | None = None) -> int:
        if view is None:
            view = self._view(np.ascontiguousarray(arr).tobytes())
        a = {"bufferView": view, "componentType": ctype, "type": type_,
             "count": int(count if count is not None else len(arr))}
        if offset:
            a["byteOffset"] = offset
        self.doc["accessors"].append(a)
        return len(self.doc["accessors"]) - 1

    def interleaved(self, pos: np.ndarray, nrm: np.ndarray):
        """POSITION and NORMAL in one view with byteStride 24."""
        data = np.concatenate([pos, nrm], 1).astype(np.float32)
        view = self._view(data.tobytes(), stride=24)
        return (self.accessor(None, 5126, "VEC3", view, 0, len(pos)),
                self.accessor(None, 5126, "VEC3", view, 12, len(pos)))

    def image(self, png: bytes) -> int:
        self.doc["images"].append({"bufferView": self._view(png), "mimeType": "image/png"})
        self.doc["textures"].append({"source": len(self.doc["images"]) - 1})
        return len(self.doc["textures"]) - 1

    def material(self, base=None, metallic=None, roughness=None, emissive=None,
                 base_tex=None, mr_tex=None, normal_tex=None, emissive_tex=None) -> int:
        m = {}
        pbr = {}
        if base is not None:
            pbr["baseColorFactor"] = list(map(float, base))
        if metallic is not None:
            pbr["metallicFactor"] = float(metallic)
        if roughness is not None:
            pbr["roughnessFactor"] = float(roughness)
        if base_tex is not None:
            pbr["baseColorTexture"] = {"index": base_tex}
        if mr_tex is not None:
            pbr["metallicRoughnessTexture"] = {"index": mr_tex}
        if pbr:
            m["pbrMetallicRoughness"] = pbr
        if emissive is not None:
            m["emissiveFactor"] = list(map(float, emissive))
        if normal_tex is not None:
            m["normalTexture"] = {"index": normal_tex}
        if emissive_tex is not None:
            m["emissiveTexture"] = {"index": emissive_tex}
        self.doc["materials"].append(m)
        return len(self.doc["materials"]) - 1

    def mesh(self, prims: list) -> None:
        self.doc["meshes"].append({"primitives": prims})

    def write_glb(self, path) -> None:
        self.doc["buffers"] = [{"byteLength": len(self.bin)}]
        js = json.dumps(self._clean()).encode()
        js += b" " * ((4 - len(js) % 4) % 4)
        b = bytes(self.bin) + b"\0" * ((4 - len(self.bin) % 4) % 4)
        total = 12 + 8 + len(js) + 8 + len(b)
        with open(path, "wb") as f:
            f.write(struct.pack("<4sII", b"glTF", 2, total))
            f.write(struct.pack("<II", len(js), 0x4E4F534A) + js)
            f.write(struct.pack("<II", len(b), 0x004E4942) + b)

    def write_gltf(self, path, external_image: bytes | None = None) -> None:
        """.gltf with the buffer as a base64 data URI; optionally one more
        image stored next to it as a file."""
        doc = self._clean()
        doc["buffers"] = [{"byteLength": len(self.bin), "uri": "data:application/octet-stream;"
                           "base64," + base64.b64encode(bytes(self.bin)).decode()}]
        if external_image is not None:
            import os
            name = os.path.splitext(os.path.basename(path))[0] + "_ext.png"
            with open(os.path.join(os.path.dirname(path), name), "wb") as f:
                f.write(external_image)
            doc.setdefault("images", []).append({"uri": name})
            doc.setdefault("textures", []).append({"source": len(doc["images"]) - 1})
        with open(path, "w") as f:
            json.dump(doc, f)

    def _clean(self):
        return {k: v for k, v in self.doc.items() if v or k in ("asset", "buffers")}


def grid(n: int, z: float = 0.0, jitter: float = 0.0, seed: int = 0):
    """An n x n vertex grid in [-1,1]^2 at height z with per-vertex normals,
    uvs and tangents, and its triangle indices."""
    rng = np.random.default_rng(seed)
    u = np.linspace(0, 1, n)
    x, y = np.meshgrid(u * 2 - 1, u * 2 - 1)
    h = z + jitter * rng.standard_normal(x.shape)
    pos = np.stack([x, h, y], -1).reshape(-1, 3).astype(np.float32)
    nrm = np.stack([0.2 * x, np.ones_like(x), -0.1 * y], -1).reshape(-1, 3).astype(np.float32)
    uv = np.stack(np.meshgrid(u * 2, u * 3), -1).reshape(-1, 2).astype(np.float32)
    tan = np.tile(np.array([[1, 0, 0, 1]], np.float32), (n * n, 1))
    tan[::3, 3] = -1
    idx = []
    for j in range(n - 1):
        for i in range(n - 1):
            a, b, c, d = j * n + i, j * n + i + 1, (j + 1) * n + i + 1, (j + 1) * n + i
            idx += [a, b, c, a, c, d]
    return pos, nrm, uv, tan, np.array(idx, np.uint32)


def feature_file(path, as_gltf: bool = False) -> None:
    """One file with every feature the ingest handles."""
    rng = np.random.default_rng(1)
    b = Builder()
    rgb = (rng.random((16, 16, 3)) * 255).astype(np.uint8)
    rgba = (rng.random((8, 12, 4)) * 255).astype(np.uint8)
    grey = (rng.random((8, 8)) * 255).astype(np.uint8)
    t_rgb = b.image(png_bytes(rgb))
    t_rgba = b.image(png_bytes(rgba))
    t_grey = b.image(png_bytes(grey, "L"))
    from PIL import Image
    pal_img = Image.fromarray((rng.random((8, 8, 3)) * 255).astype(np.uint8)).convert(
        "P", palette=Image.ADAPTIVE, colors=16)
    buf = io.BytesIO()
    pal_img.save(buf, format="PNG")
    t_pal = b.image(buf.getvalue())
    t_16 = b.image(png16_rgb((rng.random((6, 6, 3)) * 65535).astype(np.uint16)))
    m0 = b.material(base=(0.9, 0.5, 0.2, 1.0), metallic=0.3, roughness=0.7,
                    emissive=(0.0, 0.1, 0.0), base_tex=t_rgb, mr_tex=t_rgba, normal_tex=t_grey)
    m1 = b.material(base_tex=t_pal, emissive_tex=t_16)
    m2 = b.material(metallic=0.0, roughness=0.2)
    # primitive 1: float everything, u16 indices
    pos, nrm, uv, tan, idx = grid(6, 0.0, 0.02, seed=2)
    p = {"attributes": {"POSITION": b.accessor(pos, 5126, "VEC3"),
                        "NORMAL": b.accessor(nrm, 5126, "VEC3"),
                        "TEXCOORD_0": b.accessor(uv, 5126, "VEC2"),
                        "TANGENT": b.accessor(tan, 5126, "VEC4")},
         "indices": b.accessor(idx.astype(np.uint16), 5123, "SCALAR"), "material": m0}
    # primitive 2: interleaved position / normal, u16-normalized uvs, u32 indices
    pos2, nrm2, uv2, _, idx2 = grid(5, 0.5, 0.0, seed=3)
    a_pos, a_nrm = b.interleaved(pos2 * 0.6, nrm2)
    q = {"attributes": {"POSITION": a_pos, "NORMAL": a_nrm,
                        "TEXCOORD_0": b.accessor((np.clip(uv2 / 3, 0, 1) * 65535).astype(np.uint16),
                                                 5123, "VEC2")},
         "indices": b.accessor(idx2, 5125, "SCALAR"), "material": m1}
    b.mesh([p, q])
    # a second mesh: u8-normalized uvs, u8 indices, no normals; then a
    # non-indexed primitive without a material; then a line primitive (skipped)
    pos3, _, uv3, _, idx3 = grid(4, -0.3, 0.01, seed=4)
    r = {"attributes": {"POSITION": b.accessor(pos3 * 0.8, 5126, "VEC3"),
                        "TEXCOORD_0": b.accessor((np.clip(uv3 / 3, 0, 1) * 255).astype(np.uint8),
                                                 5121, "VEC2")},
         "indices": b.accessor(idx3.astype(np.uint8), 5121, "SCALAR"), "material": m2}
    soup = pos3[idx3][:18] + np.float32(0.05)
    s = {"attributes": {"POSITION": b.accessor(soup, 5126, "VEC3")}}
    line = {"attributes": {"POSITION": b.accessor(pos3[:4], 5126, "VEC3")}, "mode": 1}
    b.mesh([r, s, line])
    if as_gltf:
        b.write_gltf(str(path))
    else:
        b.write_glb(str(path))
