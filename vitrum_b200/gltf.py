"""glTF 2.0 -> Scene, the asset ingestion in front of the engine (the
reference's gltfToScene, packages/gltf-adapter/src/gltfToScene.ts).

Covered: .gltf (JSON with data-URI or external buffers) and .glb; float32
positions and uint8 / uint16 / uint32 indices, interleaved buffer views;
primitive modes triangles, strip and fan (points and lines are skipped); the
node hierarchy (matrix or TRS) with meshes placed as instances of prototype
meshes (one per mesh primitive) or flattened; metallic-roughness materials with
KHR_materials_emissive_strength / transmission / ior / specular and doubleSided;
KHR_lights_punctual (gltfToScene.ts:4308-4440: point, spot with penumbra
1 - inner / outer, directional, range as a distance cutoff, decay 2); the
first perspective camera.  Textures, skins, morph targets, animations and
compressed geometry are not read.
"""
from __future__ import annotations

import base64
import json
import math
import os
import struct
from typing import List, Optional, Tuple

import numpy as np

from .engine import Camera, DirectionalLight, Instance, Material, Mesh, PointLight, Scene, SpotLight

_COMPONENT = {5120: np.int8, 5121: np.uint8, 5122: np.int16, 5123: np.uint16, 5125: np.uint32, 5126: np.float32}
_WIDTH = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4, "MAT4": 16}


class GltfImportError(ValueError):
    """The asset is malformed or uses a feature this importer does not read."""


def _read_glb(data: bytes) -> Tuple[dict, Optional[bytes]]:
    magic, version, length = struct.unpack_from("<4sII", data, 0)
    if magic != b"glTF" or version != 2:
        raise GltfImportError("not a glTF 2.0 binary")
    off, doc, binc = 12, None, None
    while off + 8 <= min(length, len(data)):
        clen, ctype = struct.unpack_from("<I4s", data, off)
        chunk = data[off + 8: off + 8 + clen]
        if ctype == b"JSON":
            doc = json.loads(chunk.decode("utf-8"))
        elif ctype == b"BIN\x00" and binc is None:
            binc = bytes(chunk)
        off += 8 + clen + (-clen % 4)
    if doc is None:
        raise GltfImportError("glb without a JSON chunk")
    return doc, binc


def _buffers(doc: dict, base_dir: str, glb_bin: Optional[bytes]) -> List[bytes]:
    out = []
    for i, b in enumerate(doc.get("buffers", [])):
        uri = b.get("uri")
        if uri is None:
            if glb_bin is None:
                raise GltfImportError(f"buffer {i} has no uri and there is no binary chunk")
            data = glb_bin
        elif uri.startswith("data:"):
            data = base64.b64decode(uri.split(",", 1)[1])
        else:
            with open(os.path.join(base_dir, uri), "rb") as f:
                data = f.read()
        if len(data) < b.get("byteLength", 0):
            raise GltfImportError(f"buffer {i} is shorter than its byteLength")
        out.append(data)
    return out


def _accessor(doc: dict, bufs: List[bytes], index: int) -> np.ndarray:
    acc = doc["accessors"][index]
    if "sparse" in acc:
        raise GltfImportError(f"accessor {index}: sparse accessors are not read")
    dt = np.dtype(_COMPONENT[acc["componentType"]])
    width = _WIDTH[acc["type"]]
    count = acc["count"]
    if "bufferView" not in acc:
        return np.zeros((count, width), dt)
    view = doc["bufferViews"][acc["bufferView"]]
    data = bufs[view["buffer"]]
    start = view.get("byteOffset", 0) + acc.get("byteOffset", 0)
    elem = dt.itemsize * width
    stride = view.get("byteStride", elem) or elem
    end = start + stride * (count - 1) + elem if count else start
    if end > view.get("byteOffset", 0) + view["byteLength"] or end > len(data):
        raise GltfImportError(f"accessor {index} reads past its buffer view")
    raw = np.frombuffer(data, np.uint8, count=max(0, end - start), offset=start)
    if stride == elem:
        return raw.view(dt).reshape(count, width).copy()
    rows = np.lib.stride_tricks.as_strided(raw, shape=(count, elem), strides=(stride, 1))
    return np.ascontiguousarray(rows).view(dt).reshape(count, width)


def _triangles(mode: int, idx: np.ndarray) -> Optional[np.ndarray]:
    """Triangle list of a primitive (triangulation of strips and fans); None for points / lines."""
    if mode == 4:
        return idx[: len(idx) // 3 * 3].reshape(-1, 3)
    if mode == 5:  # strip: alternate winding
        tris = [(idx[i], idx[i + 1], idx[i + 2]) if i % 2 == 0 else (idx[i + 1], idx[i], idx[i + 2])
                for i in range(len(idx) - 2)]
        return np.asarray(tris, np.uint32).reshape(-1, 3)
    if mode == 6:  # fan
        tris = [(idx[0], idx[i], idx[i + 1]) for i in range(1, len(idx) - 1)]
        return np.asarray(tris, np.uint32).reshape(-1, 3)
    return None


def _local_matrix(node: dict) -> np.ndarray:
    if "matrix" in node:
        return np.asarray(node["matrix"], np.float64).reshape(4, 4).T  # column-major in the file
    t = np.asarray(node.get("translation", (0, 0, 0)), np.float64)
    x, y, z, w = node.get("rotation", (0, 0, 0, 1))
    r = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                  [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                  [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    s = np.asarray(node.get("scale", (1, 1, 1)), np.float64)
    m = np.eye(4)
    m[:3, :3] = r * s[None, :]
    m[:3, 3] = t
    return m


def _material(m: dict) -> Material:
    pbr = m.get("pbrMetallicRoughness", {})
    ext = m.get("extensions", {})
    base = pbr.get("baseColorFactor", (1, 1, 1, 1))
    strength = ext.get("KHR_materials_emissive_strength", {}).get("emissiveStrength", 1.0)
    emission = tuple(float(c) * strength for c in m.get("emissiveFactor", (0, 0, 0)))
    return Material(base_color=tuple(float(c) for c in base[:3]),
                    roughness=float(pbr.get("roughnessFactor", 1.0)),
                    metallic=float(pbr.get("metallicFactor", 1.0)),
                    transmission=float(ext.get("KHR_materials_transmission", {}).get("transmissionFactor", 0.0)),
                    ior=float(ext.get("KHR_materials_ior", {}).get("ior", 1.5)),
                    emission=emission,
                    double_sided=bool(m.get("doubleSided", False)),
                    specular_intensity=float(ext.get("KHR_materials_specular", {}).get("specularFactor", 1.0)))


def _light(light: dict, world: np.ndarray, where: str):
    kind = light.get("type")
    color = np.asarray(light.get("color", (1, 1, 1)), np.float64)
    intensity = float(light.get("intensity", 1.0))
    if not math.isfinite(intensity) or intensity < 0:
        raise GltfImportError(f"{where}.intensity must be finite and non-negative")
    rng = light.get("range")
    if rng is not None and not (math.isfinite(rng) and rng > 0):
        raise GltfImportError(f"{where}.range must be finite and > 0")
    rgb = tuple(color * intensity)
    pos = tuple(world[:3, 3])
    d = -world[:3, 2]  # lights shine along local -Z
    scale = np.abs(d).max()
    if kind != "point" and not (scale > 0 and np.isfinite(scale)):
        raise GltfImportError(f"{where}: the node transform gives no light direction")
    if kind != "point":
        d = d / scale
        d = tuple(d / np.linalg.norm(d))
    if kind == "point":
        if rng:
            return SpotLight(pos, (0.0, -1.0, 0.0), rgb, angle=math.pi, penumbra=0.0, distance=float(rng), decay=2.0)
        return PointLight(pos, rgb)
    if kind == "spot":
        spot = light.get("spot", {})
        inner, outer = float(spot.get("innerConeAngle", 0.0)), float(spot.get("outerConeAngle", math.pi / 4))
        if not (0 <= inner < outer <= math.pi / 2):
            raise GltfImportError(f"{where}.spot: need 0 <= innerConeAngle < outerConeAngle <= pi/2")
        pen = min(1.0, max(0.0, 1.0 - inner / outer)) if outer > 1e-10 else 0.0
        return SpotLight(pos, d, rgb, angle=outer, penumbra=pen, distance=float(rng or 0.0), decay=2.0)
    if kind == "directional":
        return DirectionalLight(d, rgb)  # travelling along the node's -Z
    raise GltfImportError(f"{where}: unknown light type {kind!r}")


def gltf_to_scene(source, instanced: Optional[bool] = None, scene_index: Optional[int] = None
                  ) -> Tuple[Scene, Optional[Camera]]:
    """Scene (and the first camera, or None) from a .gltf / .glb path, raw .glb
    bytes or an already parsed glTF dict (buffers as data URIs).  instanced:
    every mesh primitive is one prototype mesh placed by Instances (a two-level
    scene); False: the placed triangles are flattened into one mesh per
    placement; None (default): instanced unless a placement is emissive (the
    engine samples emitters from flat scenes only)."""
    base_dir, glb_bin = ".", None
    if isinstance(source, dict):
        doc = source
    elif isinstance(source, (bytes, bytearray)):
        doc, glb_bin = _read_glb(bytes(source))
    else:
        base_dir = os.path.dirname(os.path.abspath(source))
        with open(source, "rb") as f:
            raw = f.read()
        doc, glb_bin = _read_glb(raw) if raw[:4] == b"glTF" else (json.loads(raw.decode("utf-8")), None)
    if not str(doc.get("asset", {}).get("version", "2.0")).startswith("2"):
        raise GltfImportError("only glTF 2.0 is read")
    bufs = _buffers(doc, base_dir, glb_bin)
    materials = [_material(m) for m in doc.get("materials", [])]
    default_mat = len(materials)
    materials.append(Material(base_color=(1.0, 1.0, 1.0), metallic=1.0, roughness=1.0, double_sided=False))

    # prototypes: one per (mesh, primitive) with triangles
    protos: List[List[int]] = []
    meshes: List[Mesh] = []
    for mi, mesh in enumerate(doc.get("meshes", [])):
        ids = []
        for pi, prim in enumerate(mesh.get("primitives", [])):
            if "POSITION" not in prim.get("attributes", {}):
                continue
            pacc = doc["accessors"][prim["attributes"]["POSITION"]]
            if pacc["componentType"] != 5126 or pacc["type"] != "VEC3" or pacc.get("normalized"):
                raise GltfImportError(f"meshes[{mi}].primitives[{pi}]: positions must be float32 VEC3")
            pos = _accessor(doc, bufs, prim["attributes"]["POSITION"]).astype(np.float32)
            if "indices" in prim:
                idx = _accessor(doc, bufs, prim["indices"]).reshape(-1).astype(np.uint32)
            else:
                idx = np.arange(len(pos), dtype=np.uint32)
            tris = _triangles(prim.get("mode", 4), idx)
            if tris is None or len(tris) == 0:
                continue
            if tris.max() >= len(pos):
                raise GltfImportError(f"meshes[{mi}].primitives[{pi}]: index out of range")
            mat = prim.get("material", default_mat)
            if not 0 <= mat < default_mat + 1:
                raise GltfImportError(f"meshes[{mi}].primitives[{pi}]: no material {mat}")
            ids.append(len(meshes))
            meshes.append(Mesh(pos, np.ascontiguousarray(tris, np.uint32), int(mat)))
        protos.append(ids)

    scenes_ = doc.get("scenes", [])
    si = scene_index if scene_index is not None else doc.get("scene", 0)
    if scenes_:
        roots = scenes_[si]["nodes"] if si < len(scenes_) else []
    else:
        children = {c for n in doc.get("nodes", []) for c in n.get("children", [])}
        roots = [i for i in range(len(doc.get("nodes", []))) if i not in children]
    nodes = doc.get("nodes", [])
    lights_def = doc.get("extensions", {}).get("KHR_lights_punctual", {}).get("lights", [])
    instances: List[Instance] = []
    sc = Scene(meshes=meshes, materials=materials)
    camera: Optional[Camera] = None
    stack = [(r, np.eye(4), 0) for r in reversed(roots)]
    while stack:
        ni, parent, depth = stack.pop()
        if depth > 256:
            raise GltfImportError("node hierarchy deeper than 256 (or cyclic)")
        node = nodes[ni]
        world = parent @ _local_matrix(node)
        if "mesh" in node:
            for p in protos[node["mesh"]]:
                instances.append(Instance(p, world.astype(np.float32), meshes[p].material))
        if "camera" in node and camera is None:
            cam = doc["cameras"][node["camera"]]
            if cam.get("type") == "perspective":
                per = cam["perspective"]
                eye = world[:3, 3]
                fwd = -world[:3, 2] / np.linalg.norm(world[:3, 2])
                up = world[:3, 1] / np.linalg.norm(world[:3, 1])
                camera = Camera(eye=tuple(eye), target=tuple(eye + fwd), up=tuple(up),
                                fov_y_deg=math.degrees(per["yfov"]), near=float(per.get("znear", 0.01)),
                                far=float(per.get("zfar", 1000.0)))
        li = node.get("extensions", {}).get("KHR_lights_punctual", {}).get("light")
        if li is not None:
            lt = _light(lights_def[li], world, f"extensions.KHR_lights_punctual.lights[{li}]")
            {PointLight: sc.point_lights, SpotLight: sc.spot_lights,
             DirectionalLight: sc.directional_lights}[type(lt)].append(lt)
        for c in reversed(node.get("children", [])):
            stack.append((c, world, depth + 1))
    sc.instances = instances
    emissive = any(any(c > 0 for c in materials[i.material].emission) for i in instances)
    if instanced and emissive:
        raise GltfImportError("emissive materials are placed: import flattened (instanced=False or None)")
    if instanced is False or (instanced is None and emissive):
        sc = sc.flattened()
    return sc, camera
