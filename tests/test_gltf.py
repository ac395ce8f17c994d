"""glTF 2.0 import (vitrum_b200.gltf, the reference's gltfToScene,
packages/gltf-adapter/src/gltfToScene.ts): accessors with strides, strip
triangulation, node hierarchy, instancing and flattening (mirrored winding),
materials with their KHR extensions, KHR_lights_punctual and the camera, from
a .gltf dict and from the same asset packed as .glb."""
import base64
import json
import math
import struct

import numpy as np
import pytest

from vitrum_b200.engine import DirectionalLight, PointLight, SpotLight
from vitrum_b200.gltf import GltfImportError, gltf_to_scene


def asset(as_glb=False):
    quad = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    interleaved = np.zeros((4, 4), np.float32)  # positions with a 16-byte stride
    interleaved[:, :3] = quad
    quad_idx = np.array([0, 1, 2, 0, 2, 3], np.uint16)
    strip = np.array([[0, 0, 1], [1, 0, 1], [0, 1, 1], [1, 1, 1]], np.float32)
    blob = interleaved.tobytes() + quad_idx.tobytes() + b"\0" * 4 + strip.tobytes()
    views = [{"buffer": 0, "byteOffset": 0, "byteLength": 64, "byteStride": 16},
             {"buffer": 0, "byteOffset": 64, "byteLength": 12},
             {"buffer": 0, "byteOffset": 80, "byteLength": 48}]
    accessors = [{"bufferView": 0, "componentType": 5126, "count": 4, "type": "VEC3"},
                 {"bufferView": 1, "componentType": 5123, "count": 6, "type": "SCALAR"},
                 {"bufferView": 2, "componentType": 5126, "count": 4, "type": "VEC3"}]
    s = math.sqrt(0.5)
    doc = {
        "asset": {"version": "2.0"},
        "buffers": [{"byteLength": len(blob)}],
        "bufferViews": views, "accessors": accessors,
        "materials": [
            {"pbrMetallicRoughness": {"baseColorFactor": [0.2, 0.4, 0.6, 1], "metallicFactor": 0.0,
                                      "roughnessFactor": 0.5},
             "emissiveFactor": [1, 0.5, 0], "doubleSided": True,
             "extensions": {"KHR_materials_emissive_strength": {"emissiveStrength": 2.0},
                            "KHR_materials_transmission": {"transmissionFactor": 0.3},
                            "KHR_materials_ior": {"ior": 1.4},
                            "KHR_materials_specular": {"specularFactor": 0.7}}},
            {}],
        "meshes": [{"primitives": [{"attributes": {"POSITION": 0}, "indices": 1, "material": 0}]},
                   {"primitives": [{"attributes": {"POSITION": 2}, "mode": 5, "material": 1},
                                   {"attributes": {"POSITION": 2}, "mode": 1}]}],  # lines: skipped
        "cameras": [{"type": "perspective", "perspective": {"yfov": 0.7, "znear": 0.05, "zfar": 50.0}}],
        "extensions": {"KHR_lights_punctual": {"lights": [
            {"type": "spot", "color": [1, 0.5, 0.25], "intensity": 4.0,
             "spot": {"innerConeAngle": 0.2, "outerConeAngle": 0.8}},
            {"type": "directional", "intensity": 3.0},
            {"type": "point", "intensity": 5.0, "range": 7.0},
            {"type": "point", "color": [0, 1, 0], "intensity": 2.0}]}},
        "nodes": [
            {"translation": [1, 2, 3], "children": [1, 2, 3]},
            {"mesh": 0, "scale": [2, 2, 2]},
            {"mesh": 0, "rotation": [0, s, 0, s]},                     # 90 degrees about +y
            {"mesh": 1, "matrix": [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 5, 0, 0, 1]},
            {"camera": 0, "translation": [0, 0, 10]},
            {"rotation": [-s, 0, 0, s], "translation": [0, 4, 0],     # -Z turned to -Y
             "extensions": {"KHR_lights_punctual": {"light": 0}}},
            {"extensions": {"KHR_lights_punctual": {"light": 1}}},
            {"translation": [3, 3, 3], "extensions": {"KHR_lights_punctual": {"light": 2}}},
            {"translation": [-1, 0, 0], "extensions": {"KHR_lights_punctual": {"light": 3}}},
            {"mesh": 0, "scale": [-1, 1, 1]},                          # mirrored
        ],
        "scenes": [{"nodes": [0, 4, 5, 6, 7, 8, 9]}],
        "scene": 0,
    }
    if not as_glb:
        doc["buffers"][0]["uri"] = "data:application/octet-stream;base64," + base64.b64encode(blob).decode()
        return doc
    js = json.dumps(doc).encode()
    js += b" " * (-len(js) % 4)
    binc = blob + b"\0" * (-len(blob) % 4)
    body = struct.pack("<I4s", len(js), b"JSON") + js + struct.pack("<I4s", len(binc), b"BIN\0") + binc
    return struct.pack("<4sII", b"glTF", 2, 12 + len(body)) + body


def check(sc, cam, emission=(2, 1, 0)):
    assert len(sc.meshes) == 2  # one prototype per triangle primitive
    q, st = sc.meshes
    assert np.array_equal(q.positions[:, 2], np.zeros(4)) and q.indices.tolist() == [[0, 1, 2], [0, 2, 3]]
    assert st.indices.tolist() == [[0, 1, 2], [2, 1, 3]]  # strip: alternate winding
    assert [i.mesh for i in sc.instances] == [0, 0, 1, 0]
    M = [np.asarray(i.local_to_world, np.float64) for i in sc.instances]
    assert np.allclose(M[0], [[2, 0, 0, 1], [0, 2, 0, 2], [0, 0, 2, 3], [0, 0, 0, 1]])
    assert np.allclose(M[1][:3, :3], [[0, 0, 1], [0, 1, 0], [-1, 0, 0]], atol=1e-6)
    assert np.allclose(M[1][:3, 3], [1, 2, 3]) and np.allclose(M[2][:3, 3], [6, 2, 3])
    assert np.allclose(M[3][:3, :3], np.diag([-1, 1, 1]))
    m0 = sc.materials[0]
    assert np.allclose(m0.base_color, (0.2, 0.4, 0.6)) and m0.metallic == 0 and m0.roughness == 0.5
    assert np.allclose(m0.emission, emission) and m0.transmission == pytest.approx(0.3)
    assert m0.ior == pytest.approx(1.4) and m0.specular_intensity == pytest.approx(0.7) and m0.double_sided
    m1 = sc.materials[1]  # glTF defaults: metallic 1, roughness 1, single-sided
    assert m1.metallic == 1 and m1.roughness == 1 and not m1.double_sided and m1.base_color == (1.0, 1.0, 1.0)
    assert [i.material for i in sc.instances] == [0, 0, 1, 0]
    # lights: spot (penumbra 1 - inner/outer, pointing down), directional along -Z, point with range, point
    sp = [l for l in sc.spot_lights if l.angle < 3]
    assert len(sp) == 1
    assert np.allclose(sp[0].position, (0, 4, 0)) and np.allclose(sp[0].direction, (0, -1, 0), atol=1e-6)
    assert sp[0].angle == pytest.approx(0.8) and sp[0].penumbra == pytest.approx(0.75)
    assert np.allclose(sp[0].intensity, (4, 2, 1))
    assert len(sc.directional_lights) == 1 and np.allclose(sc.directional_lights[0].direction, (0, 0, -1))
    ranged = [l for l in sc.spot_lights if l.angle > 3]
    assert len(ranged) == 1 and ranged[0].distance == 7.0 and np.allclose(ranged[0].position, (3, 3, 3))
    assert len(sc.point_lights) == 1 and np.allclose(sc.point_lights[0].intensity, (0, 2, 0))
    assert cam is not None and np.allclose(cam.eye, (0, 0, 10)) and np.allclose(cam.target, (0, 0, 9))
    assert cam.fov_y_deg == pytest.approx(math.degrees(0.7)) and cam.near == 0.05 and cam.far == 50.0


def test_gltf_dict_and_glb_import():
    doc = asset()
    doc["materials"][0]["emissiveFactor"] = [0, 0, 0]  # instancing needs non-emissive placements
    sc, cam = gltf_to_scene(doc)
    check(sc, cam, emission=(0, 0, 0))
    # the same asset packed as .glb, emissive: imported flattened by default, refused instanced
    sc2, cam2 = gltf_to_scene(asset(as_glb=True))
    assert not sc2.instances and len(sc2.meshes) == 4 and np.allclose(sc2.materials[0].emission, (2, 1, 0))
    with pytest.raises(GltfImportError):
        gltf_to_scene(asset(as_glb=True), instanced=True)
    glb = asset(as_glb=True)
    sc3, cam3 = gltf_to_scene(glb, instanced=None)
    assert np.allclose(sc3.meshes[0].positions, sc2.meshes[0].positions)


def test_flattened_import():
    sc, _ = gltf_to_scene(asset(), instanced=False)
    assert not sc.instances and len(sc.meshes) == 4
    assert np.allclose(sc.meshes[0].positions[2], (3, 4, 3))          # (1,1,0) * 2 + (1,2,3)
    assert np.allclose(sc.meshes[2].positions[3], (7, 3, 4))          # strip vertex (1,1,1) + (5,0,0) + (1,2,3)
    assert sc.meshes[3].indices.tolist() == [[0, 2, 1], [0, 3, 2]]    # mirrored: winding reversed
    assert len(sc.spot_lights) == 2 and len(sc.directional_lights) == 1  # lights survive flattening


def test_import_errors():
    doc = asset()
    doc["accessors"][1]["count"] = 60  # past its view
    with pytest.raises(GltfImportError):
        gltf_to_scene(doc)
    doc = asset()
    doc["extensions"]["KHR_lights_punctual"]["lights"][0]["spot"]["innerConeAngle"] = 0.9
    with pytest.raises(GltfImportError):
        gltf_to_scene(doc)
    doc = asset()
    doc["accessors"][0]["componentType"] = 5123
    with pytest.raises(GltfImportError):
        gltf_to_scene(doc)
    with pytest.raises(GltfImportError):
        gltf_to_scene(b"glTF\x01\x00\x00\x00\x0c\x00\x00\x00")


@pytest.mark.gpu
def test_imported_scene_renders_the_same_instanced_and_flattened(cuda):
    from vitrum_b200.engine import Engine
    imgs = []
    doc = asset()
    doc["materials"][0]["emissiveFactor"] = [0, 0, 0]
    for instanced in (True, False):
        sc, cam = gltf_to_scene(doc, instanced=instanced)
        e = Engine(max_bounces=3)
        e.set_scene(sc)
        e.render_frame(cam, 40, 30, samples=16, frame_seed=7)
        imgs.append(e.capture_frame().copy())
        e.dispose()
    assert imgs[0][..., :3].max() > 0
    assert np.isclose(imgs[0], imgs[1], rtol=1e-4, atol=1e-6).mean() > 0.999
