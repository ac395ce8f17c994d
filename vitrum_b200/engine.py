"""The vitrum Engine contract on the B200 path tracer.

Mirrors @vitrum/core's Engine (packages/core/src/engine/index.ts:109-466) as
implemented by pt-webgpu (packages/pt-webgpu/src/index.ts): a Scene goes in
through set_scene(), render_frame() adds samples to a progressive
accumulation, capture_frame() returns the running mean as RGBA float32
(row-major, top-left), debug.pick_primitive(x, y) returns the triangle under a
pixel, reset() clears the accumulation, dispose() releases the device state.
All work happens in libvitrum_pt.so (vt_create ... vt_destroy).
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _native as N


# ---------------------------------------------------------------- C structs
class _EngineOptions(ctypes.Structure):
    _fields_ = [("max_bounces", ctypes.c_int32), ("max_samples_per_pixel", ctypes.c_int32),
                ("debug", ctypes.c_int32), ("oracle_accumulation", ctypes.c_int32),
                ("sort_by_material", ctypes.c_int32), ("wave_paths", ctypes.c_int32),
                ("bvh_max_leaf", ctypes.c_int32), ("light_selection", ctypes.c_int32),
                ("scene_build", ctypes.c_int32), ("bvh_width", ctypes.c_int32)]


class _BvhShapeTrial(ctypes.Structure):
    _fields_ = [("bvh_width", ctypes.c_int32), ("bvh_max_leaf", ctypes.c_int32), ("frame_ms", ctypes.c_double)]


class _MaterialDesc(ctypes.Structure):
    _fields_ = [("base_color", ctypes.c_float * 3), ("roughness", ctypes.c_float), ("metallic", ctypes.c_float),
                ("transmission", ctypes.c_float), ("ior", ctypes.c_float), ("emission", ctypes.c_float * 3),
                ("flags", ctypes.c_uint32), ("specular_intensity", ctypes.c_float)]


class _MeshDesc(ctypes.Structure):
    _fields_ = [("positions", ctypes.c_void_p), ("vertex_count", ctypes.c_size_t), ("indices", ctypes.c_void_p),
                ("triangle_count", ctypes.c_size_t), ("material", ctypes.c_uint32)]


class _PointLightDesc(ctypes.Structure):
    _fields_ = [("position", ctypes.c_float * 3), ("intensity", ctypes.c_float * 3)]


class _InstanceDesc(ctypes.Structure):
    _fields_ = [("mesh", ctypes.c_uint32), ("material", ctypes.c_uint32), ("local_to_world", ctypes.c_float * 16)]


class _DirectionalDesc(ctypes.Structure):
    _fields_ = [("direction", ctypes.c_float * 3), ("irradiance", ctypes.c_float * 3), ("angular_radius", ctypes.c_float)]


class _RectDesc(ctypes.Structure):
    _fields_ = [("corner", ctypes.c_float * 3), ("edge_u", ctypes.c_float * 3), ("edge_v", ctypes.c_float * 3),
                ("radiance", ctypes.c_float * 3)]


class _SpotDesc(ctypes.Structure):
    _fields_ = [("position", ctypes.c_float * 3), ("direction", ctypes.c_float * 3), ("intensity", ctypes.c_float * 3),
                ("angle", ctypes.c_float), ("penumbra", ctypes.c_float), ("distance", ctypes.c_float),
                ("decay", ctypes.c_float)]


class _DiscDesc(ctypes.Structure):
    _fields_ = [("center", ctypes.c_float * 3), ("normal", ctypes.c_float * 3), ("radius", ctypes.c_float),
                ("radiance", ctypes.c_float * 3)]


class _Capabilities(ctypes.Structure):
    _fields_ = [("max_bounces_limit", ctypes.c_int32), ("max_samples_per_pixel", ctypes.c_int32),
                ("max_viewport", ctypes.c_int32), ("emitter_kinds", ctypes.c_uint32),
                ("material_features", ctypes.c_uint32), ("features", ctypes.c_uint32)]


class _PresentOptions(ctypes.Structure):
    _fields_ = [("tonemap", ctypes.c_int32), ("exposure", ctypes.c_float), ("srgb", ctypes.c_int32)]


class _SceneDesc(ctypes.Structure):
    _fields_ = [("meshes", ctypes.c_void_p), ("mesh_count", ctypes.c_size_t), ("instances", ctypes.c_void_p),
                ("instance_count", ctypes.c_size_t), ("materials", ctypes.c_void_p),
                ("material_count", ctypes.c_size_t), ("point_lights", ctypes.c_void_p),
                ("point_light_count", ctypes.c_size_t), ("environment_rgb", ctypes.c_void_p),
                ("environment_width", ctypes.c_int32), ("environment_height", ctypes.c_int32),
                ("environment_intensity", ctypes.c_float), ("directional_lights", ctypes.c_void_p),
                ("directional_light_count", ctypes.c_size_t), ("rect_lights", ctypes.c_void_p),
                ("rect_light_count", ctypes.c_size_t), ("spot_lights", ctypes.c_void_p),
                ("spot_light_count", ctypes.c_size_t), ("disc_lights", ctypes.c_void_p),
                ("disc_light_count", ctypes.c_size_t), ("environment_rotation_y", ctypes.c_float)]


class _FrameInput(ctypes.Structure):
    _fields_ = [("view", ctypes.c_float * 16), ("projection", ctypes.c_float * 16), ("width", ctypes.c_int32),
                ("height", ctypes.c_int32), ("frame_seed", ctypes.c_uint32), ("samples", ctypes.c_int32),
                ("bounces", ctypes.c_int32)]


class _FrameOutput(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("samples_accumulated", ctypes.c_int32), ("is_converged", ctypes.c_int32),
                ("width", ctypes.c_int32), ("height", ctypes.c_int32), ("radiance_device", ctypes.c_void_p)]


class _StageTimes(ctypes.Structure):
    _fields_ = [("raygen_ms", ctypes.c_double), ("trace_closest_ms", ctypes.c_double), ("sort_ms", ctypes.c_double),
                ("shade_ms", ctypes.c_double), ("trace_shadow_ms", ctypes.c_double), ("resolve_ms", ctypes.c_double),
                ("accumulate_ms", ctypes.c_double), ("frame_ms", ctypes.c_double),
                ("trace_closest_launches", ctypes.c_int32), ("trace_shadow_launches", ctypes.c_int32),
                ("nrc_train_ms", ctypes.c_double), ("nrc_query_ms", ctypes.c_double)]


class _NrcRenderOptions(ctypes.Structure):
    from .nrc import _Config as _NrcConfig
    _fields_ = [("enabled", ctypes.c_int32), ("prefix_bounces", ctypes.c_int32), ("train_steps", ctypes.c_int32),
                ("train_batch", ctypes.c_int32), ("train_paths", ctypes.c_int32), ("warmup_frames", ctypes.c_int32),
                ("cache", _NrcConfig), ("fallback_error", ctypes.c_float), ("fallback_tile", ctypes.c_int32),
                ("spread_c", ctypes.c_float)]


class _EngineStats(ctypes.Structure):
    _fields_ = [("closest_rays", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64),
                ("last_frame_ms", ctypes.c_double), ("triangle_count", ctypes.c_int64),
                ("emitter_count", ctypes.c_int64)]


# ---------------------------------------------------------------- scene types
@dataclass
class Material:
    """core MaterialSpec subset with the reference's base BSDF.  transmission > 0
    with metallic 0: dielectric interface (delta at roughness 0, rough GGX
    otherwise); anything else opaque: Lambert diffuse under a GGX specular layer
    (F0 = mix(specular_intensity * ((ior-1)/(ior+1))^2, base_color, metallic),
    Kulla-Conty multiple scattering).  specular_intensity=0 with metallic 0 is a
    pure Lambertian.  emission is front-face radiance."""
    base_color: Sequence[float] = (0.8, 0.8, 0.8)
    roughness: float = 1.0
    metallic: float = 0.0
    transmission: float = 0.0
    ior: float = 1.5
    emission: Sequence[float] = (0.0, 0.0, 0.0)
    double_sided: bool = True   # False: back-face hits are skipped by every ray
    cast_shadow: bool = True    # False: shadow rays pass through (castShadow: false)
    specular_intensity: float = 1.0  # KHR_materials_specular factor (MaterialSpec.specularIntensity)

    @property
    def flags(self) -> int:
        return (0 if self.double_sided else 1) | (0 if self.cast_shadow else 2)


@dataclass
class Mesh:
    positions: np.ndarray  # (V, 3) float32 world space
    indices: np.ndarray    # (T, 3) uint32
    material: int = 0


@dataclass
class Instance:
    """A placement of meshes[mesh] (core instanced mesh; TLAS instance, shared-bvh/src/tlas.ts:859).

    local_to_world is a 4x4 row-major matrix (affine, invertible)."""
    mesh: int
    local_to_world: np.ndarray
    material: int = 0


@dataclass
class PointLight:
    position: Sequence[float]
    intensity: Sequence[float]


@dataclass
class DirectionalLight:
    """Light travelling along `direction`; angular_radius 0: delta light of that
    irradiance, else a disc of that angular radius and irradiance."""
    direction: Sequence[float]
    irradiance: Sequence[float]
    angular_radius: float = 0.0


@dataclass
class SpotLight:
    """core SpotEmitter: delta light at `position` emitting `intensity` into the cone of
    half-angle `angle` (radians) around `direction`, with a smooth edge from
    angle * (1 - penumbra), falloff 1 / d^decay and an optional range `distance` (0: none)."""
    position: Sequence[float]
    direction: Sequence[float]
    intensity: Sequence[float]
    angle: float
    penumbra: float = 0.0
    distance: float = 0.0
    decay: float = 2.0


@dataclass
class DiscLight:
    """core DiscAreaEmitter: disc of `radius` at `center` emitting `radiance` towards `normal`."""
    center: Sequence[float]
    normal: Sequence[float]
    radius: float
    radiance: Sequence[float]


@dataclass
class RectLight:
    """corner + [0,1] edge_u + [0,1] edge_v emitting `radiance` towards edge_u x edge_v
    (an analytic emitter: never an occluder)."""
    corner: Sequence[float]
    edge_u: Sequence[float]
    edge_v: Sequence[float]
    radiance: Sequence[float]


@dataclass
class Environment:
    rgb: np.ndarray        # (H, W, 3) float32 equirectangular: row 0 at +y, u = atan2(z, x)/2pi + 0.5
    intensity: float = 1.0
    rotation_y: float = 0.0  # CCW rotation of the dome about +y, radians (HdriEnvironment.rotationY)


@dataclass
class Scene:
    meshes: List[Mesh] = field(default_factory=list)
    materials: List[Material] = field(default_factory=list)
    instances: List[Instance] = field(default_factory=list)
    point_lights: List[PointLight] = field(default_factory=list)
    environment: Optional[Environment] = None
    directional_lights: List[DirectionalLight] = field(default_factory=list)
    rect_lights: List[RectLight] = field(default_factory=list)
    spot_lights: List[SpotLight] = field(default_factory=list)
    disc_lights: List[DiscLight] = field(default_factory=list)

    @property
    def triangle_count(self) -> int:
        """Distinct triangles (prototype meshes count once however often they are placed)."""
        return int(sum(m.indices.shape[0] for m in self.meshes))

    @property
    def instanced_triangle_count(self) -> int:
        if not self.instances:
            return self.triangle_count
        return int(sum(self.meshes[i.mesh].indices.shape[0] for i in self.instances))

    def flattened(self) -> "Scene":
        """The same scene with every instance baked into a world-space mesh (a
        mirroring placement reverses the winding, so front faces stay front
        faces, as the two-level traversal's transformed normals keep them)."""
        if not self.instances:
            return self
        out = []
        for inst in self.instances:
            m = self.meshes[inst.mesh]
            M = np.asarray(inst.local_to_world, np.float64).reshape(4, 4)
            p = np.asarray(m.positions, np.float64).reshape(-1, 3) @ M[:3, :3].T + M[:3, 3]
            t = np.asarray(m.indices, np.uint32).reshape(-1, 3)
            if np.linalg.det(M[:3, :3]) < 0:
                t = t[:, [0, 2, 1]]
            out.append(Mesh(p.astype(np.float32), np.ascontiguousarray(t), inst.material))
        return dataclasses.replace(self, meshes=out, instances=[])


@dataclass
class Camera:
    eye: Sequence[float]
    target: Sequence[float]
    up: Sequence[float] = (0.0, 1.0, 0.0)
    fov_y_deg: float = 40.0
    near: float = 0.01
    far: float = 1000.0

    def matrices(self, aspect: float):
        """(view, projection) column-major float32[16], OpenGL conventions."""
        e = np.asarray(self.eye, np.float64)
        t = np.asarray(self.target, np.float64)
        u = np.asarray(self.up, np.float64)
        f = t - e
        f /= np.linalg.norm(f)
        s = np.cross(f, u)
        s /= np.linalg.norm(s)
        uu = np.cross(s, f)
        view = np.eye(4)
        view[0, :3], view[1, :3], view[2, :3] = s, uu, -f
        view[0, 3], view[1, 3], view[2, 3] = -s @ e, -uu @ e, f @ e
        k = 1.0 / math.tan(math.radians(self.fov_y_deg) / 2)
        n, fa = self.near, self.far
        proj = np.zeros((4, 4))
        proj[0, 0] = k / aspect
        proj[1, 1] = k
        proj[2, 2] = (fa + n) / (n - fa)
        proj[2, 3] = 2 * fa * n / (n - fa)
        proj[3, 2] = -1.0
        return view.T.reshape(-1).astype(np.float32), proj.T.reshape(-1).astype(np.float32)


def _marshal_scene(scene: "Scene"):
    """(vt_scene_desc, list of arrays that must outlive the call)."""
    keep = []
    meshes = (_MeshDesc * max(1, len(scene.meshes)))()
    for i, m in enumerate(scene.meshes):
        p = np.ascontiguousarray(m.positions, np.float32).reshape(-1, 3)
        ix = np.ascontiguousarray(m.indices, np.uint32).reshape(-1, 3)
        keep += [p, ix]
        meshes[i] = _MeshDesc(p.ctypes.data, p.shape[0], ix.ctypes.data, ix.shape[0], int(m.material))
    mats = (_MaterialDesc * max(1, len(scene.materials)))()
    for i, m in enumerate(scene.materials):
        mats[i] = _MaterialDesc((ctypes.c_float * 3)(*m.base_color), m.roughness, m.metallic, m.transmission,
                                m.ior, (ctypes.c_float * 3)(*m.emission), m.flags, m.specular_intensity)
    pls = (_PointLightDesc * max(1, len(scene.point_lights)))()
    for i, l in enumerate(scene.point_lights):
        pls[i] = _PointLightDesc((ctypes.c_float * 3)(*l.position), (ctypes.c_float * 3)(*l.intensity))
    env_ptr, ew, eh, ei = None, 0, 0, 1.0
    if scene.environment is not None:
        env = np.ascontiguousarray(scene.environment.rgb, np.float32)
        keep.append(env)
        env_ptr, eh, ew, ei = env.ctypes.data, env.shape[0], env.shape[1], scene.environment.intensity
    insts = (_InstanceDesc * max(1, len(scene.instances)))()
    for i, inst in enumerate(scene.instances):
        M = np.asarray(inst.local_to_world, np.float32).reshape(4, 4)
        insts[i] = _InstanceDesc(int(inst.mesh), int(inst.material), (ctypes.c_float * 16)(*M.T.reshape(-1)))
    dls = (_DirectionalDesc * max(1, len(scene.directional_lights)))()
    for i, l in enumerate(scene.directional_lights):
        dls[i] = _DirectionalDesc((ctypes.c_float * 3)(*l.direction), (ctypes.c_float * 3)(*l.irradiance),
                                  l.angular_radius)
    rls = (_RectDesc * max(1, len(scene.rect_lights)))()
    for i, r in enumerate(scene.rect_lights):
        rls[i] = _RectDesc((ctypes.c_float * 3)(*r.corner), (ctypes.c_float * 3)(*r.edge_u),
                           (ctypes.c_float * 3)(*r.edge_v), (ctypes.c_float * 3)(*r.radiance))
    sls = (_SpotDesc * max(1, len(scene.spot_lights)))()
    for i, l in enumerate(scene.spot_lights):
        sls[i] = _SpotDesc((ctypes.c_float * 3)(*l.position), (ctypes.c_float * 3)(*l.direction),
                           (ctypes.c_float * 3)(*l.intensity), l.angle, l.penumbra, l.distance, l.decay)
    dcs = (_DiscDesc * max(1, len(scene.disc_lights)))()
    for i, l in enumerate(scene.disc_lights):
        dcs[i] = _DiscDesc((ctypes.c_float * 3)(*l.center), (ctypes.c_float * 3)(*l.normal), l.radius,
                           (ctypes.c_float * 3)(*l.radiance))
    desc = _SceneDesc(ctypes.cast(meshes, ctypes.c_void_p), len(scene.meshes),
                      ctypes.cast(insts, ctypes.c_void_p) if scene.instances else None, len(scene.instances),
                      ctypes.cast(mats, ctypes.c_void_p),
                      len(scene.materials), ctypes.cast(pls, ctypes.c_void_p), len(scene.point_lights), env_ptr,
                      ew, eh, ei, ctypes.cast(dls, ctypes.c_void_p), len(scene.directional_lights),
                      ctypes.cast(rls, ctypes.c_void_p), len(scene.rect_lights),
                      ctypes.cast(sls, ctypes.c_void_p), len(scene.spot_lights),
                      ctypes.cast(dcs, ctypes.c_void_p), len(scene.disc_lights),
                      0.0 if scene.environment is None else float(scene.environment.rotation_y))
    return desc, (keep, meshes, insts, mats, pls, dls, rls, sls, dcs)


# ---------------------------------------------------------------- engine
def debug_fail_device_allocation(nth: int) -> None:
    """Failure-injection hook (vt_debug_fail_device_allocation): the nth device
    allocation the library makes on this thread from now on fails as an
    out-of-memory cudaMalloc would; 0 disarms."""
    N.call("vt_debug_fail_device_allocation", int(nth))


class _Debug:
    def __init__(self, engine: "Engine"):
        self._e = engine

    def set_wait_limit(self, cycles: int) -> None:
        """Failure-detection hook (vt_engine_set_wait_limit): bound the first
        wait of the cache kernels' and the staging copy's bounded waits to
        `cycles` clocks (0: the default of about a second)."""
        N.call("vt_engine_set_wait_limit", self._e.handle, int(cycles))

    def pick_triangle(self, x: float, y: float) -> Optional[int]:
        """vt_pick as it is: under pixel (x, y) of the last frame's camera, the
        source triangle index (single-level scene) or the instance index (scene
        with instances); None on a miss."""
        out = ctypes.c_int32(-1)
        N.call("vt_pick", self._e.handle, float(x), float(y), ctypes.byref(out))
        return None if out.value < 0 else int(out.value)

    def pick_primitive(self, x: float, y: float) -> Optional[int]:
        """Engine.debug.pickPrimitive (engine/debug.ts:33-35, pickPrimitiveCpu.ts:674):
        the scene primitive under pixel (x, y) -- the index of the mesh hit (the
        placed mesh for an instance) -- or None on a miss."""
        hit = self.pick_triangle(x, y)
        sc = self._e._scene
        if hit is None or sc is None:
            return None
        if sc.instances:
            return int(sc.instances[hit].mesh)
        ends = np.cumsum([m.indices.shape[0] for m in sc.meshes])
        return int(np.searchsorted(ends, hit, side="right"))


class Engine:
    """createPTEngine (pt-webgpu factory, index.ts:2363) on the CUDA backend."""

    def __init__(self, device: int = 0, max_bounces: int = 8, max_samples_per_pixel: int = 4096,
                 debug: bool = False, oracle_accumulation: bool = False, sort_by_material: bool = False,
                 wave_paths: int = 0, bvh_max_leaf: int = 0, light_selection: str = "tree",
                 scene_build: str = "gpu", bvh_width: int = 0):
        opts = _EngineOptions(max_bounces, max_samples_per_pixel, 1 if debug else 0, 1 if oracle_accumulation else 0,
                              1 if sort_by_material else 0, wave_paths, bvh_max_leaf,
                              {"tree": 0, "uniform": 1}[light_selection], {"gpu": 0, "host": 1}[scene_build],
                              bvh_width)
        h = ctypes.c_void_p()
        N.call("vt_create", device, ctypes.byref(opts), ctypes.byref(h))
        self._h = h
        self.device = device
        self.debug = _Debug(self) if debug else None
        self._scene = None
        self._keep = []
        self.width = self.height = 0

    @property
    def handle(self):
        if not self._h:
            raise RuntimeError("engine is disposed")
        return self._h

    def set_scene(self, scene: Scene) -> None:
        desc, keep = _marshal_scene(scene)
        N.call("vt_set_scene", self.handle, ctypes.byref(desc))
        self._scene = scene

    EMITTER_KINDS = {1: "point", 2: "spot", 4: "directional", 8: "rect-area", 16: "disc-area", 32: "mesh-area",
                     64: "environment"}
    FEATURES = {1: "instances", 2: "instance-updates", 4: "radiance-cache", 8: "batch", 16: "pick",
                32: "output-capture", 64: "fp64-moments", 128: "aux-outputs", 256: "mesh-updates"}

    @property
    def capabilities(self) -> dict:
        """Engine.capabilities (vt_get_capabilities): limits, emitter kinds, features."""
        c = _Capabilities()
        N.call("vt_get_capabilities", self.handle, ctypes.byref(c))
        return {"maxBouncesLimit": c.max_bounces_limit, "maxSamplesPerPixel": c.max_samples_per_pixel,
                "maxViewport": c.max_viewport,
                "emitterKinds": sorted(v for k, v in self.EMITTER_KINDS.items() if c.emitter_kinds & k),
                "features": sorted(v for k, v in self.FEATURES.items() if c.features & k),
                "materialFeatures": c.material_features}

    def update_instances(self, instances: Sequence[Instance], rebuild: bool = False) -> None:
        """New placements (mesh, material, transform) for the current scene's
        instances, same count (vt_update_instances): the top level is refitted
        (refitTlasTransforms) or, with rebuild, rebuilt over the new bounds
        (rebuildTlasReuseBlas); bottom levels are kept.  Clears the accumulation."""
        arr = (_InstanceDesc * max(1, len(instances)))()
        for i, inst in enumerate(instances):
            M = np.asarray(inst.local_to_world, np.float32).reshape(4, 4)
            arr[i] = _InstanceDesc(int(inst.mesh), int(inst.material), (ctypes.c_float * 16)(*M.T.reshape(-1)))
        N.call("vt_update_instances", self.handle, ctypes.cast(arr, ctypes.c_void_p), len(instances),
               1 if rebuild else 0)
        if self._scene is not None:
            self._scene = dataclasses.replace(self._scene, instances=list(instances))

    def update_mesh(self, index: int, mesh: "Mesh", rebuild: bool = False) -> None:
        """New geometry and material for mesh `index` of a scene with instances
        (vt_update_mesh, the reference's rebuildPrimitiveBlas): its bottom level
        is rebuilt and spliced in, the top level refitted (or rebuilt).  Clears
        the accumulation."""
        p = np.ascontiguousarray(mesh.positions, np.float32).reshape(-1, 3)
        ix = np.ascontiguousarray(mesh.indices, np.uint32).reshape(-1, 3)
        d = _MeshDesc(p.ctypes.data, p.shape[0], ix.ctypes.data, ix.shape[0], int(mesh.material))
        N.call("vt_update_mesh", self.handle, int(index), ctypes.byref(d), 1 if rebuild else 0)
        if self._scene is not None:
            meshes = list(self._scene.meshes)
            meshes[index] = mesh
            self._scene = dataclasses.replace(self._scene, meshes=meshes)

    def set_previous_camera(self, camera: "Camera | None", aspect: "float | None" = None) -> None:
        """FrameInput.prevViewMatrix / prevProjMatrix for the next frame's motion
        output (that frame only), the camera at `aspect` (width / height); None clears."""
        if camera is None:
            N.call("vt_set_previous_camera", self.handle, None, None)
            return
        if not aspect or aspect <= 0:
            raise ValueError("aspect (width / height) must be positive")
        view, proj = camera.matrices(aspect)
        N.call("vt_set_previous_camera", self.handle, (ctypes.c_float * 16)(*view), (ctypes.c_float * 16)(*proj))

    def render_frame(self, camera: Camera, width: int, height: int, samples: int = 1, bounces: int = 0,
                     frame_seed: int = 0, prev_camera: "Camera | None" = None) -> dict:
        if prev_camera is not None:
            self.set_previous_camera(prev_camera, width / height)
        view, proj = camera.matrices(width / height)
        fin = _FrameInput((ctypes.c_float * 16)(*view), (ctypes.c_float * 16)(*proj), width, height, frame_seed,
                          samples, bounces)
        out = _FrameOutput()
        N.call("vt_render_frame", self.handle, ctypes.byref(fin), ctypes.byref(out))
        self.width, self.height = out.width, out.height
        return {"kind": "rendered" if out.kind == 0 else "skipped", "samplesAccumulated": out.samples_accumulated,
                "isConverged": bool(out.is_converged),
                "primaryRadiance": {"devicePtr": out.radiance_device, "width": out.width, "height": out.height,
                                    "format": "rgba32f-sum-count"}}

    def profile_frame(self, camera: Camera, width: int, height: int, samples: int = 1, bounces: int = 0,
                      frame_seed: int = 0) -> dict:
        """render_frame with per-stage device timings (no graph replay)."""
        view, proj = camera.matrices(width / height)
        fin = _FrameInput((ctypes.c_float * 16)(*view), (ctypes.c_float * 16)(*proj), width, height, frame_seed,
                          samples, bounces)
        out = _FrameOutput()
        tm = _StageTimes()
        N.call("vt_profile_frame", self.handle, ctypes.byref(fin), ctypes.byref(out), ctypes.byref(tm))
        self.width, self.height = out.width, out.height
        return {f: getattr(tm, f) for f, _ in _StageTimes._fields_}

    TONEMAPS = {"aces": 0, "agx": 1, "reinhard": 2, "linear": 3, "none": 4}

    def capture_frame(self, color_space: str = "linear", tonemap: str = "aces", exposure: float = 1.0,
                      output_color_space: str = "srgb", out: "np.ndarray | None" = None) -> np.ndarray:
        """(H, W, 4) float32, alpha 1 (Engine.captureFrame).  color_space 'linear':
        the mean radiance; 'output': the present pass (exposure, `tonemap` of
        aces / agx / reinhard / linear / none, sRGB encoding unless
        output_color_space is 'linear').  out: an (H, W, 4) float32 C-contiguous
        array to fill (page-locked memory makes the copy a direct DMA)."""
        if out is None:
            out = np.empty((self.height, self.width, 4), np.float32)
        elif out.shape != (self.height, self.width, 4) or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous (height, width, 4) float32 array")
        if color_space == "linear":
            N.call("vt_capture", self.handle, ctypes.c_void_p(out.ctypes.data), out.size)
        elif color_space == "output":
            if tonemap not in self.TONEMAPS or output_color_space not in ("srgb", "linear"):
                raise ValueError("tonemap must be one of %s and output_color_space srgb or linear"
                                 % sorted(self.TONEMAPS))
            o = _PresentOptions(self.TONEMAPS[tonemap], exposure, 1 if output_color_space == "srgb" else 0)
            N.call("vt_capture_output", self.handle, ctypes.byref(o), ctypes.c_void_p(out.ctypes.data), out.size)
        else:
            raise ValueError("color_space must be 'linear' or 'output'")
        return out

    def capture_moments(self):
        """FP64 per-pixel mean and per-sample variance, each (H, W, 3)."""
        m = np.empty((self.height, self.width, 3), np.float64)
        v = np.empty_like(m)
        N.call("vt_capture_moments", self.handle, ctypes.c_void_p(m.ctypes.data), ctypes.c_void_p(v.ctypes.data),
               m.size)
        return m, v

    def export_scene(self):
        """The device node words (uint32, 20 per wide node) and triangle records
        (float32, 16 per record) of the current scene (vt_engine_export_scene)."""
        nw, nf = ctypes.c_size_t(), ctypes.c_size_t()
        N.call("vt_engine_export_scene", self.handle, None, 0, None, 0, ctypes.byref(nw), ctypes.byref(nf))
        words = np.empty(nw.value, np.uint32)
        recs = np.empty(nf.value, np.float32)
        N.call("vt_engine_export_scene", self.handle, ctypes.c_void_p(words.ctypes.data), words.size,
               ctypes.c_void_p(recs.ctypes.data), recs.size, ctypes.byref(nw), ctypes.byref(nf))
        return words, recs

    def capture_luminance_moments(self):
        """Per-pixel FP64 shape of the luminance samples, (H, W, 4): mean,
        per-sample variance, skewness, excess kurtosis (oracle_accumulation)."""
        out = np.empty((self.height, self.width, 4), np.float64)
        N.call("vt_capture_luminance_moments", self.handle, ctypes.c_void_p(out.ctypes.data), out.size)
        return out

    AUX = {"normal_depth": 0, "albedo": 1, "motion": 2, "variance": 3}

    def capture_aux(self, kind: str) -> np.ndarray:
        """Auxiliary output (H, W, 4) float32: 'normal_depth' (n * 0.5 + 0.5,
        distance), 'albedo', 'motion' (pixels) of the first hit of the latest
        frame's last sample, or 'variance' (luminance variance in channel 0)."""
        if kind not in self.AUX:
            raise ValueError("kind must be one of %s" % sorted(self.AUX))
        out = np.empty((self.height, self.width, 4), np.float32)
        N.call("vt_capture_aux", self.handle, self.AUX[kind], ctypes.c_void_p(out.ctypes.data), out.size)
        return out

    def trace_rays(self, rays: np.ndarray):
        """Closest hits of (n, 8) float32 rays [ox oy oz tmin dx dy dz tmax] against the scene.

        Returns (hits, instances): a HIT_DTYPE array (prim, t, u, v) and an
        int32 array of instance indices (-1 on a miss or without instances)."""
        from .bvh import HIT_DTYPE
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        hits = np.empty(r.shape[0], HIT_DTYPE)
        inst = np.empty(r.shape[0], np.int32)
        N.call("vt_trace_rays", self.handle, ctypes.c_void_p(r.ctypes.data), r.shape[0],
               ctypes.c_void_p(hits.ctypes.data), ctypes.c_void_p(inst.ctypes.data))
        return hits, inst

    def set_nrc(self, enabled: bool = True, prefix_bounces: int = 1, train_steps: int = 4, train_batch: int = 65536,
                train_paths: int = 0, warmup_frames: int = 0, cache=None, fallback_error: float = 0.0,
                fallback_tile: int = 16, spread_c: float = 0.0) -> None:
        """Path tracing with the neural radiance cache (vt_set_nrc): each frame
        trains the cache on its own training paths, then ends the render paths
        in a cache query after `prefix_bounces` bounces (0: at the first vertex
        whose path spread exceeds spread_c * a0, default c 0.01).  fallback_error > 0:
        screen tiles whose cache error estimate exceeds it keep path tracing."""
        from .nrc import NrcConfig
        cfg = (cache or NrcConfig()).to_c()
        o = _NrcRenderOptions(1 if enabled else 0, prefix_bounces, train_steps, train_batch, train_paths,
                              warmup_frames, cfg, fallback_error, fallback_tile, spread_c)
        N.call("vt_set_nrc", self.handle, ctypes.byref(o))

    def autotune(self, camera: Camera, width: int, height: int, samples: int = 1, bounces: int = 0,
                 frame_seed: int = 0):
        """The project's autotuner (vt_engine_autotune): times candidate launch
        shapes (wave size, material sort, traversal CTAs per SM) on this frame
        and keeps the fastest.  Returns the trials [(tuning dict, ms)]."""
        from .batch import _Trial, _Tuning
        view, proj = camera.matrices(width / height)
        fin = _FrameInput((ctypes.c_float * 16)(*view), (ctypes.c_float * 16)(*proj), width, height, frame_seed,
                          samples, bounces)
        trials = (_Trial * 32)()
        n = ctypes.c_size_t()
        N.call("vt_engine_autotune", self.handle, ctypes.byref(fin), ctypes.cast(trials, ctypes.c_void_p), 32,
               ctypes.byref(n))
        self.width, self.height = width, height
        return [dict({f: getattr(trials[i].tuning, f) for f, _ in _Tuning._fields_}, frame_ms=trials[i].frame_ms)
                for i in range(min(n.value, 32))]

    def autotune_bvh(self, scene: Scene, camera: Camera, width: int, height: int, samples: int = 1,
                     bounces: int = 0, frame_seed: int = 0):
        """The BVH-shape autotuner (vt_engine_autotune_bvh): rebuilds `scene` with
        candidate leaf sizes and collapse widths, times this frame with each and
        keeps the fastest (the scene stays set).  Returns the trials."""
        desc, keep = _marshal_scene(scene)
        view, proj = camera.matrices(width / height)
        fin = _FrameInput((ctypes.c_float * 16)(*view), (ctypes.c_float * 16)(*proj), width, height, frame_seed,
                          samples, bounces)
        trials = (_BvhShapeTrial * 16)()
        n = ctypes.c_size_t()
        N.call("vt_engine_autotune_bvh", self.handle, ctypes.byref(desc), ctypes.byref(fin),
               ctypes.cast(trials, ctypes.c_void_p), 16, ctypes.byref(n))
        self._scene = scene
        self.width, self.height = width, height
        return [{f: getattr(trials[i], f) for f, _ in _BvhShapeTrial._fields_} for i in range(min(n.value, 16))]

    @property
    def tuning(self) -> dict:
        from .batch import _Tuning
        t = _Tuning()
        N.call("vt_engine_get_tuning", self.handle, ctypes.byref(t))
        return {f: getattr(t, f) for f, _ in _Tuning._fields_}

    def set_tuning(self, wave_paths: int = 1 << 24, sort_by_material: bool = False, trace_blocks_per_sm: int = 0,
                   stage_hot_nodes: bool = False, sort_rays: int = 0, nrc_infer_tiles: int = 0) -> None:
        """Launch shape for later frames (vt_engine_set_tuning); `tuning` of
        another engine or an autotune trial can be passed back as keywords.
        sort_rays: 0 queue order, 1 direction octant, 2 origin cell and octant
        (True / False read as 1 / 0).  nrc_infer_tiles: query tiles per inference
        CTA of the radiance cache (1..4; 0 leaves it)."""
        from .batch import _Tuning
        t = _Tuning(int(wave_paths), 1 if sort_by_material else 0, int(trace_blocks_per_sm),
                    1 if stage_hot_nodes else 0, int(sort_rays), int(nrc_infer_tiles))
        N.call("vt_engine_set_tuning", self.handle, ctypes.byref(t))

    def export_tlas(self):
        """The scene's top-level tree in the reference layout (tlasNodes,
        tlasInstanceIndices of packSceneFromCore, scenePack.ts:1104-1310)."""
        count = ctypes.c_size_t(0)
        N.call("vt_engine_export_tlas", self.handle, None, 0, None, 0, ctypes.byref(count))
        nodes = np.zeros((count.value, 8), np.uint32)
        perm = np.zeros(max(count.value, 1), np.uint32)
        N.call("vt_engine_export_tlas", self.handle, ctypes.c_void_p(nodes.ctypes.data), nodes.size,
               ctypes.c_void_p(perm.ctypes.data), perm.size, ctypes.byref(count))
        leaf = (nodes[:, 7] >> 16) == 0xFFFF
        n_inst = int((nodes[leaf, 7] & 0xFFFF).sum())
        return nodes, perm[:n_inst].copy()

    def stats(self) -> dict:
        s = _EngineStats()
        N.call("vt_engine_get_stats", self.handle, ctypes.byref(s))
        return {f: getattr(s, f) for f, _ in _EngineStats._fields_}

    def reset(self) -> None:
        N.call("vt_reset", self.handle)

    def dispose(self) -> None:
        if self._h:
            N.call("vt_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass


def create_engine(**options) -> Engine:
    """createPTEngine_CUDA(options) -> Engine (options: max_bounces, max_samples_per_pixel, debug, ...)."""
    return Engine(**options)
