"""Many scenes rendered together on one GPU (vt_batch_* in libvitrum_pt.so).

Every scene contributes one frame (its own resolution, samples and bounce
count); the paths of all frames share each wave, traversal takes a per-ray
root in the concatenated BVH arena, and the whole batch frame is one CUDA
graph.  The launch shape (wave size, material sort, traversal CTAs per SM)
comes from the project's autotuner (vt_batch_autotune) or is set directly.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

from . import _native as N
from .engine import Camera, Scene, _EngineOptions, _FrameInput, _marshal_scene


class _BatchStats(ctypes.Structure):
    _fields_ = [("frame_ms", ctypes.c_double), ("closest_rays", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64),
                ("waves", ctypes.c_int32), ("kernel_launches", ctypes.c_int32)]


class _Tuning(ctypes.Structure):
    _fields_ = [("wave_paths", ctypes.c_int32), ("sort_by_material", ctypes.c_int32),
                ("trace_blocks_per_sm", ctypes.c_int32), ("stage_hot_nodes", ctypes.c_int32),
                ("sort_rays", ctypes.c_int32), ("nrc_infer_tiles", ctypes.c_int32)]


class _Trial(ctypes.Structure):
    _fields_ = [("tuning", _Tuning), ("frame_ms", ctypes.c_double)]


@dataclass
class BatchItem:
    scene: Scene
    camera: Camera
    width: int
    height: int
    samples: int
    bounces: int = 0
    frame_seed: int = 0


class Batch:
    def __init__(self, items: Sequence[BatchItem], device: int = 0, max_bounces: int = 8):
        opts = _EngineOptions(max_bounces, 1 << 20, 0, 0, 0, 0, 0)
        h = ctypes.c_void_p()
        N.call("vt_batch_create", device, ctypes.byref(opts), ctypes.byref(h))
        self._h = h
        self.items = list(items)
        keep = []
        from .engine import _SceneDesc
        arr = (_SceneDesc * len(self.items))()
        frames = (_FrameInput * len(self.items))()
        for i, it in enumerate(self.items):
            d, k = _marshal_scene(it.scene)
            keep.append(k)
            arr[i] = d
            view, proj = it.camera.matrices(it.width / it.height)
            frames[i] = _FrameInput((ctypes.c_float * 16)(*view), (ctypes.c_float * 16)(*proj), it.width, it.height,
                                    it.frame_seed, it.samples, it.bounces)
        N.call("vt_batch_set_scenes", self._h, ctypes.cast(arr, ctypes.c_void_p), ctypes.cast(frames, ctypes.c_void_p),
               len(self.items))

    @property
    def handle(self):
        if not self._h:
            raise RuntimeError("batch is disposed")
        return self._h

    def render(self) -> dict:
        st = _BatchStats()
        N.call("vt_batch_render", self.handle, ctypes.byref(st))
        return {f: getattr(st, f) for f, _ in _BatchStats._fields_}

    def capture(self, index: int) -> np.ndarray:
        it = self.items[index]
        out = np.empty((it.height, it.width, 4), np.float32)
        N.call("vt_batch_capture", self.handle, index, ctypes.c_void_p(out.ctypes.data), out.size)
        return out

    @property
    def tuning(self) -> dict:
        t = _Tuning()
        N.call("vt_batch_get_tuning", self.handle, ctypes.byref(t))
        return {f: getattr(t, f) for f, _ in _Tuning._fields_}

    def set_tuning(self, wave_paths: int, sort_by_material: bool = False, trace_blocks_per_sm: int = 0,
                   stage_hot_nodes: bool = False, sort_rays: bool = False) -> None:
        t = _Tuning(wave_paths, 1 if sort_by_material else 0, trace_blocks_per_sm, 1 if stage_hot_nodes else 0,
                    1 if sort_rays else 0, 0)
        N.call("vt_batch_set_tuning", self.handle, ctypes.byref(t))

    def autotune(self) -> List[dict]:
        """Times the candidate launch shapes (one render each after a warm-up) and keeps the fastest."""
        trials = (_Trial * 32)()
        n = ctypes.c_size_t()
        N.call("vt_batch_autotune", self.handle, ctypes.cast(trials, ctypes.c_void_p), 32, ctypes.byref(n))
        return [dict({f: getattr(trials[i].tuning, f) for f, _ in _Tuning._fields_}, frame_ms=trials[i].frame_ms)
                for i in range(min(n.value, 32))]

    def close(self):
        if self._h:
            N.call("vt_batch_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
