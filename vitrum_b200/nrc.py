"""Neural radiance cache on the B200 (vt_nrc_* in libvitrum_pt.so).

Mirrors the reference NRC subsystem (packages/walkaround-hybrid/src/neural/nrc/
nrcSubsystem.ts): a multiresolution hash-grid encoding of the query position
plus direction and surface features, a fully fused 64-wide MLP (5 hidden ReLU
layers, 3 linear outputs) with fp16 weights/activations and fp32 accumulation
on the tcgen05 tensor cores, relative-L2 luminance loss, Adam.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import _native as N

RECORD_FLOATS = 16
SAMPLE_FLOATS = 20
WEIGHT_COUNT = 6 * 64 * 64


class _Config(ctypes.Structure):
    _fields_ = [("levels", ctypes.c_int32), ("log2_table_size", ctypes.c_int32),
                ("base_resolution", ctypes.c_float), ("growth", ctypes.c_float),
                ("learning_rate", ctypes.c_float), ("table_learning_rate", ctypes.c_float),
                ("aabb_min", ctypes.c_float * 3), ("aabb_max", ctypes.c_float * 3), ("seed", ctypes.c_uint32),
                ("infer_tiles", ctypes.c_int32)]


@dataclass
class NrcConfig:
    """Hash grid 16 levels x 2^19 entries x 2 fp16 features, base resolution 16,
    growth 1.5; Adam lr 1e-2 (MLP and table)."""
    levels: int = 16
    log2_table_size: int = 19
    base_resolution: float = 16.0
    growth: float = 1.5
    learning_rate: float = 1e-2
    table_learning_rate: float = 1e-2
    aabb_min: Sequence[float] = (0.0, 0.0, 0.0)
    aabb_max: Sequence[float] = (1.0, 1.0, 1.0)
    seed: int = 1
    infer_tiles: int = 0  # query tiles of 128 in flight per inference CTA (1..4; 0: the default)

    def to_c(self) -> _Config:
        return _Config(self.levels, self.log2_table_size, self.base_resolution, self.growth, self.learning_rate,
                       self.table_learning_rate, (ctypes.c_float * 3)(*self.aabb_min),
                       (ctypes.c_float * 3)(*self.aabb_max), self.seed, self.infer_tiles)

    @property
    def table_floats(self) -> int:
        return self.levels * (1 << self.log2_table_size) * 2


def _p(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


class RadianceCache:
    """One cache on one GPU: query, train_step, gradients, parameter snapshots."""

    def __init__(self, config: NrcConfig = NrcConfig(), device: int = 0):
        self.config = config
        h = ctypes.c_void_p()
        N.call("vt_nrc_create", device, ctypes.byref(config.to_c()), ctypes.byref(h))
        self._h = h

    @property
    def handle(self):
        if not self._h:
            raise RuntimeError("cache is disposed")
        return self._h

    def close(self):
        if self._h:
            N.call("vt_nrc_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def query(self, records: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(records, np.float32).reshape(-1, RECORD_FLOATS)
        out = np.empty((r.shape[0], 3), np.float32)
        N.call("vt_nrc_query", self.handle, _p(r), r.shape[0], _p(out))
        return out

    def query_device(self, records_ptr: int, n: int, rgb_ptr: int, stream: int = 0) -> None:
        """Enqueue a query on device arrays (16 floats per record in, 3 floats out)."""
        N.call("vt_nrc_query_device", self.handle, ctypes.c_void_p(records_ptr), n, ctypes.c_void_p(rgb_ptr),
               ctypes.c_void_p(stream))

    def train_step_device(self, samples_ptr: int, n: int, stream: int = 0) -> None:
        """Enqueue one optimiser step on a device array of n samples (20 floats each)."""
        N.call("vt_nrc_train_device", self.handle, ctypes.c_void_p(samples_ptr), n, ctypes.c_void_p(stream))

    def train_step(self, samples: np.ndarray) -> float:
        s = np.ascontiguousarray(samples, np.float32).reshape(-1, SAMPLE_FLOATS)
        loss = ctypes.c_float()
        N.call("vt_nrc_train", self.handle, _p(s), s.shape[0], ctypes.byref(loss))
        return float(loss.value)

    def gradients(self, samples: np.ndarray):
        """(dW (6, 64, 64), d_table (levels, T, 2), mean loss) without an update."""
        s = np.ascontiguousarray(samples, np.float32).reshape(-1, SAMPLE_FLOATS)
        gw = np.empty(WEIGHT_COUNT, np.float32)
        gt = np.empty(self.config.table_floats, np.float32)
        loss = ctypes.c_float()
        N.call("vt_nrc_gradients", self.handle, _p(s), s.shape[0], _p(gw), _p(gt), ctypes.byref(loss))
        return gw.reshape(6, 64, 64), gt.reshape(self.config.levels, -1, 2), float(loss.value)

    def get_params(self):
        w = np.empty(WEIGHT_COUNT, np.float32)
        t = np.empty(self.config.table_floats, np.float32)
        N.call("vt_nrc_get_params", self.handle, _p(w), _p(t))
        return w.reshape(6, 64, 64), t.reshape(self.config.levels, -1, 2)

    def set_params(self, weights=None, table=None):
        w = None if weights is None else np.ascontiguousarray(weights, np.float32).reshape(-1)
        t = None if table is None else np.ascontiguousarray(table, np.float32).reshape(-1)
        N.call("vt_nrc_set_params", self.handle, _p(w) if w is not None else None,
               _p(t) if t is not None else None)
