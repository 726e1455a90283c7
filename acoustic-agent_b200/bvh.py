"""BVH of the reference (``acoustic_agent/bvh.py:8-77``, ``build_bvh``) built on the GPU.

The reference builds it in Python once per geometry (``steam_rt.py:881``,
inside ``_scene_kernel_arrays``): a top-down median split with stable argsorts,
emitted in preorder with escape links.  ``ac_bvh_build_device`` builds the same
tree, array for array, from device-resident surface bounds; it is meant for
scenes of thousands to millions of surfaces, where the reference's recursion
takes seconds to minutes.

``build_bvh`` is the drop-in (numpy in, numpy out, the reference's dict and
error messages); ``DeviceBvhBuilder.build`` keeps everything on the device.
There is no CPU fallback: without a CUDA device both raise.
"""
from __future__ import annotations

import ctypes
import threading
from dataclasses import dataclass
from typing import Any

import numpy as np
import torch

from acoustic_agent_b200 import _lib, runtime


@dataclass
class DeviceBvh:
    """The arrays of build_bvh (bvh.py:66-77) as device tensors."""

    bounds_min: torch.Tensor   # [nodes, 3] float64
    bounds_max: torch.Tensor   # [nodes, 3] float64
    start: torch.Tensor        # [nodes] int64, -1 for inner nodes
    count: torch.Tensor        # [nodes] int64, 0 for inner nodes
    escape: torch.Tensor       # [nodes] int64
    primitives: torch.Tensor   # [surfaces] int64
    node_count: int
    leaf_count: int
    max_depth: int
    leaf_size: int
    inputs: tuple = ()         # the bounds the build reads, kept alive until it has run

    def to_numpy(self) -> dict[str, Any]:
        return {
            "bounds_min": self.bounds_min.cpu().numpy(), "bounds_max": self.bounds_max.cpu().numpy(),
            "start": self.start.cpu().numpy(), "count": self.count.cpu().numpy(),
            "escape": self.escape.cpu().numpy(), "primitives": self.primitives.cpu().numpy(),
            "node_count": self.node_count, "leaf_count": self.leaf_count, "max_depth": self.max_depth,
            "leaf_size": self.leaf_size,
        }


def _check_shapes(lower_shape, upper_shape) -> int:
    """bvh.py:17-20: the reference's shape checks and messages."""
    if tuple(lower_shape) != tuple(upper_shape) or len(lower_shape) != 2 or lower_shape[1] != 3:
        raise ValueError("BVH bounds must have shape [surface, 3]")
    if lower_shape[0] < 1:
        raise ValueError("BVH requires at least one surface")
    return int(lower_shape[0])


def _raise_status(status: int) -> None:
    """bvh.py:21-24 for the device-side value checks; the other bits are build failures."""
    if status & _lib.AC_BVH_STATUS_NONFINITE:
        raise ValueError("BVH bounds must be finite")
    if status & _lib.AC_BVH_STATUS_ORDER:
        raise ValueError("BVH maximum bounds must not be below minimum bounds")
    if status:
        raise RuntimeError(f"ac_bvh_build_device failed on the device (status {status})")


class DeviceBvhBuilder:
    """Workspace, pinned plan staging and status word of ac_bvh_build_device, reused across builds.

    Builds through one builder are serialised: a build waits until the previous one has finished on the device
    before it reuses the workspace, and the status word describes the latest build only."""

    def __init__(self, device: torch.device | int = 0) -> None:
        self.device = runtime.require_cuda(device.index if isinstance(device, torch.device) else int(device))
        self.workspace: torch.Tensor | None = None
        self.staging: torch.Tensor | None = None
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._copied: torch.cuda.Event | None = None
        self._lock = threading.Lock()

    def _buffers(self, ws_bytes: int, staging_bytes: int) -> None:
        if self._copied is not None:
            self._copied.synchronize()   # the previous build's plan copy has left the staging
            self._copied = None
        if self.workspace is None or self.workspace.numel() < ws_bytes:
            self.workspace = torch.empty(max(ws_bytes, 1 << 16), dtype=torch.uint8, device=self.device)
        if self.staging is None or self.staging.numel() < staging_bytes:
            self.staging = torch.empty(max(staging_bytes, 1 << 12), dtype=torch.uint8, pin_memory=True)

    def build(self, lower: torch.Tensor, upper: torch.Tensor, *, leaf_size: int = 4,
              stream: torch.cuda.Stream | None = None, check: bool = True) -> DeviceBvh:
        """The BVH of device bounds [S,3] (float64).  With check=False the call stays asynchronous and the
        caller reads ``self.status`` (0 = valid) after the stream reaches it."""
        n = _check_shapes(lower.shape, upper.shape)
        if lower.dtype != torch.float64 or upper.dtype != torch.float64:
            raise ValueError("device BVH bounds must be float64 tensors")
        if lower.device != self.device or upper.device != self.device:
            raise ValueError(f"device BVH bounds must live on {self.device}")
        with self._lock:
            return self._build(lower.contiguous(), upper.contiguous(), n, leaf_size, stream, check)

    def _build(self, lower: torch.Tensor, upper: torch.Tensor, n: int, leaf_size: int,
               stream: torch.cuda.Stream | None, check: bool) -> DeviceBvh:
        ws_bytes, staging_bytes, nodes = _lib.device_bvh_plan(n, leaf_size)
        self._buffers(ws_bytes, staging_bytes)
        assert self.workspace is not None and self.staging is not None
        f64 = dict(dtype=torch.float64, device=self.device)
        i64 = dict(dtype=torch.int64, device=self.device)
        out = DeviceBvh(torch.empty((nodes, 3), **f64), torch.empty((nodes, 3), **f64), torch.empty(nodes, **i64),
                        torch.empty(nodes, **i64), torch.empty(nodes, **i64), torch.empty(n, **i64), nodes, 0, 0,
                        max(1, int(leaf_size)))
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int64)
        desc = _lib.ACBvh(ctypes.cast(out.bounds_min.data_ptr(), dp), ctypes.cast(out.bounds_max.data_ptr(), dp),
                          ctypes.cast(out.start.data_ptr(), ip), ctypes.cast(out.count.data_ptr(), ip),
                          ctypes.cast(out.escape.data_ptr(), ip), ctypes.cast(out.primitives.data_ptr(), ip), 0, 0, 0)
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().ac_bvh_build_device(
                ctypes.c_void_p(lower.data_ptr()), ctypes.c_void_p(upper.data_ptr()), n, int(leaf_size),
                ctypes.byref(desc), ctypes.c_void_p(self.status.data_ptr()),
                ctypes.c_void_p(self.workspace.data_ptr()), self.workspace.numel(),
                ctypes.c_void_p(self.staging.data_ptr()), ctypes.c_void_p(s.cuda_stream)), "ac_bvh_build_device")
            ev = torch.cuda.Event()
            ev.record(s)
            self._copied = ev
        out.node_count, out.leaf_count, out.max_depth = int(desc.node_count), int(desc.leaf_count), int(desc.max_depth)
        out.inputs = (lower, upper)
        if check:
            ev.synchronize()
            _raise_status(int(self.status.item()))
        return out


_BUILDERS: dict[int, DeviceBvhBuilder] = {}
_BUILDERS_LOCK = threading.Lock()


def builder(device: int = 0) -> DeviceBvhBuilder:
    """The process's shared builder for one device."""
    with _BUILDERS_LOCK:
        if device not in _BUILDERS:
            _BUILDERS[device] = DeviceBvhBuilder(device)
        return _BUILDERS[device]


def build_bvh(bounds_min: np.ndarray, bounds_max: np.ndarray, *, leaf_size: int = 4, device: int = 0) -> dict[str, Any]:
    """Drop-in for bvh.py:8-77: the same dict, built on the GPU (bounds copied up, arrays copied back)."""
    lower = np.asarray(bounds_min, dtype=np.float64)
    upper = np.asarray(bounds_max, dtype=np.float64)
    _check_shapes(lower.shape, upper.shape)
    b = builder(device)
    lo = torch.from_numpy(np.ascontiguousarray(lower)).to(b.device, non_blocking=False)
    hi = torch.from_numpy(np.ascontiguousarray(upper)).to(b.device, non_blocking=False)
    return b.build(lo, hi, leaf_size=leaf_size).to_numpy()
