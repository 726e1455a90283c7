"""Host-side scene compiler: room description -> surface SoA arrays + BVH.

Restates the parts of Acoustic Agent that turn a room into the flat arrays
its tracers consume, so that the GPU backend can run without the reference
installed:

- ``acoustic_agent/steam_rt.py:291-307``  ``RoomRayScene.__init__`` (surface order:
  boundary walls, floor, ceiling, object boxes)
- ``acoustic_agent/steam_rt.py:85-116``   ``_WallSurface`` (z range clamp, normal)
- ``acoustic_agent/steam_rt.py:184-198``  ``_BoxSurface`` (size clamp, axes, z range)
- ``acoustic_agent/steam_rt.py:524-568``  ``_boundary_wall_surfaces``
- ``acoustic_agent/steam_rt.py:613-648``  ``_object_box_surfaces`` (material-library
  fallback branch: proxy boxes with the wall material)
- ``acoustic_agent/steam_rt.py:738-831``  ``_object_proxy_boxes``
- ``acoustic_agent/steam_rt.py:234-262``  ``_surface_bounds``
- ``acoustic_agent/steam_rt.py:834-924``  ``_scene_kernel_arrays``
- ``acoustic_agent/geometry.py:194-212``  ``point_in_polygon`` (+ boundary test)
- ``acoustic_agent/materials.py:511-535`` ``fallback_material`` absorption table

The BVH itself is built by the native library (``ac_bvh_build``), which
restates ``acoustic_agent/bvh.py:8-77`` exactly.

A scene description ("spec") is a plain dict:

``corners`` [[x, y], ...], ``height``, ``materials`` {kind: {"absorption": [6] or
{band: a}, "scattering": ...}}, optional ``surface_segments`` and ``objects``
(same item format as ``Room.metadata``), and optional per-surface overrides
``surface_absorption`` [S, 6] / ``surface_scattering`` [S] applied after the
surfaces are built (the reference keys materials per surface kind only).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any, Mapping, Sequence

import numpy as np

FREQUENCY_BANDS: tuple[str, ...] = ("125", "250", "500", "1000", "2000", "4000")
NUM_BANDS = 6
_EPS = 1e-6
_BVH_BOUNDS_EPS = 2.0e-6

# materials.py:512-525 fallback absorption by semantic; scattering 0.12.
_FALLBACK_ALPHA = {
    "wall": 0.06, "floor": 0.10, "ceiling": 0.08, "door": 0.14, "carpet": 0.45, "carpet_rug": 0.45,
    "curtain": 0.45, "curtain_blind": 0.45, "sofa": 0.55, "sofa_couch": 0.55, "window": 0.08,
    "window_glass": 0.08,
}

KIND_WALL = 0
KIND_HORIZONTAL = 1
KIND_BOX = 2


def _band_values(material: Mapping[str, Any] | None, attr: str, default: float) -> np.ndarray:
    """steam_rt.py:3432 ``_band_array``: per-band values with a default for missing bands."""
    table = (material or {}).get(attr)
    if table is None:
        return np.full(NUM_BANDS, float(default))
    if isinstance(table, Mapping):
        return np.asarray([float(table.get(b, default)) for b in FREQUENCY_BANDS], dtype=float)
    arr = np.asarray(table, dtype=float).reshape(-1)
    if arr.size == 1:
        return np.full(NUM_BANDS, float(arr[0]))
    if arr.size != NUM_BANDS:
        raise ValueError(f"material {attr} must have {NUM_BANDS} bands")
    return arr.astype(float)


def _fallback_material(semantic: str) -> dict[str, Any]:
    alpha = _FALLBACK_ALPHA.get(semantic, 0.20)
    return {"absorption": [alpha] * NUM_BANDS, "scattering": [0.12] * NUM_BANDS}


def _point_on_boundary(point: tuple[float, float], corners: Sequence[Sequence[float]], tol: float = 1e-8) -> bool:
    p = np.asarray(point, dtype=float)
    pts = np.asarray(corners, dtype=float)
    for a, b in zip(pts, np.roll(pts, -1, axis=0)):
        ab = b - a
        denom = float(np.dot(ab, ab))
        if denom <= tol:
            continue
        t = float(np.clip(np.dot(p - a, ab) / denom, 0.0, 1.0))
        if float(np.linalg.norm(a + t * ab - p)) <= tol:
            return True
    return False


def point_in_polygon(point: Sequence[float], corners: Sequence[Sequence[float]]) -> bool:
    """Even-odd test plus the on-boundary check used to keep object boxes (geometry.py:194-212)."""
    x, y = float(point[0]), float(point[1])
    inside = False
    pts = [tuple(float(v) for v in c[:2]) for c in corners]
    j = len(pts) - 1
    for i, (xi, yi) in enumerate(pts):
        xj, yj = pts[j]
        if (yi > y) != (yj > y):
            denom = yj - yi
            if abs(denom) <= 1e-12:
                j = i
                continue
            x_at_y = (xj - xi) * (y - yi) / denom + xi
            if x < x_at_y:
                inside = not inside
        j = i
    return inside or _point_on_boundary((x, y), pts)


def object_proxy_boxes(item: Mapping[str, Any], room_height: float) -> list[dict[str, Any]]:
    """Proxy boxes for one furniture object (steam_rt.py:738-831)."""
    try:
        size = np.asarray(item.get("size", (1.0, 1.0, 1.0)), dtype=float)
        if size.shape != (3,) or not np.all(np.isfinite(size)) or float(np.min(size)) <= 0.0:
            return []
        position = item.get("position", (0.0, 0.0))
        center = np.asarray((float(position[0]), float(position[1])), dtype=float)
        rotation = float(item.get("rotation", 0.0))
        z_center = float(item.get("z", size[2] * 0.5))
    except Exception:
        return []
    object_type = str(item.get("type", "furniture"))
    height = float(size[2])
    angle = math.radians(rotation)
    axis_u = np.asarray([math.cos(angle), math.sin(angle)], dtype=float)
    axis_v = np.asarray([-math.sin(angle), math.cos(angle)], dtype=float)
    if object_type == "table":
        leg_h = max(0.05, height)
        boxes = [{
            "part": "top", "center": center,
            "size": np.asarray([size[0], size[1], min(0.08, max(0.04, height * 0.16))], dtype=float),
            "z": min(room_height, height), "rotation": rotation,
        }]
        for leg_index, (sx, sy) in enumerate(((-1.0, -1.0), (1.0, -1.0), (-1.0, 1.0), (1.0, 1.0))):
            offset = axis_u * (sx * size[0] * 0.42) + axis_v * (sy * size[1] * 0.38)
            boxes.append({
                "part": f"leg{leg_index}", "center": center + offset,
                "size": np.asarray([0.08, 0.08, leg_h], dtype=float),
                "z": min(room_height, leg_h * 0.5), "rotation": rotation,
            })
        return boxes
    if object_type == "sanitary_fixture":
        base_z = z_center - height * 0.5
        wall_height = height * 0.72
        boxes = [{
            "part": "base", "center": center,
            "size": np.asarray([size[0] * 0.82, size[1] * 0.72, height * 0.16], dtype=float),
            "z": min(room_height, base_z + height * 0.08), "rotation": rotation,
        }]
        for part, offset in (("back", -0.44), ("front", 0.44)):
            boxes.append({
                "part": part, "center": center + axis_v * (size[1] * offset),
                "size": np.asarray([size[0], size[1] * 0.12, wall_height], dtype=float),
                "z": min(room_height, base_z + wall_height * 0.5), "rotation": rotation,
            })
        for part, offset in (("left", -0.445), ("right", 0.445)):
            boxes.append({
                "part": part, "center": center + axis_u * (size[0] * offset),
                "size": np.asarray([size[0] * 0.11, size[1] * 0.76, wall_height], dtype=float),
                "z": min(room_height, base_z + wall_height * 0.5), "rotation": rotation,
            })
        return boxes
    if object_type == "structural_element":
        base_z = z_center - height * 0.5
        return [
            {"part": "base", "center": center, "size": np.asarray([size[0], size[1], height * 0.06], dtype=float),
             "z": min(room_height, base_z + height * 0.03), "rotation": rotation},
            {"part": "shaft", "center": center,
             "size": np.asarray([size[0] * 0.78, size[1] * 0.78, height * 0.88], dtype=float),
             "z": min(room_height, base_z + height * 0.5), "rotation": rotation},
            {"part": "capital", "center": center, "size": np.asarray([size[0], size[1], height * 0.06], dtype=float),
             "z": min(room_height, base_z + height * 0.97), "rotation": rotation},
        ]
    return [{"part": "body", "center": center, "size": size, "z": z_center, "rotation": rotation}]


@dataclass
class _Surface:
    kind: int
    name: str
    absorption: np.ndarray
    scattering: np.ndarray
    normal: np.ndarray
    a: np.ndarray | None = None
    b: np.ndarray | None = None
    z_min: float = 0.0
    z_max: float = 0.0
    z: float = 0.0
    center: np.ndarray | None = None
    axis_u: np.ndarray | None = None
    axis_v: np.ndarray | None = None
    half_width: float = 0.0
    half_depth: float = 0.0


def _wall(a, b, height, name, absorption, scattering, z_min=0.0, z_max=None) -> _Surface:
    zmin = max(0.0, float(z_min))
    zmax = min(float(height), float(height if z_max is None else z_max))
    seg = b - a
    normal_xy = np.asarray([seg[1], -seg[0]], dtype=float)
    n = float(np.linalg.norm(normal_xy))
    normal = np.asarray([normal_xy[0] / n, normal_xy[1] / n, 0.0], dtype=float) if n > _EPS else np.asarray([1.0, 0.0, 0.0])
    return _Surface(KIND_WALL, name, absorption, scattering, normal, a=a, b=b, z_min=zmin, z_max=zmax)


def _box(center, size, rotation_deg, z_center, name, absorption, scattering) -> _Surface:
    center = np.asarray(center, dtype=float)
    size = np.maximum(np.asarray(size, dtype=float), 1e-3)
    angle = math.radians(float(rotation_deg))
    axis_u = np.asarray([math.cos(angle), math.sin(angle)], dtype=float)
    axis_v = np.asarray([-math.sin(angle), math.cos(angle)], dtype=float)
    half_height = float(size[2] * 0.5)
    z_min = float(max(0.0, z_center - half_height))
    z_max = float(max(z_min + 1e-3, z_center + half_height))
    return _Surface(KIND_BOX, name, absorption, scattering, np.asarray([0.0, 0.0, 1.0]), center=center,
                    axis_u=axis_u, axis_v=axis_v, half_width=float(size[0] * 0.5), half_depth=float(size[1] * 0.5),
                    z_min=z_min, z_max=z_max)


def _surfaces_from_spec(spec: Mapping[str, Any]) -> tuple[list[_Surface], np.ndarray, float]:
    corners_xy = [np.asarray(c[:2], dtype=float) for c in spec["corners"]]
    height = float(spec["height"])
    materials: Mapping[str, Any] = spec.get("materials") or {}
    wall = materials.get("wall") or (next(iter(materials.values())) if materials else {})
    floor = materials.get("floor", wall)
    ceiling = materials.get("ceiling", wall)
    surfaces: list[_Surface] = []

    segments = []
    raw_segments = spec.get("surface_segments")
    if isinstance(raw_segments, list):
        for item in raw_segments:
            if not isinstance(item, Mapping):
                continue
            try:
                a = np.asarray(item.get("a"), dtype=float)
                b = np.asarray(item.get("b"), dtype=float)
                kind = str(item.get("type", "wall")).lower()
                z_min = float(item.get("z_min", 0.0))
                z_max = float(item.get("z_max", height))
                name = str(item.get("name", f"{kind}_{len(segments)}"))
            except (TypeError, ValueError):
                continue
            valid = (a.shape == (2,) and b.shape == (2,) and np.all(np.isfinite(a)) and np.all(np.isfinite(b))
                     and math.isfinite(z_min) and math.isfinite(z_max) and z_max - z_min > _EPS)
            if valid and float(np.linalg.norm(b - a)) > _EPS:
                segments.append((a, b, kind if kind in {"wall", "door", "window"} else "wall", z_min, z_max, name))
    if not segments:
        segments = [(a, corners_xy[(i + 1) % len(corners_xy)], "wall", 0.0, height, f"wall_{i}")
                    for i, a in enumerate(corners_xy)]
    for a, b, kind, z_min, z_max, name in segments:
        material = materials.get(kind, wall if kind == "wall" else _fallback_material(kind))
        surfaces.append(_wall(a, b, height, name, _band_values(material, "absorption", 0.1),
                              _band_values(material, "scattering", 0.12), z_min=z_min, z_max=z_max))

    surfaces.append(_Surface(KIND_HORIZONTAL, "floor", _band_values(floor, "absorption", 0.12),
                             _band_values(floor, "scattering", 0.1), np.asarray([0.0, 0.0, 1.0]), z=0.0))
    surfaces.append(_Surface(KIND_HORIZONTAL, "ceiling", _band_values(ceiling, "absorption", 0.1),
                             _band_values(ceiling, "scattering", 0.1), np.asarray([0.0, 0.0, -1.0]), z=height))

    raw_objects = spec.get("objects") or []
    if isinstance(raw_objects, list):
        corners_list = [tuple(float(v) for v in c[:2]) for c in spec["corners"]]
        for index, item in enumerate(raw_objects):
            if not isinstance(item, Mapping) or str(item.get("semantic", "")) == "small_objects_ignore":
                continue
            # The reference samples a library material here; without the library it
            # falls back to the wall material and the proxy boxes (steam_rt.py:625-629).
            absorption = _band_values(wall, "absorption", 0.2)
            scattering = _band_values(wall, "scattering", 0.18)
            for box in object_proxy_boxes(item, height):
                center = np.asarray(box["center"], dtype=float)
                if not point_in_polygon(center, corners_list):
                    continue
                surfaces.append(_box(center, box["size"], float(box["rotation"]), float(box["z"]),
                                     f"object_{index}_{str(item.get('type', 'furniture'))}_{str(box['part'])}",
                                     absorption, scattering))

    override_a = spec.get("surface_absorption")
    if override_a is not None:
        override_a = np.asarray(override_a, dtype=float)
        if override_a.shape != (len(surfaces), NUM_BANDS):
            raise ValueError(f"surface_absorption must have shape [{len(surfaces)}, {NUM_BANDS}]")
        for surface, row in zip(surfaces, override_a):
            surface.absorption = row.copy()
    override_s = spec.get("surface_scattering")
    if override_s is not None:
        override_s = np.asarray(override_s, dtype=float)
        if override_s.ndim == 1:
            override_s = np.repeat(override_s[:, None], NUM_BANDS, axis=1)
        if override_s.shape != (len(surfaces), NUM_BANDS):
            raise ValueError(f"surface_scattering must have {len(surfaces)} rows")
        for surface, row in zip(surfaces, override_s):
            surface.scattering = row.copy()
    return surfaces, np.asarray(spec["corners"], dtype=np.float64)[:, :2], height


def count_surfaces(spec: Mapping[str, Any]) -> int:
    """Number of surfaces the spec compiles to (before any per-surface override)."""
    plain = {k: v for k, v in spec.items() if k not in ("surface_absorption", "surface_scattering")}
    return len(_surfaces_from_spec(plain)[0])


def surface_bounds(arrays: Mapping[str, Any]) -> tuple[np.ndarray, np.ndarray]:
    """Per-surface AABBs padded by 2e-6 (steam_rt.py:234-262)."""
    kinds = np.asarray(arrays["kinds"])
    S = kinds.shape[0]
    lower = np.zeros((S, 3))
    upper = np.zeros((S, 3))
    corners = np.asarray(arrays["corners"], dtype=np.float64)
    for i in range(S):
        if kinds[i] == KIND_WALL:
            a = arrays["wall_a"][i]
            b = arrays["wall_a"][i] + arrays["wall_delta"][i]
            bb = arrays["_wall_b"][i] if "_wall_b" in arrays else b
            lower[i] = [min(float(a[0]), float(bb[0])), min(float(a[1]), float(bb[1])), float(arrays["wall_z"][i, 0])]
            upper[i] = [max(float(a[0]), float(bb[0])), max(float(a[1]), float(bb[1])), float(arrays["wall_z"][i, 1])]
        elif kinds[i] == KIND_BOX:
            extent = (np.abs(arrays["box_axis_u"][i]) * float(arrays["box_half"][i, 0])
                      + np.abs(arrays["box_axis_v"][i]) * float(arrays["box_half"][i, 1]))
            c = arrays["box_center"][i]
            lower[i] = [float(c[0] - extent[0]), float(c[1] - extent[1]), float(arrays["box_z"][i, 0])]
            upper[i] = [float(c[0] + extent[0]), float(c[1] + extent[1]), float(arrays["box_z"][i, 1])]
        else:
            z = float(arrays["z_values"][i])
            lower[i] = [float(np.min(corners[:, 0])), float(np.min(corners[:, 1])), z]
            upper[i] = [float(np.max(corners[:, 0])), float(np.max(corners[:, 1])), z]
    return lower - _BVH_BOUNDS_EPS, upper + _BVH_BOUNDS_EPS


@dataclass
class SceneArrays:
    """The surface SoA contract of ``_scene_kernel_arrays`` (steam_rt.py:897-923), float64."""

    arrays: dict[str, Any] = field(default_factory=dict)

    def __getitem__(self, key: str) -> Any:
        return self.arrays[key]

    def __contains__(self, key: str) -> bool:
        return key in self.arrays

    @property
    def num_surfaces(self) -> int:
        return int(np.asarray(self.arrays["kinds"]).shape[0])

    @property
    def names(self) -> tuple[str, ...]:
        return tuple(self.arrays["names"])

    def triangle_equivalents(self) -> int:
        """Triangles an equivalent mesh would need: wall 2, box 12, polygon C-2."""
        kinds = np.asarray(self.arrays["kinds"])
        corners = np.asarray(self.arrays["corners"]).shape[0]
        return int(2 * np.sum(kinds == KIND_WALL) + 12 * np.sum(kinds == KIND_BOX)
                   + (corners - 2) * np.sum(kinds == KIND_HORIZONTAL))


def compile_scene(spec: Mapping[str, Any], *, bvh_builder=None) -> SceneArrays:
    """Build the SoA arrays and BVH for a room spec (steam_rt.py:834-924)."""
    surfaces, corners, height = _surfaces_from_spec(spec)
    S = len(surfaces)
    kinds = np.zeros(S, dtype=np.int64)
    wall_a = np.zeros((S, 2))
    wall_b = np.zeros((S, 2))
    wall_z = np.zeros((S, 2))
    wall_z[:, 1] = float(height)
    z_values = np.zeros(S)
    box_center = np.zeros((S, 2))
    box_axis_u = np.zeros((S, 2))
    box_axis_v = np.zeros((S, 2))
    box_half = np.zeros((S, 2))
    box_z = np.zeros((S, 2))
    normals = np.zeros((S, 3))
    absorption = np.zeros((S, NUM_BANDS))
    scattering = np.zeros(S)
    names = []
    for i, s in enumerate(surfaces):
        names.append(str(s.name))
        normals[i] = np.asarray(s.normal, dtype=np.float64)
        absorption[i] = np.asarray(s.absorption, dtype=np.float64)
        scattering[i] = float(np.mean(s.scattering))
        if s.kind == KIND_WALL:
            kinds[i] = 0
            wall_a[i] = s.a
            wall_b[i] = s.b
            wall_z[i] = [s.z_min, s.z_max]
        elif s.kind == KIND_BOX:
            kinds[i] = 2
            box_center[i] = s.center
            box_axis_u[i] = s.axis_u
            box_axis_v[i] = s.axis_v
            box_half[i] = [s.half_width, s.half_depth]
            box_z[i] = [s.z_min, s.z_max]
        else:
            kinds[i] = 1
            z_values[i] = float(s.z)
    arrays: dict[str, Any] = {
        "kinds": kinds, "wall_a": wall_a, "wall_delta": wall_b - wall_a, "wall_z": wall_z, "z_values": z_values,
        "box_center": box_center, "box_axis_u": box_axis_u, "box_axis_v": box_axis_v, "box_half": box_half,
        "box_z": box_z, "normals": normals, "absorption": absorption, "reflection": 1.0 - absorption,
        "scattering": scattering, "names": tuple(names), "corners": corners, "height": float(height),
        "_wall_b": wall_b,
    }
    lower, upper = surface_bounds(arrays)
    del arrays["_wall_b"]
    arrays["surface_bounds_min"] = lower
    arrays["surface_bounds_max"] = upper
    if bvh_builder is None:
        from acoustic_agent_b200 import _lib
        bvh_builder = _lib.build_bvh
    bvh = bvh_builder(lower, upper)
    arrays.update({
        "bvh_bounds_min": bvh["bounds_min"], "bvh_bounds_max": bvh["bounds_max"], "bvh_start": bvh["start"],
        "bvh_count": bvh["count"], "bvh_escape": bvh["escape"], "bvh_primitives": bvh["primitives"],
        "bvh_node_count": int(bvh["node_count"]), "bvh_leaf_count": int(bvh["leaf_count"]),
        "bvh_max_depth": int(bvh["max_depth"]), "bvh_leaf_size": int(bvh["leaf_size"]),
    })
    return SceneArrays(arrays)


def from_reference_arrays(arrays: Mapping[str, Any]) -> SceneArrays:
    """Wrap the reference's own ``_scene_kernel_arrays`` dict (drop-in path)."""
    required = ("kinds", "wall_a", "wall_delta", "wall_z", "z_values", "box_center", "box_axis_u", "box_axis_v",
                "box_half", "box_z", "normals", "reflection", "scattering", "corners", "names", "bvh_bounds_min",
                "bvh_bounds_max", "bvh_start", "bvh_count", "bvh_escape", "bvh_primitives")
    missing = [key for key in required if key not in arrays]
    if missing:
        raise ValueError(f"scene arrays missing keys: {missing}")
    return SceneArrays(dict(arrays))
