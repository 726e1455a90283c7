"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No dataset or material library is needed: every scene is generated from a
seed as a plain room spec (see ``scene.py``) plus trace settings.

* ``shoebox``    6 x 4 x 3 m, 6 surfaces, per-surface six-band absorption
* ``u_furnished`` U-shaped 6 x 10 x 2.8 m room (api.py:920-925 corner formula) with 20
  seeded cabinet boxes, cardioid source, 8-mic circular array (mic.py:31-34, 65-77)
* ``apartment``  6-8 grid-tiled rooms, 0.15 m thick shared walls as two faces,
  0.9 x 2.1 m door gaps with headers, 10-25 furniture objects per room
* ``mixed_batch`` scenes log-uniform between shoebox and apartment, 1-4 sources,
  1-8 channels, 1e4-1e6 rays
* ``request_stream`` Poisson arrivals over the mixed-batch population, 20% moving sources
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import Any

import numpy as np

from acoustic_agent_b200.scene import count_surfaces, point_in_polygon


@dataclass(frozen=True)
class TraceConfig:
    """The SimConfig fields the reflection path reads (models.py:64-116)."""

    fs: int = 16000
    c: float = 343.0
    duration_s: float = 1.0
    rt_duration_s: float = 1.0
    rt_num_rays: int = 10000
    rt_num_bounces: int = 50
    rt_bin_duration_s: float = 0.01
    rt_specular_exponent: float = 100.0
    rt_irradiance_min_distance: float = 1.0
    rt_source_radius: float = 0.1
    rt_listener_radius: float = 0.1
    intersection_backend: str = "linear"
    bvh_min_surfaces: int = 16
    seed: int = 1729
    rt_precision: str = "float32"
    rt_accelerator: str = "b200"
    rt_cuda_device: int = 0
    collect_visual_paths: bool = False
    render_ambisonics: bool = False

    @property
    def num_bins(self) -> int:
        return max(1, int(math.ceil(max(self.rt_duration_s, self.duration_s) / self.rt_bin_duration_s)))

    @property
    def max_path_length(self) -> float:
        return max(self.rt_duration_s, self.duration_s) * self.c


@dataclass
class Workload:
    name: str
    spec: dict[str, Any]
    sources: list[tuple[float, float, float]]
    listeners: list[tuple[float, float, float]]   # one entry per receiver channel
    source_model: str | dict[str, Any] | None
    config: TraceConfig
    meta: dict[str, Any] = field(default_factory=dict)

    @property
    def num_traces(self) -> int:
        return len(self.sources) * len(self.listeners)


def _uniform_materials() -> dict[str, Any]:
    return {"wall": {"absorption": [0.06] * 6, "scattering": [0.12] * 6},
            "floor": {"absorption": [0.10] * 6, "scattering": [0.10] * 6},
            "ceiling": {"absorption": [0.08] * 6, "scattering": [0.10] * 6}}


def with_surface_materials(spec: dict[str, Any], seed: int, *, absorption=(0.05, 0.5),
                           scattering: float | tuple[float, float] = 0.1) -> dict[str, Any]:
    """Per-surface six-band absorption drawn from the seed (and scattering, fixed or drawn)."""
    rng = np.random.default_rng(seed)
    n = count_surfaces(spec)
    out = dict(spec)
    out["surface_absorption"] = rng.uniform(absorption[0], absorption[1], (n, 6)).tolist()
    if isinstance(scattering, tuple):
        out["surface_scattering"] = rng.uniform(scattering[0], scattering[1], n).tolist()
    else:
        out["surface_scattering"] = [float(scattering)] * n
    return out


def circular_array(center: tuple[float, float, float], count: int = 8, radius: float = 0.05,
                   orientation_deg: float = 0.0) -> list[tuple[float, float, float]]:
    """Channel positions of mic.py:65-77 (offsets rounded to 1e-6 like the reference)."""
    start = math.radians(orientation_deg)
    out = []
    for index in range(count):
        dx = round(math.cos(start + 2.0 * math.pi * index / count) * radius, 6)
        dy = round(math.sin(start + 2.0 * math.pi * index / count) * radius, 6)
        out.append((center[0] + dx, center[1] + dy, center[2] + 0.0))
    return out


def u_shape_corners(width: float, depth: float, opening_width: float = 0.42, opening_depth: float = 0.82,
                    opening_offset: float = 0.5) -> list[tuple[float, float]]:
    """api.py:920-925 ``_parametric_corners('u_shape', ...)``."""
    clamp = lambda value, lo, hi: max(lo, min(hi, float(value)))
    opening_w = width * clamp(opening_width, 0.2, 0.72)
    opening_d = depth * clamp(opening_depth, 0.18, 0.82)
    opening_x = (width - opening_w) * clamp(opening_offset, 0.0, 1.0)
    left_x, right_x, inner_y = opening_x, opening_x + opening_w, depth - opening_d
    return [(0.0, 0.0), (width, 0.0), (width, depth), (right_x, depth), (right_x, inner_y), (left_x, inner_y),
            (left_x, depth), (0.0, depth)]


def shoebox(seed: int = 1729, *, rays: int = 10000, bounces: int = 50) -> Workload:
    spec = {"corners": [(0.0, 0.0), (6.0, 0.0), (6.0, 4.0), (0.0, 4.0)], "height": 3.0,
            "materials": _uniform_materials()}
    spec = with_surface_materials(spec, seed, scattering=0.1)
    cfg = TraceConfig(fs=16000, duration_s=1.0, rt_duration_s=1.0, rt_num_rays=rays, rt_num_bounces=bounces,
                      rt_bin_duration_s=0.01, intersection_backend="linear", seed=seed)
    return Workload("shoebox_6x4x3", spec, [(1.5, 1.2, 1.5)], [(4.2, 2.9, 1.6)], None, cfg,
                    {"triangles_nominal": 12})


def _place_boxes(rng: np.random.Generator, corners, count: int, keep_clear: list[tuple[float, float]],
                 *, side=(0.3, 2.0), clear_radius: float = 0.6, height_limit: float = 2.6,
                 types=("cabinet",), type_weights=None, region=None) -> list[dict[str, Any]]:
    xs = [c[0] for c in corners]
    ys = [c[1] for c in corners]
    x0, x1, y0, y1 = (min(xs), max(xs), min(ys), max(ys)) if region is None else region
    objects = []
    attempts = 0
    while len(objects) < count and attempts < 200 * max(count, 1):
        attempts += 1
        size = rng.uniform(side[0], side[1], 3)
        size[2] = min(size[2], height_limit)
        center = (float(rng.uniform(x0, x1)), float(rng.uniform(y0, y1)))
        if not point_in_polygon(center, corners):
            continue
        reach = 0.5 * math.hypot(size[0], size[1])
        if any(math.hypot(center[0] - p[0], center[1] - p[1]) < reach + clear_radius for p in keep_clear):
            continue
        kind = str(rng.choice(types, p=type_weights)) if len(types) > 1 else types[0]
        objects.append({"type": kind, "size": [float(v) for v in size], "position": [center[0], center[1]],
                        "rotation": float(rng.uniform(0.0, 90.0)), "z": float(size[2] * 0.5)})
    return objects


def u_furnished(seed: int = 1729, *, rays: int = 200_000, bounces: int = 100, channels: int = 8) -> Workload:
    corners = u_shape_corners(6.0, 10.0, 0.42, 0.82, 0.5)
    source = (5.766, 2.587, 1.231)
    mic_center = (1.079, 6.252, 1.348)
    rng = np.random.default_rng(seed)
    objects = _place_boxes(rng, corners, 20, [source[:2], mic_center[:2]])
    spec = {"corners": corners, "height": 2.8, "materials": _uniform_materials(), "objects": objects}
    spec = with_surface_materials(spec, seed + 1, scattering=(0.05, 0.5))
    cfg = TraceConfig(fs=48000, duration_s=2.0, rt_duration_s=2.0, rt_num_rays=rays, rt_num_bounces=bounces,
                      rt_bin_duration_s=0.001, intersection_backend="bvh", seed=seed)
    listeners = circular_array(mic_center, count=8, radius=0.05)[:channels]
    return Workload("u_room_20_boxes", spec, [source], listeners, "cardioid", cfg)


def apartment(seed: int = 1729, *, rays: int = 1_000_000, bounces: int = 200, rooms: int | None = None,
              objects_per_room: tuple[int, int] = (10, 25), fs: int = 48000, duration: float = 2.0,
              bin_duration: float = 0.001) -> Workload:
    """Grid-tiled multi-room apartment with thick shared walls and open doors."""
    rng = np.random.default_rng(seed)
    n_rooms = int(rooms if rooms is not None else rng.integers(6, 9))
    cols = int(math.ceil(math.sqrt(n_rooms * 1.5)))
    cols = max(1, min(cols, n_rooms))
    rows = int(math.ceil(n_rooms / cols))
    widths = rng.uniform(2.5, 6.0, cols)
    depths = rng.uniform(2.5, 6.0, rows)
    xs = np.concatenate([[0.0], np.cumsum(widths)])
    ys = np.concatenate([[0.0], np.cumsum(depths)])
    W, D, H = float(xs[-1]), float(ys[-1]), 2.7
    half_t = 0.075
    door_w, door_h = 0.9, 2.1
    cells = [(r, c) for r in range(rows) for c in range(cols)][:n_rooms]
    cell_set = set(cells)
    # Adjacent pairs and a door plan that keeps every room reachable.
    pairs = []
    for (r, c) in cells:
        if (r, c + 1) in cell_set:
            pairs.append(((r, c), (r, c + 1), "v"))
        if (r + 1, c) in cell_set:
            pairs.append(((r, c), (r + 1, c), "h"))
    order = rng.permutation(len(pairs))
    parent = {cell: cell for cell in cells}

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    doors = set()
    for k in order:
        a, b, _ = pairs[k]
        if find(a) != find(b):
            parent[find(a)] = find(b)
            doors.add(k)
    target = int(rng.integers(4, 8))
    for k in order:
        if len(doors) >= target:
            break
        doors.add(k)

    segments: list[dict[str, Any]] = []

    def add(a, b, z0=0.0, z1=H, kind="wall"):
        segments.append({"a": [float(a[0]), float(a[1])], "b": [float(b[0]), float(b[1])], "type": kind,
                         "z_min": float(z0), "z_max": float(z1), "name": f"{kind}_{len(segments)}"})

    # Hull of the occupied cells (row-major fill) traced as axis-aligned outline.
    hull = _grid_hull(cells, xs, ys)
    for i in range(len(hull)):
        add(hull[i], hull[(i + 1) % len(hull)])
    for k, (a, b, orient) in enumerate(pairs):
        (r, c), _ = a, b
        if orient == "v":  # wall at x = xs[c+1] between rows ys[r]..ys[r+1]
            x = xs[c + 1]
            lo, hi = ys[r] + half_t, ys[r + 1] - half_t
            for face in (x - half_t, x + half_t):
                if k in doors:
                    mid = float(rng.uniform(lo + 0.2 + door_w / 2, hi - 0.2 - door_w / 2)) if hi - lo > door_w + 0.4 else (lo + hi) / 2
                    add((face, lo), (face, mid - door_w / 2))
                    add((face, mid + door_w / 2), (face, hi))
                    add((face, mid - door_w / 2), (face, mid + door_w / 2), door_h, H)
                else:
                    add((face, lo), (face, hi))
        else:  # wall at y = ys[r+1] between cols xs[c]..xs[c+1]
            y = ys[r + 1]
            lo, hi = xs[c] + half_t, xs[c + 1] - half_t
            for face in (y - half_t, y + half_t):
                if k in doors:
                    mid = float(rng.uniform(lo + 0.2 + door_w / 2, hi - 0.2 - door_w / 2)) if hi - lo > door_w + 0.4 else (lo + hi) / 2
                    add((lo, face), (mid - door_w / 2, face))
                    add((mid + door_w / 2, face), (hi, face))
                    add((mid - door_w / 2, face), (mid + door_w / 2, face), door_h, H)
                else:
                    add((lo, face), (hi, face))
    # Source and listener in two different rooms, away from walls.
    src_cell, lst_cell = cells[0], cells[-1]

    def room_point(cell, z):
        r, c = cell
        return (float(rng.uniform(xs[c] + 0.8, xs[c + 1] - 0.8)), float(rng.uniform(ys[r] + 0.8, ys[r + 1] - 0.8)), z)

    source = room_point(src_cell, 1.5)
    listener = room_point(lst_cell, 1.6)
    objects: list[dict[str, Any]] = []
    for (r, c) in cells:
        count = int(rng.integers(objects_per_room[0], objects_per_room[1] + 1))
        region = (xs[c] + 0.3, xs[c + 1] - 0.3, ys[r] + 0.3, ys[r + 1] - 0.3)
        objects += _place_boxes(rng, hull, count, [source[:2], listener[:2]], side=(0.3, 1.2), region=region,
                                clear_radius=0.4, height_limit=2.2,
                                types=("cabinet", "table", "sanitary_fixture", "structural_element"),
                                type_weights=(0.55, 0.25, 0.1, 0.1))
    spec = {"corners": hull, "height": H, "materials": _uniform_materials(), "surface_segments": segments,
            "objects": objects}
    spec = with_surface_materials(spec, seed + 1, scattering=(0.05, 0.5))
    cfg = TraceConfig(fs=fs, duration_s=duration, rt_duration_s=duration, rt_num_rays=rays, rt_num_bounces=bounces,
                      rt_bin_duration_s=bin_duration, intersection_backend="bvh", seed=seed)
    return Workload(f"apartment_{n_rooms}_rooms", spec, [source], [listener], None, cfg,
                    {"rooms": n_rooms, "doors": len(doors)})


def _grid_hull(cells, xs, ys) -> list[tuple[float, float]]:
    """Counter-clockwise outline of a set of grid cells filled row-major from the origin."""
    rows = max(r for r, _ in cells) + 1
    cols_per_row = [max(c for r2, c in cells if r2 == r) + 1 for r in range(rows)]
    pts = [(0.0, 0.0)]
    # bottom row extends to cols_per_row[0]; rows above may be shorter (only the last can be partial)
    pts.append((float(xs[cols_per_row[0]]), 0.0))
    for r in range(rows):
        x_edge = float(xs[cols_per_row[r]])
        if r + 1 < rows and cols_per_row[r + 1] != cols_per_row[r]:
            pts.append((x_edge, float(ys[r + 1])))
            pts.append((float(xs[cols_per_row[r + 1]]), float(ys[r + 1])))
    pts.append((float(xs[cols_per_row[-1]]), float(ys[rows])))
    pts.append((0.0, float(ys[rows])))
    cleaned = []
    for p in pts:
        if not cleaned or (abs(p[0] - cleaned[-1][0]) > 1e-12 or abs(p[1] - cleaned[-1][1]) > 1e-12):
            cleaned.append(p)
    return cleaned


def mixed_batch(seed: int = 1729, count: int = 256, *, max_rays: int = 1_000_000, min_rays: int = 10_000,
                fs: int = 16000) -> list[Workload]:
    """Scenes log-uniform in size between the shoebox and the apartment."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        u = float(rng.uniform())
        rooms = 1 + int(round(u * 7))
        rays = int(round(math.exp(rng.uniform(math.log(min_rays), math.log(max_rays)))))
        bounces = int(round(50 * 4 ** u))
        duration = float(rng.uniform(1.0, 2.0))
        n_sources = int(rng.integers(1, 5))
        n_channels = int(rng.integers(1, 9))
        sub_seed = int(rng.integers(0, 2**31 - 1))
        if rooms == 1:
            base = _single_room(sub_seed, u)
        else:
            base = apartment(sub_seed, rays=rays, bounces=bounces, rooms=rooms,
                             objects_per_room=(int(2 + 8 * u), int(5 + 20 * u)), fs=fs, duration=duration,
                             bin_duration=0.01)
        srng = np.random.default_rng(sub_seed + 17)
        sources = [base.sources[0]] + [_jitter(srng, base.sources[0], base.spec) for _ in range(n_sources - 1)]
        listeners = circular_array(base.listeners[0], count=max(3, n_channels), radius=0.05)[:n_channels] \
            if n_channels > 1 else [base.listeners[0]]
        cfg = replace(base.config, fs=fs, duration_s=duration, rt_duration_s=duration, rt_num_rays=rays,
                      rt_num_bounces=bounces, rt_bin_duration_s=0.01, seed=sub_seed,
                      intersection_backend="bvh" if count_surfaces(base.spec) >= 16 else "linear")
        out.append(Workload(f"mix_{k}", base.spec, sources, listeners, None, cfg, {"size_quantile": u}))
    return out


def _single_room(seed: int, u: float) -> Workload:
    rng = np.random.default_rng(seed)
    w, d = float(rng.uniform(3.0, 8.0)), float(rng.uniform(3.0, 8.0))
    corners = [(0.0, 0.0), (w, 0.0), (w, d), (0.0, d)]
    source = (float(rng.uniform(0.8, w - 0.8)), float(rng.uniform(0.8, d - 0.8)), 1.5)
    listener = (float(rng.uniform(0.8, w - 0.8)), float(rng.uniform(0.8, d - 0.8)), 1.6)
    n_obj = int(round(10 * u))
    objects = _place_boxes(rng, corners, n_obj, [source[:2], listener[:2]], side=(0.3, 1.5))
    spec = {"corners": corners, "height": 3.0, "materials": _uniform_materials(), "objects": objects}
    spec = with_surface_materials(spec, seed + 1, scattering=(0.05, 0.5))
    return Workload("room", spec, [source], [listener], None, TraceConfig(seed=seed))


def _jitter(rng: np.random.Generator, point, spec, radius: float = 1.5) -> tuple[float, float, float]:
    corners = spec["corners"]
    for _ in range(100):
        cand = (point[0] + float(rng.uniform(-radius, radius)), point[1] + float(rng.uniform(-radius, radius)), point[2])
        if point_in_polygon(cand[:2], corners):
            return cand
    return tuple(point)


def request_stream(seed: int = 1729, rate_hz: float = 100.0, duration_s: float = 10.0, *,
                   population: list[Workload] | None = None, moving_fraction: float = 0.2,
                   keyframes: int = 8, path_length_m: float = 3.0) -> list[dict[str, Any]]:
    """Poisson arrivals; a moving-source request becomes `keyframes` solves along a seeded polyline."""
    rng = np.random.default_rng(seed)
    pool = population if population is not None else mixed_batch(seed + 1, 64)
    t = 0.0
    out = []
    while True:
        t += float(rng.exponential(1.0 / rate_hz))
        if t > duration_s:
            break
        base = pool[int(rng.integers(0, len(pool)))]
        moving = bool(rng.uniform() < moving_fraction)
        sources = [base.sources[0]]
        if moving:
            heading = float(rng.uniform(0.0, 2.0 * math.pi))
            step = path_length_m / max(1, keyframes - 1)
            pts = [base.sources[0]]
            for _ in range(keyframes - 1):
                heading += float(rng.uniform(-0.6, 0.6))
                cand = (pts[-1][0] + step * math.cos(heading), pts[-1][1] + step * math.sin(heading), pts[-1][2])
                pts.append(cand if point_in_polygon(cand[:2], base.spec["corners"]) else pts[-1])
            sources = pts
        out.append({"arrival_s": t, "workload": base, "sources": sources, "moving": moving})
    return out
