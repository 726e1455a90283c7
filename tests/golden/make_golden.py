"""Generate golden vectors by running Acoustic Agent's own reflection tracer.

Run in a checkout that has the reference importable (this script reads it
from the directory given by --reference, default /root/reference):

    NUMBA_NUM_THREADS=8 python tests/golden/make_golden.py

The reference imports shapely and h5py at module level but the tracer never
calls them, so empty stand-ins are inserted into sys.modules.  Rooms are built
directly from ``models.Room`` / ``models.Material`` (the material SQLite
database is not needed).  For every case the script stores the reference's
scene arrays (``_scene_kernel_arrays``, including its BVH), the trace outputs
of ``_trace_energy_kernel`` in float64, and the per-ray hit-surface sequence
(the kernel's visual-candidate slots with one slot per ray).  Synthesis cases
store ``reconstruct_band_irs`` outputs.  The fixtures are what the oracle and
the GPU kernels are checked against; nothing at test time imports the
reference.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent


class _Stub(types.ModuleType):
    def __getattr__(self, item):
        if item.startswith("__"):
            raise AttributeError(item)
        return type(item, (), {})


def import_reference(path: str):
    for name in ("shapely", "shapely.geometry", "shapely.geometry.base", "shapely.ops", "h5py"):
        sys.modules.setdefault(name, _Stub(name))
    sys.modules["shapely"].affinity = _Stub("shapely.affinity")
    try:
        import networkx  # noqa: F401
    except Exception:
        sys.modules.setdefault("networkx", _Stub("networkx"))
    sys.path.insert(0, path)
    from acoustic_agent import steam_rt, models, directivity  # noqa: E402
    return steam_rt, models, directivity


def reference_room(models, spec):
    bands = models.FREQUENCY_BANDS

    def material(kind, data):
        absorption = data.get("absorption", [0.1] * 6)
        scattering = data.get("scattering", [0.1] * 6)
        return models.Material(id=f"golden_{kind}", name=kind, semantic=kind,
                               absorption={b: float(v) for b, v in zip(bands, absorption)},
                               scattering={b: float(v) for b, v in zip(bands, scattering)})

    materials = {k: material(k, v) for k, v in spec.get("materials", {}).items()}
    metadata = {}
    if spec.get("surface_segments") is not None:
        metadata["surface_segments"] = [dict(s) for s in spec["surface_segments"]]
    if spec.get("objects") is not None:
        metadata["objects"] = [dict(o) for o in spec["objects"]]
    return models.Room(id="golden", name="golden", corners=tuple((float(x), float(y)) for x, y in spec["corners"]),
                       height_m=float(spec["height"]), materials=materials, metadata=metadata)


def reference_arrays(steam_rt, models, spec):
    steam_rt._clear_static_caches()
    scene = steam_rt.RoomRayScene(reference_room(models, spec))
    if spec.get("surface_absorption") is not None:
        for surface, row in zip(scene.surfaces, spec["surface_absorption"]):
            surface.absorption = np.asarray(row, dtype=float)
    if spec.get("surface_scattering") is not None:
        for surface, value in zip(scene.surfaces, spec["surface_scattering"]):
            surface.scattering = np.full(6, float(value))
    arrays = steam_rt._scene_kernel_arrays(scene)
    return scene, arrays


VISUAL_POINT_RAYS = 64

ARRAY_KEYS = ("kinds", "wall_a", "wall_delta", "wall_z", "z_values", "box_center", "box_axis_u", "box_axis_v",
              "box_half", "box_z", "normals", "reflection", "scattering", "corners", "surface_bounds_min",
              "surface_bounds_max", "bvh_bounds_min", "bvh_bounds_max", "bvh_start", "bvh_count", "bvh_escape",
              "bvh_primitives")


def run_trace(steam_rt, directivity, arrays, trace):
    emitter = directivity.source_directivity(trace.get("source_model"))
    forward = directivity.source_forward(emitter)
    R = max(1, int(trace["rays"]))
    B = int(trace["bounces"])
    directions = steam_rt._sphere_samples(R, int(trace["seed"]))
    bank = steam_rt._diffuse_sample_bank(128)
    rnd, idx = steam_rt._diffuse_random_sequence(R, B, bank.shape[0], int(trace["seed"]))
    duration = float(trace["duration"])
    c = 343.0
    bin_dur = float(trace["bin_dur"])
    num_bins = max(1, int(math.ceil(duration / bin_dur)))
    src = np.asarray(trace["source"], dtype=float)
    lst = np.asarray(trace["listener"], dtype=float)
    direct_delay = float(np.linalg.norm(src - lst)) / c
    use_bvh = trace["backend"] == "bvh"
    res = steam_rt._trace_energy_kernel(
        src, lst, directions, bank, rnd, idx, arrays["kinds"], arrays["wall_a"], arrays["wall_delta"],
        arrays["wall_z"], arrays["z_values"], arrays["box_center"], arrays["box_axis_u"], arrays["box_axis_v"],
        arrays["box_half"], arrays["box_z"], arrays["normals"], arrays["bvh_bounds_min"], arrays["bvh_bounds_max"],
        arrays["bvh_start"], arrays["bvh_count"], arrays["bvh_escape"], arrays["bvh_primitives"], use_bvh,
        arrays["reflection"], arrays["scattering"], arrays["corners"], float(arrays["height"]), B, num_bins,
        bin_dur, c, duration * c, direct_delay, 0.1, 0.1, 1.0, 100.0, np.asarray(forward, dtype=float),
        float(emitter["dipole_weight"]), float(emitter["dipole_power"]), R, 1, bool(trace.get("ambisonics", False)))
    (echogram, ambisonic, hits, contrib, energy, actual, active, vhp, vsurf, vray, vord, vdist, vgain) = res
    return {
        "echogram": echogram, "ambisonic": ambisonic, "hit_counts": hits, "contrib_counts": contrib,
        "surface_energy": energy, "actual_bounces": int(actual), "active_ray_count": int(active),
        "ray_surfaces": vsurf.astype(np.int16), "num_bins": num_bins, "direct_delay": direct_delay,
        # visual-candidate slots with one slot per ray: every ray's strongest contribution, and
        # the hit points of the first VISUAL_POINT_RAYS rays
        "visual_rays": vray.astype(np.int32), "visual_orders": vord.astype(np.int32),
        "visual_distances": vdist, "visual_gains": vgain,
        "visual_hit_points": vhp[:VISUAL_POINT_RAYS],
        "source_forward": np.asarray(forward), "dipole_weight": float(emitter["dipole_weight"]),
        "dipole_power": float(emitter["dipole_power"]),
    }


def cases():
    sys.path.insert(0, str(REPO))
    from acoustic_agent_b200 import workloads  # noqa: E402

    mats = workloads._uniform_materials()
    out = []
    cfg0 = workloads.shoebox(1729)
    base0 = {"source": cfg0.sources[0], "listener": cfg0.listeners[0], "rays": 10000, "bounces": 50, "seed": 1729,
             "duration": 1.0, "bin_dur": 0.01}
    out.append(("shoebox_linear", cfg0.spec, dict(base0, backend="linear")))
    out.append(("shoebox_bvh", cfg0.spec, dict(base0, backend="bvh")))
    u_corners = [(0.0, 0.0), (6.0, 0.0), (6.0, 4.0), (4.26, 4.0), (4.26, 2.08), (1.74, 2.08), (1.74, 4.0), (0.0, 4.0)]
    out.append(("u_room_kat", {"corners": u_corners, "height": 2.8, "materials": mats},
                {"source": (0.8, 3.2, 1.4), "listener": (5.2, 3.2, 1.4), "rays": 512, "bounces": 12, "seed": 4107,
                 "duration": 0.4, "bin_dur": 0.01, "backend": "linear", "ambisonics": True}))
    circle = [(4.0 + math.cos(2 * math.pi * i / 24) * 4.0, 3.0 + math.sin(2 * math.pi * i / 24) * 3.0) for i in range(24)]
    out.append(("circle24_bvh", {"corners": circle, "height": 2.8, "materials": mats},
                {"source": (1.0, 3.0, 1.4), "listener": (7.0, 3.0, 1.4), "rays": 256, "bounces": 6, "seed": 1729,
                 "duration": 0.3, "bin_dur": 0.01, "backend": "bvh"}))
    cfg1 = workloads.u_furnished(1729, rays=2048)
    base1 = {"source": cfg1.sources[0], "listener": cfg1.listeners[0], "rays": 2048, "bounces": 100, "seed": 1729,
             "duration": 2.0, "bin_dur": 0.001, "source_model": "cardioid"}
    out.append(("u_furnished_bvh", cfg1.spec, dict(base1, backend="bvh")))
    out.append(("u_furnished_linear", cfg1.spec, dict(base1, backend="linear", rays=512)))
    objects = [
        {"type": "table", "size": [1.6, 0.9, 0.75], "position": [2.0, 2.0], "rotation": 30.0},
        {"type": "sanitary_fixture", "size": [0.8, 0.6, 0.9], "position": [5.5, 1.2], "rotation": 10.0, "z": 0.45},
        {"type": "structural_element", "size": [0.5, 0.5, 3.0], "position": [4.0, 3.8], "rotation": 45.0, "z": 1.5},
        {"type": "cabinet", "size": [1.2, 0.5, 2.0], "position": [6.3, 4.2], "rotation": 75.0},
        {"type": "cabinet", "size": [0.9, 0.9, 0.9], "position": [1.0, 4.2], "rotation": 0.0},
        {"type": "cabinet", "size": [0.5, 0.5, 0.5], "position": [9.0, 9.0], "rotation": 0.0},
    ]
    out.append(("objects_mix_bvh", {"corners": [(0, 0), (7, 0), (7, 5), (0, 5)], "height": 3.0, "materials": mats,
                                    "objects": objects},
                {"source": (3.5, 1.0, 1.2), "listener": (1.5, 3.5, 1.6), "rays": 1024, "bounces": 30, "seed": 11,
                 "duration": 0.5, "bin_dur": 0.01, "backend": "bvh", "source_model": "cardioid"}))
    apt = workloads.apartment(7, rooms=3, objects_per_room=(3, 6), rays=2048, bounces=60)
    out.append(("apartment3_bvh", apt.spec,
                {"source": apt.sources[0], "listener": apt.listeners[0], "rays": 2048, "bounces": 60, "seed": 7,
                 "duration": 1.0, "bin_dur": 0.01, "backend": "bvh"}))
    rect = [(0.0, 0.0), (6.0, 0.0), (6.0, 4.0), (0.0, 4.0)]
    out.append(("foa_single_ray", {"corners": rect, "height": 2.8, "materials": mats},
                {"source": (4.0, 2.0, 1.4), "listener": (1.0, 1.0, 1.4), "rays": 1, "bounces": 12, "seed": 0,
                 "duration": 1.0, "bin_dur": 0.01, "backend": "linear", "ambisonics": True}))
    open_walls = [{"a": [0, 0], "b": [6, 0], "type": "wall"}, {"a": [6, 0], "b": [6, 4], "type": "wall"},
                  {"a": [6, 4], "b": [0, 4], "type": "door", "z_min": 0.0, "z_max": 2.1}]
    for backend in ("linear", "bvh"):
        out.append((f"open_room_{backend}", {"corners": rect, "height": 3.0, "materials": mats,
                                             "surface_segments": open_walls,
                                             "objects": [{"type": "cabinet", "size": [0.6, 0.6, 1.0],
                                                          "position": [3.0, 2.0], "rotation": 20.0}]},
                    {"source": (4.5, 1.0, 1.5), "listener": (2.0, 1.5, 1.5), "rays": 512, "bounces": 20, "seed": 5,
                     "duration": 0.5, "bin_dur": 0.01, "backend": backend}))
    return out


BANDS = ("125", "250", "500", "1000", "2000", "4000")
DESIGN_CASES = ((16000, 1729, (1.2, 1.0, 0.9, 0.8, 0.6, 0.4)), (48000, 7, (0.5, 0.5, 0.45, 0.4, 0.35, 0.3)),
                (8000, 81, (1.2, 0.0, 0.9, 0.05, 0.6, 2.5)))
RENDER_CASES = (
    ("basic", {"rt60": (1.2,) * 6}, {}),
    ("breakpoint", {"rt60": (1.0, 0.9, 0.8, 0.8, 0.7, 0.6),
                    "profiles": {"125": {"model": "double_slope", "transition_time_s": 0.2,
                                         "selected_target_source": "fitted_late_slope"},
                                 "250": {"model": "double_slope", "transition_time_s": 0.15,
                                         "selected_target_source": "steam_single_slope"}}}, {}),
    ("zero_band", {"rt60": (1.2, 0.9, 0.0, 0.05, 0.6, 0.4)}, {}),
    ("disabled", {"rt60": (1.2,) * 6}, {"late_tail": False}),
)


def late_reverb_golden(steam_rt, SimConfig) -> None:
    """FDN design, FDN impulse and the hybrid late-tail render (steam_rt.py:2235-2640)."""
    out = {}
    for k, (fs, seed, rt60) in enumerate(DESIGN_CASES):
        delays = steam_rt._steam_fdn_delays(fs, seed)
        absorptive, tone = steam_rt._steam_fdn_filter_coefficients(delays, dict(zip(BANDS, rt60)), fs)
        out[f"design{k}_meta"] = np.asarray([fs, seed, *rt60], dtype=np.float64)
        out[f"design{k}_delays"] = delays
        out[f"design{k}_absorptive"] = absorptive
        out[f"design{k}_tone"] = tone
    # the network alone, at 8 kHz with the third design (a zero and a short RT60 band)
    allpass = np.asarray((225, 341, 441, 556), dtype=np.int64)
    out["impulse"] = steam_rt._fdn_impulse_kernel_jit(out["design2_delays"], out["design2_absorptive"], 6000,
                                                      allpass, out["design2_tone"])
    fs, N = 8000, 4000
    rng = np.random.default_rng(81)
    env = np.exp(-3.0 * math.log(10.0) * (np.arange(N, dtype=np.float64) / fs) / 1.2)
    traced = np.vstack([rng.uniform(-1.0, 1.0, N) * env for _ in BANDS]).astype(np.float32)
    out["render_traced"] = traced
    for name, case, overrides in RENDER_CASES:
        cfg = SimConfig(fs=fs, duration_s=N / fs, hybrid_transition_s=0.3, hybrid_overlap_fraction=0.25, seed=1729,
                        **overrides)
        rendered, fdn, meta = steam_rt._render_parametric_fdn_late_reverb(
            traced, {"bin_duration_s": 0.01}, dict(zip(BANDS, case["rt60"])), cfg,
            decay_profiles=case.get("profiles"))
        out[f"render_{name}_out"] = rendered
        out[f"render_{name}_fdn"] = fdn
        out[f"render_{name}_meta"] = np.asarray(json.dumps(meta))
        out[f"render_{name}_case"] = np.asarray(json.dumps({"rt60": case["rt60"], "profiles": case.get("profiles"),
                                                            **overrides}))
    np.savez_compressed(HERE / "late_reverb.npz", **out)


DIRECT_SCENES = ("shoebox_linear", "u_furnished_bvh", "objects_mix_bvh", "apartment3_bvh", "open_room_bvh")
DIRECT_CONFIGS = (
    ("volumetric", {}),
    ("raycast", {"direct_occlusion_mode": "raycast"}),
    ("wide_opaque", {"direct_occlusion_samples": 45, "direct_occlusion_radius_m": 0.4, "direct_transmission": False,
                     "num_transmission_rays": 2}),
)


def direct_golden(steam_rt, models, SimConfig) -> None:
    """simulate_direct (steam_rt.py:1315-1350) on seeded source/listener pairs of five golden scenes."""
    out = {}
    for name in DIRECT_SCENES:
        g = np.load(HERE / f"{name}.npz")
        spec = json.loads(str(g["spec_json"]))
        trace = json.loads(str(g["trace_json"]))
        scene, _ = reference_arrays(steam_rt, models, spec)
        corners = np.asarray(spec["corners"], dtype=float)
        lo, hi = corners.min(axis=0), corners.max(axis=0)
        rng = np.random.default_rng(31)
        pairs = [(trace["source"], trace["listener"])]
        for _ in range(15):
            a = np.r_[rng.uniform(lo, hi), rng.uniform(0.3, float(spec["height"]) - 0.3)]
            b = np.r_[rng.uniform(lo, hi), rng.uniform(0.3, float(spec["height"]) - 0.3)]
            pairs.append((a, b))
        pairs = np.asarray(pairs, dtype=float)
        out[f"{name}_pairs"] = pairs
        out[f"{name}_names"] = np.asarray([str(srf.name) for srf in scene.surfaces])
        out[f"{name}_transmission"] = np.stack([np.asarray(srf.transmission, dtype=float) for srf in scene.surfaces])
        for label, overrides in DIRECT_CONFIGS:
            cfg = SimConfig(**overrides)
            res = [steam_rt.simulate_direct(scene, p[0], p[1], cfg, "cardioid") for p in pairs]
            out[f"{name}_{label}_occlusion"] = np.asarray([r["occlusion"] for r in res])
            out[f"{name}_{label}_transmission"] = np.stack([np.asarray(r["transmission"], dtype=float) for r in res])
            out[f"{name}_{label}_surface"] = np.asarray([r["occlusion_surface"] or "" for r in res])
            out[f"{name}_{label}_gains"] = np.asarray([[r["band_gains"][b] for b in BANDS] for r in res])
    for count in (32, 45):
        out[f"sphere_samples_{count}"] = steam_rt._sphere_volume_samples(count)
    out["configs_json"] = np.asarray(json.dumps({label: {k: getattr(SimConfig(**o), k) for k in (
        "direct_occlusion", "direct_occlusion_mode", "direct_occlusion_radius_m", "direct_occlusion_samples",
        "direct_transmission", "num_transmission_rays", "min_distance_m", "c")} for label, o in DIRECT_CONFIGS}))
    np.savez_compressed(HERE / "direct.npz", **out)


RT60_CASES = (("shoebox_linear", 0.01), ("u_furnished_bvh", 0.001), ("apartment3_bvh", 0.01),
              ("objects_mix_bvh", 0.01))


def rt60_golden(steam_rt, SimConfig) -> None:
    """estimate_reverb_times (steam_rt.py:2727-2742) on golden echograms, as float64 and as float32."""
    out = {}
    cfg = SimConfig()
    for name, bin_dur in RT60_CASES:
        echogram = np.load(HERE / f"{name}.npz")["echogram"]
        for label, e in (("f64", echogram.astype(np.float64)), ("f32", echogram.astype(np.float32))):
            field = {"echogram": e, "bin_duration_s": bin_dur, "num_bins": e.shape[1]}
            rt = steam_rt.estimate_reverb_times(field, cfg)
            out[f"{name}_{label}"] = np.asarray([rt[b] for b in BANDS])
        out[f"{name}_bin"] = np.asarray(bin_dur)
    out["speed_of_sound"] = np.asarray(float(cfg.c))
    np.savez_compressed(HERE / "rt60.npz", **out)


BVH_KEYS = ("bounds_min", "bounds_max", "start", "count", "escape", "primitives")


def bvh_golden(reference_path: str) -> None:
    """The reference's build_bvh (bvh.py:8-77) on the seeded inputs of bvh_cases.py."""
    sys.path.insert(0, str(HERE))
    import bvh_cases  # noqa: E402
    import_reference(reference_path)
    from acoustic_agent.bvh import build_bvh  # noqa: E402
    out = {}
    for name in bvh_cases.CASES:
        lo, hi, leaf = bvh_cases.inputs(name)
        tree = build_bvh(lo, hi, leaf_size=leaf)
        for k in BVH_KEYS:
            out[f"{name}_{k}"] = np.asarray(tree[k])
        out[f"{name}_meta"] = np.asarray([tree["node_count"], tree["leaf_count"], tree["max_depth"], tree["leaf_size"]])
    np.savez_compressed(HERE / "bvh.npz", **out)


def main() -> int:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default="/root/reference")
    parser.add_argument("--only", choices=("late_reverb", "direct", "rt60", "bvh"),
                        help="regenerate one fixture file only")
    args = parser.parse_args()
    if args.only == "bvh":
        bvh_golden(args.reference)
        return 0
    steam_rt, models, directivity = import_reference(args.reference)
    if args.only is not None:
        from acoustic_agent.models import SimConfig  # noqa: E402
        if args.only == "late_reverb":
            late_reverb_golden(steam_rt, SimConfig)
        elif args.only == "rt60":
            rt60_golden(steam_rt, SimConfig)
        else:
            direct_golden(steam_rt, models, SimConfig)
        return 0
    written = []
    for name, spec, trace in cases():
        scene, arrays = reference_arrays(steam_rt, models, spec)
        res = run_trace(steam_rt, directivity, arrays, trace)
        payload = {f"array_{k}": np.asarray(arrays[k]) for k in ARRAY_KEYS}
        payload["array_names"] = np.asarray(arrays["names"])
        payload["array_height"] = np.asarray(float(arrays["height"]))
        payload.update({k: v for k, v in res.items() if k != "ambisonic"})
        if trace.get("ambisonics"):
            payload["ambisonic"] = res["ambisonic"]
        payload["spec_json"] = np.asarray(json.dumps(spec))
        payload["trace_json"] = np.asarray(json.dumps(trace))
        np.savez_compressed(HERE / f"{name}.npz", **payload)
        written.append(name)
        print(name, "surfaces", len(arrays["names"]), "energy", float(np.sum(res["echogram"])),
              "active", res["active_ray_count"], "bounces", res["actual_bounces"])

    # Band synthesis: reconstruct_band_irs on float64 and float32 echograms.
    from acoustic_agent.models import SimConfig  # noqa: E402
    shoe = np.load(HERE / "shoebox_linear.npz")
    furnished = np.load(HERE / "u_furnished_bvh.npz")
    synth = {}
    for label, echogram, fs, bin_dur, delay, seed in (
        ("shoebox_f64", shoe["echogram"], 16000, 0.01, float(shoe["direct_delay"]), 1729),
        ("shoebox_f32", shoe["echogram"].astype(np.float32), 16000, 0.01, float(shoe["direct_delay"]), 1729),
        ("furnished_f32", furnished["echogram"][:, :500].astype(np.float32), 48000, 0.001,
         float(furnished["direct_delay"]), 1729),
    ):
        field = {"echogram": echogram, "num_bins": echogram.shape[1], "bin_duration_s": bin_dur,
                 "direct_delay_s": delay}
        cfg = SimConfig(fs=fs, seed=seed)
        synth[f"{label}_input"] = echogram
        synth[f"{label}_output"] = steam_rt.reconstruct_band_irs(field, cfg)
        synth[f"{label}_meta"] = np.asarray([fs, bin_dur, delay, seed], dtype=np.float64)
    np.savez_compressed(HERE / "synthesis.npz", **synth)

    # Random workspace pins.
    rnd, idx = steam_rt._diffuse_random_sequence(1000, 5, 128, 1729)
    np.savez_compressed(HERE / "workspace.npz", sphere=steam_rt._sphere_samples(1000, 1729),
                        bank=steam_rt._diffuse_sample_bank(128), random=rnd, indices=idx)
    late_reverb_golden(steam_rt, SimConfig)
    direct_golden(steam_rt, models, SimConfig)
    rt60_golden(steam_rt, SimConfig)
    bvh_golden(args.reference)
    print("wrote", written, "synthesis", "workspace", "late_reverb", "direct", "rt60", "bvh")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
