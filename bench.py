#!/usr/bin/env python
"""Adaptation-round throughput on B200: adapted triangles per second per full
round (trinity's refine + coarsen + swap + smooth, graph heuristics and
topology repairs included), on the 2M-triangle unit-square workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step = one full adaptation of a fresh copy of the workload: the mesh is
restored on the device from its resident input (no host transfer), the metric
is recovered, then 3 rounds run. ``value`` = sum over rounds of the live
triangles at round start / sum of the rounds' device times (CUDA events on
the library's stream; the metric stage is excluded, as in the reference's
per-kernel Stats). ``e2e`` runs the same adaptation through the C ABI from
host arrays (load, metric, 3 rounds, export) with the transfers inside the
timed region. Under torchrun each rank adapts its own copy (weak scaling);
times are the max over ranks.

``--impl reference`` times trinity's own OpenMP implementation (built from its
sources into oracle/_ref/, all host cores) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

# many meshes adapt concurrently in the batched workload, one stream each:
# give the device more hardware queues than the default 8 (read at CUDA init)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

from trinity_b200 import meshgen  # noqa: E402

WORKLOAD = "c2"
# DRAM traffic per launch of the kernel that dominates the 2M-triangle step,
# measured with ncu (dram__bytes_read.sum + dram__bytes_write.sum, caches
# flushed before each launch, the 7 class launches of the timed step's first
# pass, default shape: 2 lanes a vertex, tries in one sweep, 128 registers); a
# live run has no hardware counters, so the figure is carried here
MEASURED_TRAFFIC = {"smooth_move": 410.3e6}
METRIC = "adapted triangles/s per full round"
UNIT = "triangles/s"
REF_BIN = os.path.join(REPO, "oracle", "_ref", "trinity_ref")


def workload_config(grid=None):
    m, u, c = meshgen.make_config(WORKLOAD, grid)
    cfg = {
        "workload": "unit square 1000x1000 grid, 1,002,001 vertices / 2,000,000 triangles, "
                    "interior jitter 0.2h (seed 2), field tanh+gauss+waves, target 0.7, "
                    "L^2 norm, depth 2, bucket 128, 3 rounds",
        "data": "synthetic, generated by trinity_b200/meshgen.py",
        "l2": "working set larger than L2 (mesh restored every step)",
    }
    if grid:
        cfg["workload"] = f"unit square {grid}x{grid} grid (profiling size), otherwise as the 2M-triangle workload"
    return m, u, c, cfg


def tags_of(m):
    t = np.zeros(m.nb_nodes, dtype=np.uint8)
    t[m.edges.ravel()] = 4
    t[m.corners] = 12
    return t


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def run_step(api, g, c, heur, kern, graph=False):
    """One adaptation on a mesh already holding the input; returns
    (sum of live triangles at round starts, sum of round device ms, metric ms).
    graph: each round as the mesh's captured CUDA graph."""
    api.Metrics(g, c["target"], c["norm"]).run()
    metric_ms = g.last_time_ms()
    tin, tms = 0, 0.0
    for _ in range(c["rounds"]):
        tin += g.counts()[3]
        if graph:
            g.round_graph(c["depth"])
            tms += g.last_time_ms()
            continue
        for k in kern:
            k.run()
            tms += g.last_time_ms()
    return tin, tms, metric_ms


def b200_arm(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from trinity_b200 import _lib, api

    torch.cuda.set_device(local_rank)
    dist_on = world > 1
    m, u, c, cfg = workload_config(args.grid)
    tags = tags_of(m)
    g = api.Mesh((m.nb_nodes, m.nb_elems), c["bucket"], c["depth"], 0, c["rounds"])
    g.load_arrays(m.points, m.tris, tags, u)
    g.set_options(seed=0x7472696E697479 + rank)
    heur = api.Partit(g, 8)
    kern = [api.Refine(g, c["depth"]), api.Coarse(g, heur), api.Swap(g), api.Smooth(g, heur, c["depth"])]
    tuned = g.get_tune() if args.no_tune else g.autotune(c["target"], c["norm"], depth=c["depth"], rounds=1)

    def barrier():
        if dist_on:
            dist.barrier()

    for _ in range(args.warmup):
        g.reload()
        run_step(api, g, c, heur, kern)
    torch.cuda.synchronize()

    # ---- per-kernel breakdown: untimed steps with every launch bracketed by
    # CUDA events (the events cost ~9 % of throughput, so they stay out of
    # the timed region except around the dominant kernel) ----
    _lib.profile_enable(True)
    _lib.profile_count_bytes(True, g.capacity()[0])
    for _ in range(min(args.steps, 2)):
        g.reload()
        run_step(api, g, c, heur, kern)
    prof_all = _lib.profile_read()
    _lib.profile_count_bytes(False)
    _lib.profile_enable(False)
    dom_name = max(prof_all, key=lambda r: r["ms"])["kernel"] if prof_all else None

    # ---- timed region (device-resident input); CUDA events around the
    # dominant kernel's launches only ----
    _lib.profile_only(dom_name)
    _lib.profile_enable(True)
    launches0 = _lib.launch_count()
    tin_sum, tms_sum, metric_ms = 0, 0.0, []
    barrier()
    torch.cuda.synchronize()
    with Clocks(torch.cuda.current_device()) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            g.reload()
            tin, tms, mms = run_step(api, g, c, heur, kern)
            tin_sum += tin
            tms_sum += tms
            metric_ms.append(mms)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    barrier()
    launches = _lib.launch_count() - launches0
    prof = _lib.profile_read()
    _lib.profile_enable(False)
    _lib.profile_only(None)
    final = g.counts()

    # ---- the mixed-precision form on the same workload (reported beside) ----
    forms = {}
    if not args.no_forms:
        g.set_precision("mixed")
        # launch shapes chosen again for the FP32 arithmetic (same results)
        mixed_tune = tuned if args.no_tune else g.autotune(c["target"], c["norm"], depth=c["depth"], rounds=1)
        for _ in range(args.warmup):
            g.reload()
            run_step(api, g, c, heur, kern)
        m_tin, m_tms = 0, 0.0
        torch.cuda.synchronize()
        for _ in range(args.steps):
            g.reload()
            tin, tms, _ = run_step(api, g, c, heur, kern)
            m_tin += tin
            m_tms += tms
        q = g.quality_stats()
        forms["mixed_fp32"] = {"tri_in": m_tin, "round_ms": m_tms,
                               "final_mesh": {"nodes": g.counts()[2], "triangles": g.counts()[3]},
                               "quality_min_max_mean": [round(x, 4) for x in q],
                               "launch_shapes": mixed_tune}
        g.set_precision("fp64")
        g.set_tune(tuned)
        g.reload()
        run_step(api, g, c, heur, kern)
        forms["fp64_quality_min_max_mean"] = [round(x, 4) for x in g.quality_stats()]
        for prec in ("fp64", "mixed"):
            g.set_precision(prec)
            g.set_tune(tuned if prec == "fp64" else mixed_tune)
            g.reload()
            run_step(api, g, c, heur, kern, graph=True)       # captures the round
            gt, gm = 0, 0.0
            for _ in range(args.steps):
                g.reload()
                tin, tms, _ = run_step(api, g, c, heur, kern, graph=True)
                gt += tin
                gm += tms
            forms[f"graph_{prec}"] = {"tri_in": gt, "round_ms": gm,
                                      "quality_min_max_mean": [round(x, 4) for x in g.quality_stats()]}
        g.set_precision("fp64")
        g.set_tune(tuned)
        if rank == 0:
            forms["adjoint"] = adjoint_form(args)
            forms["precision"] = precision_form(args)

    # ---- end-to-end through the C ABI from pinned host buffers ----
    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()

    pts = pinned(m.points.shape, torch.float64)
    pts[:] = m.points
    tris = pinned(m.tris.shape, torch.int32)
    tris[:] = m.tris
    tags_p = pinned(tags.shape, torch.uint8)
    tags_p[:] = tags
    u_p = pinned(u.shape, torch.float64)
    u_p[:] = u
    cap_v, cap_t = 2 * m.nb_nodes, 2 * m.nb_elems
    out = (pinned((cap_v, 2), torch.float64), pinned((cap_t, 3), torch.int32), pinned((cap_v, 3), torch.float64))
    e2e_tin, e2e_t, d2h = 0, 0.0, 0
    h2d = pts.nbytes + tris.nbytes + tags_p.nbytes + u_p.nbytes
    barrier()
    torch.cuda.synchronize()
    for _ in range(0 if args.no_e2e else args.steps):
        t0 = time.perf_counter()
        g.load_arrays(pts, tris, tags_p, u_p)
        tin, _, _ = run_step(api, g, c, heur, kern)
        res = g.export_compact(out=out)
        e2e_t += time.perf_counter() - t0
        e2e_tin += tin
        d2h = sum(a.nbytes for a in res)

    from trinity_b200.dist import reduce_stats
    agg = reduce_stats([tin_sum, tms_sum, wall, e2e_tin, e2e_t], [0, 3], [1, 2, 4],
                       device="cuda" if dist_on else "cpu")
    tin_all, tms_max, wall_max, e2e_tin_all, e2e_max = agg.tolist()
    if rank != 0:
        return None

    value = tin_all / (tms_max / 1e3)
    dom = max(prof, key=lambda r: r["ms"]) if prof else None
    roofline = None
    peaks = {}
    pk = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    if dom:
        # algorithmic bytes per launch: counted on the device in the profiled
        # steps (the same deterministic launches as the timed ones); the time
        # per launch from the timed steps' events
        dom_all = next(r for r in prof_all if r["kernel"] == dom["kernel"])
        per_launch_bytes = dom_all["bytes"] / max(dom_all["launches"], 1)
        per_launch_s = dom["ms"] / max(dom["launches"], 1) / 1e3
        achieved = per_launch_bytes / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
        roofline = {"kernel": dom["kernel"], "bound": "hbm", "achieved": round(achieved, 2),
                    "peak": hbm_peak, "peak_source": "measured" if peaks else "fallback",
                    "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                    "traffic": MEASURED_TRAFFIC.get(dom["kernel"]) if not args.grid else None,
                    "traffic_note": "DRAM read + write bytes per launch, ncu on this workload, caches flushed "
                                    "before each launch (mean of the 7 class launches of the timed step's "
                                    "first pass)",
                    "launches": dom["launches"],
                    "avg_launch_us": round(per_launch_s * 1e6, 2),
                    "algorithmic_bytes_per_launch": round(per_launch_bytes),
                    "bytes_source": "counted on the device (distinct entries per launch)"
                    if dom_all.get("bytes_counted") else "launcher's model",
                    "share_of_kernel_time": round(
                        sum(r["ms"] for r in prof_all if r["kernel"] == dom["kernel"])
                        / sum(r["ms"] for r in prof_all), 3),
                    "timing": "CUDA events on the library stream around this kernel's launches "
                              "during the timed steps; share from the profiled steps before"}
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(wall_max / args.steps * 1e3, 3),
        "round_ms_per_step": round(tms_max / args.steps, 3),
        "metric_ms_per_step": round(float(np.mean(metric_ms)), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "mode": "free (GPU heuristics)", "config": cfg,
        "e2e": {"value": round(e2e_tin_all / e2e_max, 1) if e2e_max > 0 else None, "unit": UNIT,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "note": "pinned host arrays -> C ABI load, metric, 3 rounds, compact export of the "
                        "adapted mesh (points, triangles, metric) into pinned host arrays; wall clock"},
        "gpu_launches": int(launches),
        "roofline": roofline,
        "kernels": sorted(({"kernel": r["kernel"], "launches": r["launches"], "ms": round(r["ms"], 3),
                            "gbs": round(r["bytes"] / (r["ms"] / 1e3) / 1e9, 1) if r["ms"] > 0 else None,
                            "bytes": "counted" if r.get("bytes_counted") else "model"}
                           for r in prof_all), key=lambda r: -r["ms"]),
        "kernels_note": f"{min(args.steps, 2)} profiled steps (every launch timed), before the timed region",
        "final_mesh": {"nodes": final[2], "triangles": final[3]},
        "launch_shapes": dict(tuned, chosen_by="defaults (--no-tune)" if args.no_tune
                              else "trn_autotune on this mesh (changes no result)"),
        "clocks": clk.summary(),
    }
    if "mixed_fp32" in forms:
        f = forms["mixed_fp32"]
        mixed = reduce_stats([f["tri_in"], f["round_ms"]], [0], [1], device="cuda" if dist_on else "cpu")
        line["forms"] = {
            "mixed_fp32": {"value": round(mixed[0] / (mixed[1] / 1e3), 1), "unit": UNIT,
                           "round_ms_per_step": round(mixed[1] / args.steps, 3),
                           "dtype": "f32 metric arithmetic, f64 coordinates/orientation",
                           "final_mesh": f["final_mesh"], "quality_min_max_mean": f["quality_min_max_mean"]},
            "fp64_quality_min_max_mean": forms["fp64_quality_min_max_mean"],
        }
        for prec in ("fp64", "mixed"):
            f = forms[f"graph_{prec}"]
            gg = reduce_stats([f["tri_in"], f["round_ms"]], [0], [1], device="cuda" if dist_on else "cpu")
            line["forms"][f"graph_{prec}"] = {
                "value": round(gg[0] / (gg[1] / 1e3), 1), "unit": UNIT,
                "round_ms_per_step": round(gg[1] / args.steps, 3),
                "note": "each round one captured CUDA graph (loops as device-decided loop nodes)",
                "quality_min_max_mean": f["quality_min_max_mean"]}
        for k in ("adjoint", "precision"):
            if k in forms:
                line["forms"][k] = forms[k]
    return line


# ------------------------------------------------------------------ precision
def _metric_lengths(pts, tri, ten):
    """metric length of every undirected edge (numeric.cpp:469-497), numpy FP64"""
    e = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]])
    e = np.unique(np.sort(e, axis=1), axis=0)
    w = pts[e[:, 1]] - pts[e[:, 0]]

    def quad(t):
        return np.sqrt(w[:, 0] * (t[:, 0] * w[:, 0] + t[:, 1] * w[:, 1])
                       + w[:, 1] * (t[:, 1] * w[:, 0] + t[:, 2] * w[:, 1]))
    l0, l1 = quad(ten[e[:, 0]]), quad(ten[e[:, 1]])
    lo, hi = np.minimum(l0, l1), np.maximum(l0, l1)
    r = hi / lo
    with np.errstate(divide="ignore", invalid="ignore"):
        geo = hi * (r - 1) / (r * np.log(r))
    return np.where(np.abs(l0 - l1) < 1e-9, l0, geo)


def tensor_error(t32, t64):
    """per vertex, |T32 - T64| / max |T64| over the components (m11, m12,
    m22): median, RMS, 99th percentile, max, and the fraction above 1e-5"""
    e = np.abs(t32 - t64).max(axis=1) / np.maximum(np.abs(t64).max(axis=1), 1e-300)
    return {"rel_err_median": float(np.median(e)), "rel_err_rms": float(np.sqrt(np.mean(e ** 2))),
            "rel_err_p99": float(np.percentile(e, 99)), "rel_err_max": float(e.max()),
            "fraction_above_1e-5": round(float(np.mean(e > 1e-5)), 6)}


def precision_form(args):
    """The mixed-precision form on the ~4M-triangle mesh (1414x1414 grid,
    jitter 0.2h, multi-feature field, depth 2): (1) one smoothing pass from
    the same FP64 state in both forms -> max / RMS relative error of the
    smoothed coordinates' displacement and of the tensors; (2) full 3-round
    adaptations in both forms -> throughput, final counts and the histogram
    of edge lengths in the metric."""
    import torch
    from trinity_b200 import api
    m, u, c = meshgen.make_config("c3", args.grid)
    tags = tags_of(m)
    out = {"workload": f"unit square {m.nb_nodes} vertices / {m.nb_elems} triangles, jitter 0.2h "
                       "(seed 3), field tanh+gauss+waves, target 0.7, L^2, depth 2, bucket 128"}
    # (0) the metric recovery itself in both forms, from the same input
    rec = {}
    for prec in ("fp64", "mixed"):
        g = api.Mesh((m.nb_nodes, m.nb_elems), c["bucket"], c["depth"], 0, c["rounds"])
        g.load_arrays(m.points, m.tris, tags, u)
        g.set_precision(prec)
        api.Metrics(g, c["target"], c["norm"]).run()
        rec[prec] = (g.export()[1], g.last_time_ms())
        g.close()
    out["metric_recovery"] = dict(tensor_error(rec["mixed"][0], rec["fp64"][0]),
                                  ms_fp64=round(rec["fp64"][1], 3), ms_mixed=round(rec["mixed"][1], 3),
                                  note="Metrics::run from the same input: FP32 patch means (FP64 coordinate "
                                       "and value differences), FP32 eigen-clamp and scalings, FP64 "
                                       "complexity sum, against the FP64 form (itself the oracle's "
                                       "tensors to the last bits)")
    gs = {}
    for prec in ("fp64", "mixed"):
        g = api.Mesh((m.nb_nodes, m.nb_elems), c["bucket"], c["depth"], 0, c["rounds"])
        g.load_arrays(m.points, m.tris, tags, u)
        heur = api.Partit(g, 8)
        api.Metrics(g, c["target"], c["norm"]).run()
        api.Refine(g, c["depth"]).run()
        api.Coarse(g, heur).run()
        api.Swap(g).run()
        gs[prec] = (g, heur)
    p0 = gs["fp64"][0].export()[0]
    res = {}
    for prec, (g, heur) in gs.items():
        g.set_precision(prec)
        api.Smooth(g, heur, c["depth"]).run()
        pts, ten, tri, alive, _ = g.export()
        res[prec] = (pts, ten, alive)
    (p64, t64, a64), (p32, t32, a32) = res["fp64"], res["mixed"]
    live = a64.astype(bool)
    d64 = np.linalg.norm(p64[live] - p0[live], axis=1)
    moved = d64 > 0
    derr = np.linalg.norm(p32[live] - p64[live], axis=1)[moved] / d64[moved]
    terr = (np.abs(t32[live] - t64[live]) / np.maximum(np.abs(t64[live]).max(axis=1, keepdims=True), 1e-300))
    flip = derr > 1e-3     # a different accept / back-off decision, not rounding
    same = np.ones(live.sum(), bool)
    same[np.flatnonzero(moved)[flip]] = False
    out["same_state_smoothing_pass"] = {
        "vertices_moved_fp64": int(moved.sum()),
        "decision_differs_fraction": round(float(flip.mean()), 6) if derr.size else 0.0,
        "displacement_rel_err_rms_same_decision": float(np.sqrt(np.mean(derr[~flip] ** 2))) if derr.size else 0.0,
        "displacement_rel_err_max_same_decision": float(derr[~flip].max()) if derr.size else 0.0,
        "displacement_rel_err_max": float(derr.max()) if derr.size else 0.0,
        "displacement_rel_err_rms": float(np.sqrt(np.mean(derr ** 2))) if derr.size else 0.0,
        "displacement_rel_err_median": float(np.median(derr)) if derr.size else 0.0,
        "tensor_rel_err_max": float(terr.max()), "tensor_rel_err_rms": float(np.sqrt(np.mean(terr ** 2))),
        "tensor_same_decision": tensor_error(t32[live][same], t64[live][same]),
        "note": "same FP64 state (recovered in FP64), same coloring, only the smoothing pass in FP32; "
                "tensor errors relative to each tensor's largest component"}
    for prec, (g, _) in gs.items():
        g.close()
    bins = np.concatenate([np.linspace(0, 3, 31), [np.inf]])
    hists = {}
    for prec in ("fp64", "mixed"):
        g = api.Mesh((m.nb_nodes, m.nb_elems), c["bucket"], c["depth"], 0, c["rounds"])
        g.load_arrays(m.points, m.tris, tags, u)
        g.set_precision(prec)
        heur = api.Partit(g, 8)
        kern = [api.Refine(g, c["depth"]), api.Coarse(g, heur), api.Swap(g), api.Smooth(g, heur, c["depth"])]
        run_step(api, g, c, heur, kern)
        g.reload()
        torch.cuda.synchronize()
        tin, tms, _ = run_step(api, g, c, heur, kern)
        pts, tri, ten = g.export_compact()
        ln = _metric_lengths(pts, tri, ten)
        h, _ = np.histogram(ln, bins=bins)
        hists[prec] = h / h.sum()
        out[prec] = {"value": round(tin / (tms / 1e3), 1), "unit": UNIT, "round_ms": round(tms, 3),
                     "final_triangles": int(tri.shape[0]),
                     "edges_in_unit_range": round(float(np.mean((ln >= 2 ** -0.5) & (ln <= 2 ** 0.5))), 4),
                     "quality_min_max_mean": [round(x, 4) for x in g.quality_stats()]}
        g.close()
    out["histogram_bins"] = "metric edge length, 30 bins on [0, 3] + overflow"
    out["histogram_l1_fp32_vs_fp64"] = round(float(np.abs(hists["mixed"] - hists["fp64"]).sum()), 5)
    out["speedup_mixed_vs_fp64"] = round(out["mixed"]["value"] / out["fp64"]["value"], 3)
    return out


# ------------------------------------------------------------------ files
def io_form():
    """Reading the workload's files (87 MB .mesh, 20 MB .bb): the host-side
    text parse (one thread per chunk of each section), the whole load onto
    the device (parse, copies, stencils and adjacency), and the same from the
    binary sidecar; best of three. The reference's Mesh::load on the same
    files is timed by the CPU-baseline runs of the same process."""
    import torch
    from trinity_b200 import api
    mp, bp = ensure_files()
    m_n, m_e = api.find("Vertices", mp), api.find("Triangles", mp)

    def best(fn):
        t = 1e300
        for _ in range(3):
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            t = min(t, time.perf_counter() - t0)
        return round(t * 1e3, 1)
    out = {"files_mb": round((os.path.getsize(mp) + os.path.getsize(bp)) / 1e6, 1),
           "host_threads": os.cpu_count()}
    # one parse into arrays already sized (read_mesh_files parses twice: counts, then values)
    import ctypes
    from trinity_b200 import _lib
    L = _lib.lib()
    nv, nt = ctypes.c_int(m_n), ctypes.c_int(m_e)
    arrs = [np.zeros((m_n, 2)), np.zeros((m_e, 3), np.int32), np.zeros(m_n, np.uint8), np.zeros(m_n)]
    ptrs = [a.ctypes.data_as(ctypes.c_void_p) for a in arrs]
    out["text_parse_ms"] = best(lambda: L.trn_read_mesh_files(mp.encode(), bp.encode(), ctypes.byref(nv),
                                                              ctypes.byref(nt), *ptrs, m_n, m_e))
    g = api.Mesh((m_n, m_e), 128, 2, 0, 3)
    out["text_load_to_device_ms"] = best(lambda: g.load(mp, bp))
    binp = os.path.join(os.path.dirname(mp), "c2.trnb")
    g.store_binary(binp)
    out["binary_load_to_device_ms"] = best(lambda: g.load(binp, bp))
    g.close()
    return out


# ------------------------------------------------------------------ adjoint
def adjoint_form(args):
    """The differentiation form on the 2M-triangle mesh jittered by +-0.3h with
    the multi-feature field: device time of J = sum of element qualities with
    dJ/dxy and dJ/du (through the Hessian recovery) in FP64 and FP32, then 20
    steps of gradient smoothing (log-quality objective, the vertex tensor
    following the move as in the smart Laplacian) against 20 smart-Laplacian
    passes: final min / max / mean quality and device time."""
    import torch
    from trinity_b200 import _lib, api
    m, u, c = meshgen.make_config("c4", args.grid)
    g = api.Mesh((m.nb_nodes, m.nb_elems), 64, 1, 0, 1, capa_scale=2)
    g.load_arrays(m.points, m.tris, tags_of(m), u)
    api.Metrics(g, c["target"], c["norm"]).run()
    ud = torch.tensor(u, dtype=torch.float64, device="cuda")
    margs = dict(target_factor=c["target"], Lp_norm=c["norm"])
    out = {"workload": "unit square 1000x1000 grid, 2,000,000 triangles, jitter 0.3h (seed 4), "
                       "field tanh+gauss+waves, target 0.7, L^2"
           if not args.grid else f"{args.grid}x{args.grid} grid, jitter 0.3h"}
    for prec in ("fp64", "mixed"):
        for _ in range(3):
            g.quality_adjoint(None, ud, precision=prec, **margs)
        _lib.profile_enable(True)
        ms = []
        for _ in range(max(args.steps, 3)):
            J, gxy, gu = g.quality_adjoint(None, ud, precision=prec, **margs)
            ms.append(g.last_time_ms())
        prof = _lib.profile_read()
        _lib.profile_enable(False)
        adj = [r for r in prof if r["kernel"].startswith("adjoint")]
        by = sum(r["bytes"] for r in adj)
        kt = sum(r["ms"] for r in adj)
        out[prec] = {"J": J, "ms_per_gradient": round(float(np.median(ms)), 3),
                     "triangles_per_s": round(m.nb_elems / (float(np.median(ms)) / 1e3), 1),
                     "note": "J + dJ/dxy + dJ/du incl. the metric recovery forward",
                     "adjoint_kernels_gbs": round(by / (kt / 1e3) / 1e9, 1) if kt > 0 else None}
    heur = api.Partit(g, 8)
    for kind in ("gradient", "laplacian"):
        g.reload()
        api.Metrics(g, c["target"], c["norm"]).run()
        q0 = g.quality_stats()
        st = _lib.Stats()
        if kind == "gradient":
            api.GradientSmooth(g, heur, 20).run(st)
        else:
            api.Smooth(g, heur, 20).run(st)
        out[f"smooth_{kind}_20"] = {"ms": round(g.last_time_ms(), 3),
                                    "quality_min_max_mean_before": [round(x, 5) for x in q0],
                                    "quality_min_max_mean_after": [round(x, 5) for x in g.quality_stats()],
                                    "moved": st.task, "tried": st.eval}
    g.close()
    return out


# ------------------------------------------------------------------ batch
def _batch_run(args, rank, world, local_rank, steps, candidates=None):
    """Adapt the batched workload's meshes of this rank concurrently; returns
    the rank-0 summary (aggregate triangles/s, per-mesh round times, the same
    without graphs and one mesh at a time) or None on other ranks."""
    import torch
    from trinity_b200 import api
    from trinity_b200.dist import reduce_stats, shard_meshes

    torch.cuda.set_device(local_rank)
    p = meshgen.BATCH_PARAMS
    items = list(meshgen.batch_meshes())
    mine = shard_meshes([m.nb_elems for m, _, _ in items], world)[rank]
    meshes = []
    for i in mine:
        m, u, _ = items[i]
        g = api.Mesh((m.nb_nodes, m.nb_elems), p["bucket"], p["depth"], 0, p["rounds"],
                     capa_scale=p["capa_scale"])
        g.load_arrays(m.points, m.tris, tags_of(m), u)
        g.set_swap_match(p["swap_match"])
        meshes.append(g)
    threads = args.threads or min(16, os.cpu_count() or 8)
    # launch shapes: one table for the whole batch, chosen by timing the
    # concurrent batch itself (api.batch_autotune: coordinate descent)
    tuned, trials = api.batch_autotune(meshes, p["target"], p["norm"], p["rounds"], p["depth"],
                                       threads=threads, graph=True, candidates=candidates)

    def run(nthreads, graph):
        for g in meshes:
            g.reload()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ms, tin = api.batch_adapt(meshes, p["target"], p["norm"], p["rounds"], p["depth"], threads=nthreads,
                                  graph=graph)
        torch.cuda.synchronize()
        return time.perf_counter() - t0, ms, tin

    for _ in range(args.warmup):          # the first graph round of each mesh captures it
        run(threads, True)
    l0 = _lib_launches()
    wall, tins, mss = 0.0, 0, []
    with Clocks(torch.cuda.current_device()) as clk:
        for _ in range(steps):
            w, ms, tin = run(threads, True)
            wall += w
            tins += int(tin.sum())
            mss.append(ms)
    launches = _lib_launches() - l0
    run(threads, False)
    pw, _, ptin = run(threads, False)
    seq_w, seq_ms, seq_tin = run(1, False)
    dist_on = world > 1
    agg = reduce_stats([tins, wall, int(seq_tin.sum()), seq_w, int(ptin.sum()), pw], [0, 2, 4], [1, 3, 5],
                       device="cuda" if dist_on else "cpu")
    for g in meshes:
        g.close()
    if rank != 0:
        return None
    conc = np.concatenate(mss)
    return {
        "value": round(agg[0] / agg[1], 1), "unit": UNIT, "steps": steps,
        "ms_per_step": round(agg[1] / steps * 1e3, 3),
        "workload": "256 unit-square meshes, side log-uniform in [32, 512] (seed 5), "
                    "shock field tanh(a (y - 0.5 - b sin 2 pi x)), a ~ U[10, 100], b ~ U[0, 0.3], "
                    "target 0.8, L^2, 3 rounds, depth 1, bucket 128, capacity 8x input",
        "how": f"concurrent: one stream per mesh, {threads} host threads, each round one captured "
               "CUDA graph per mesh; wall time of metric + rounds",
        "meshes_on_rank0": len(meshes),
        "gpu_launches": int(launches),
        "launch_shapes": dict(tuned, chosen_by="api.batch_autotune (whole-batch timing, "
                                                "changes no result)", trials_s=trials),
        "concurrent_without_graphs": {"value": round(agg[4] / agg[5], 1), "unit": UNIT},
        "one_at_a_time": {"value": round(agg[2] / agg[3], 1), "unit": UNIT,
                          "note": "per-stage calls, no graphs, one mesh after the other",
                          "round_ms_p50": round(float(np.percentile(seq_ms, 50)), 3),
                          "round_ms_p99": round(float(np.percentile(seq_ms, 99)), 3)},
        "per_mesh_round_ms": {"p50": round(float(np.percentile(conc, 50)), 3),
                              "p99": round(float(np.percentile(conc, 99)), 3)},
        "clocks": clk.summary(),
    }


def batch_arm(args, rank, world, local_rank):
    """The batched workload: 256 unit-square meshes of sides log-uniform in
    [32, 512] (2k-520k triangles), shock fields with random (a, b), target 0.8,
    3 rounds, depth 1; adapted concurrently (one stream per mesh, a pool of
    host threads), each round one captured CUDA graph per mesh, sharded by size
    across ranks. Compared with the same concurrency without graphs and with
    adapting the meshes one at a time with the per-stage calls."""
    r = _batch_run(args, rank, world, local_rank, args.steps)
    if r is None:
        return None
    return {
        "metric": "adapted triangles/s per full round (batch of 256 meshes)", "value": r["value"],
        "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "mode": r["how"],
        "config": {"workload": r["workload"], "meshes_on_rank0": r["meshes_on_rank0"]},
        "gpu_launches": r["gpu_launches"], "launch_shapes": r["launch_shapes"],
        "concurrent_without_graphs": r["concurrent_without_graphs"], "one_at_a_time": r["one_at_a_time"],
        "per_mesh_round_ms": r["per_mesh_round_ms"], "clocks": r["clocks"],
    }


# the batched form inside the default run: a shorter shape search (the
# smoothing block and the grouped-search lanes, the two that moved the batch
# most when the full search ran) and two timed batches
BATCH_FORM_CANDIDATES = {"group_lanes": [8, 16], "smooth_threads": [128, 256]}


def _lib_launches():
    from trinity_b200 import _lib
    return _lib.launch_count()


# ------------------------------------------------------------------ reference
def ensure_files():
    d = os.path.join(tempfile.gettempdir(), "trinity_b200_bench")
    mp, bp = os.path.join(d, f"{WORKLOAD}.mesh"), os.path.join(d, f"{WORKLOAD}.bb")
    if not (os.path.exists(mp) and os.path.exists(bp)):
        meshgen.write_config(WORKLOAD, d)
    return mp, bp


def reference_once(mp, bp, c, threads):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close", OMP_PLACES="cores")
    r = subprocess.run([REF_BIN, mp, bp, str(c["rounds"]), str(c["depth"]), str(c["bucket"]),
                        str(c["target"]), str(c["norm"]), "--capa-depth", "4", "--time"],
                       env=env, capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        raise RuntimeError(f"reference failed: {r.stderr[-400:]}")
    j = json.loads(r.stdout.strip().splitlines()[-1])
    return sum(j["tri_in"]), j["rounds_ms"], j


def physical_cores():
    try:
        import psutil
        n = psutil.cpu_count(logical=False)
        if n:
            return n
    except Exception:
        pass
    return os.cpu_count() or 1


def cpu_baseline():
    """The reference on the host cores: the median of three full adaptations
    of the workload on all physical cores, plus one on a single thread of a
    400 x 400 sample of the same generator (a full single-thread run takes
    about a minute)."""
    _, _, c = meshgen.make_config(WORKLOAD)
    if not os.path.exists(REF_BIN):
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref/trinity_ref not built"}
    mp, bp = ensure_files()
    cores = physical_cores()
    runs = sorted((reference_once(mp, bp, c, cores) for _ in range(3)), key=lambda r: r[0] / r[1])
    tin, ms, j = runs[1]
    d = os.path.join(tempfile.gettempdir(), "trinity_b200_bench")
    smp, sbp, sc = meshgen.write_config(WORKLOAD, d, 400)
    tin1, ms1, _ = reference_once(smp, sbp, sc, 1)
    return {"value": round(tin / (ms / 1e3), 1), "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"median of 3 full adaptations of the workload (metric + 3 rounds; rounds timed: "
                      f"{ms:.0f} ms, metric {j['metric_ms']:.0f} ms, Mesh::load {j.get('load_ms', 0):.0f} ms)",
            "runs_triangles_per_s": [round(r[0] / (r[1] / 1e3), 1) for r in runs],
            "mesh_load_ms": j.get("load_ms"),
            "one_thread": {"value": round(tin1 / (ms1 / 1e3), 1), "unit": UNIT, "cores": 1,
                           "sample": "the same generator at 400 x 400 (320k triangles), 3 rounds"},
            "build": "g++ -O3 -funroll-loops -march=x86-64-v3 (built where the sources are, run on "
                     "this host), OpenMP, NDEBUG",
            "final_mesh": {"nodes": j["nodes_out"], "triangles": j["elems_out"]}}


def reference_arm(args, rank, world):
    if rank != 0:
        return None
    _, _, c = meshgen.make_config(WORKLOAD)
    _, _, _, cfg = workload_config()
    if not os.path.exists(REF_BIN):
        return {"impl": "reference", "unavailable": "oracle/_ref/trinity_ref was not built "
                "(needs the reference sources at build time)"}
    mp, bp = ensure_files()
    cores = physical_cores()
    for _ in range(args.warmup):
        reference_once(mp, bp, c, cores)
    tin_sum, ms_sum, walls = 0, 0.0, []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        tin, ms, j = reference_once(mp, bp, c, cores)
        walls.append(time.perf_counter() - t0)
        tin_sum += tin
        ms_sum += ms
    value = tin_sum / (ms_sum / 1e3)
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_sum / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "mode": "reference OpenMP build, its own heuristics", "config": cfg,
        "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": "full adaptation per step (metric + 3 rounds), rounds timed by "
                                   "the harness around each kernel run"},
        "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "final_mesh": {"nodes": j["nodes_out"], "triangles": j["elems_out"]},
    }


def main():
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true", help="skip the host-buffer pass (profiling runs)")
    p.add_argument("--no-forms", action="store_true", help="skip the mixed-precision form")
    p.add_argument("--grid", type=int, default=None, help="grid side override (profiling runs)")
    p.add_argument("--workload", choices=["adapt", "batch"], default="adapt",
                   help="adapt: the 2M-triangle mesh (headline); batch: 256 meshes of uneven size")
    p.add_argument("--threads", type=int, default=0, help="host threads of the batched run")
    p.add_argument("--no-tune", action="store_true", help="default launch shapes (no autotuning)")
    args = p.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if "RANK" not in os.environ:
        world = 1

    if args.impl == "reference":
        line = reference_arm(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return

    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.workload == "batch":
            line = batch_arm(args, rank, world, local_rank)
            if line is not None:
                print(json.dumps(line), flush=True)
            return
        line = b200_arm(args, rank, world, local_rank)
        if not args.no_forms and world == 1:
            bf = _batch_run(args, rank, world, local_rank, 2, BATCH_FORM_CANDIDATES)
            if line is not None and bf is not None:
                line.setdefault("forms", {})["batch"] = bf
        if line is not None:
            if world == 1 and not args.no_forms:
                line.setdefault("forms", {})["io"] = io_form()
            if world == 1 and not args.no_cpu_baseline:
                line["cpu_baseline"] = cpu_baseline()
                if "io" in line.get("forms", {}):
                    line["forms"]["io"]["reference_mesh_load_ms"] = line["cpu_baseline"].get("mesh_load_ms")
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
