"""Python mirror of trinity's C++ API (include/trinity.h of the reference):
``Mesh``, ``Metrics``, ``Partit``, ``Refine``, ``Coarse``, ``Swap``, ``Smooth``
and ``Stats``, with the same constructor arguments and ``run(stats)`` calls,
backed by the CUDA library through its C ABI.

    mesh = Mesh(size, bucket, depth, verbosity, rounds)      # mesh.h:46
    metric = Metrics(mesh, target, norm, h_min, h_max)       # metric.h:38
    heuris = Partit(mesh, 8)                                 # partition.h:46
    refine, swap = Refine(mesh, depth), Swap(mesh)           # refinement.h:39, swapping.h:39
    coarse, smooth = Coarse(mesh, heuris), Smooth(mesh, heuris, depth)
    mesh.load(input, solut); metric.run(stats[0])
    for _ in range(rounds): refine.run(); coarse.run(); swap.run(); smooth.run()
    mesh.store(result)

As in the reference, the mesh must outlive the kernel objects, and calls are
blocking and not thread-safe on one mesh.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import Stats, TrinityError, lib

__all__ = ["Mesh", "Metrics", "Partit", "Refine", "Coarse", "Swap", "Smooth", "Stats",
           "TrinityError", "EPSILON", "H_MAX", "find", "batch_adapt", "adaptive_loop", "read_mesh_files"]

EPSILON = 1.0e-9   # header.h:50, the h_min the CLI passes (parser.cpp:95)
H_MAX = 0.4        # parser.cpp:96


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def find(key: str, path: str) -> int:
    """io::find (io.cpp:25-49): the count that follows section ``key``."""
    with open(path) as f:
        for line in f:
            s = line.lstrip()
            if s.startswith(("#", "%")):
                continue
            tok = s.split()
            if tok and tok[0] == key:
                for line2 in f:
                    t2 = line2.split()
                    if t2:
                        return int(t2[0])
    return -1


class Mesh:
    """GPU-resident mesh (Mesh, mesh.h:29-161)."""

    def __init__(self, size, bucket: int = 64, depth: int = 3, verbosity: int = 0,
                 rounds: int = 1, capa_scale: int | None = None):
        L = lib()
        self._L = L
        sz = (ctypes.c_int * 2)(int(size[0]), int(size[1]))
        h = ctypes.c_void_p()
        if capa_scale is None:
            rc = L.trn_mesh_create(sz, bucket, depth, verbosity, rounds, ctypes.byref(h))
        else:
            rc = L.trn_mesh_create_ex(sz, bucket, depth, verbosity, rounds, capa_scale, ctypes.byref(h))
        if rc:
            raise TrinityError(rc, "mesh creation failed")
        self.h = h
        self.depth = depth
        self.rounds = rounds

    def close(self):
        if getattr(self, "h", None):
            self._L.trn_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc: int):
        if rc:
            raise TrinityError(rc, self._L.trn_last_error(self.h).decode())

    def load(self, path: str, solu: str) -> None:
        self._check(self._L.trn_mesh_load(self.h, path.encode(), solu.encode() if solu else None))

    def load_arrays(self, points, tris, tags, solut) -> None:
        pts = np.ascontiguousarray(points, dtype=np.float64)
        tr = np.ascontiguousarray(tris, dtype=np.int32)
        tg = np.ascontiguousarray(tags, dtype=np.uint8)
        u = np.ascontiguousarray(solut, dtype=np.float64)
        self._check(self._L.trn_mesh_load_arrays(self.h, pts.shape[0], tr.shape[0], _p(pts), _p(tr),
                                                 _p(tg), _p(u)))

    def reload(self) -> None:
        """Back to the state right after the last load (device-side copy)."""
        self._check(self._L.trn_mesh_reload(self.h))

    def compact(self) -> None:
        """Renumber the adapted mesh on the device as a store + load would
        (live vertices and elements in slot order, full precision, boundary
        and corner tags kept); clears the nodal field."""
        self._check(self._L.trn_mesh_compact(self.h))

    def set_solution(self, solut) -> None:
        """The nodal field for the next metric run: one value per vertex slot
        in use (the rows of ``export()``)."""
        u = np.ascontiguousarray(solut, dtype=np.float64)
        self._check(self._L.trn_mesh_set_solution(self.h, _p(u), int(u.shape[0])))

    def store(self, path: str) -> None:
        self._check(self._L.trn_mesh_store(self.h, path.encode()))

    def store_binary(self, path: str) -> None:
        """The mesh in the binary form ``load`` also reads (no text parse)."""
        self._check(self._L.trn_mesh_store_binary(self.h, path.encode()))

    def store_sol(self, path: str) -> None:
        self._check(self._L.trn_mesh_store_sol(self.h, path.encode()))

    def counts(self):
        v = [ctypes.c_int() for _ in range(4)]
        self._check(self._L.trn_mesh_counts(self.h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def capacity(self):
        """(vertex slots, element slots) the mesh was created with."""
        a, b = ctypes.c_int(), ctypes.c_int()
        self._check(self._L.trn_mesh_capacity(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def export(self):
        """(points[V,2], tensor[V,3], tris[T,3], alive[V], tags[V]) of all slots in use."""
        nn, ne, _, _ = self.counts()
        pts = np.zeros((nn, 2)); ten = np.zeros((nn, 3)); tri = np.zeros((ne, 3), np.int32)
        alive = np.zeros(nn, np.uint8); tags = np.zeros(nn, np.uint8)
        self._check(self._L.trn_mesh_export(self.h, _p(pts), _p(ten), _p(tri), _p(alive), _p(tags)))
        return pts, ten, tri, alive, tags

    def export_compact(self, with_tensor: bool = True, out=None):
        """The adapted mesh without deleted entities, renumbered like
        Mesh::store: (points[V',2], tris[T',3] 0-based, tensor[V',3] or None).
        out: optional (points, tris, tensor) arrays with at least V' / T' rows
        (e.g. views of pinned host memory); the results are their leading rows."""
        _, _, nv, ne = self.counts()
        if out is not None:
            if out[0].shape[0] < nv or out[1].shape[0] < ne or (with_tensor and out[2].shape[0] < nv):
                raise ValueError("export_compact: output arrays too small")
            pts, tri = out[0][:nv], out[1][:ne]
            ten = out[2][:nv] if with_tensor else None
        else:
            pts = np.empty((nv, 2)); tri = np.empty((ne, 3), np.int32)
            ten = np.empty((nv, 3)) if with_tensor else None
        a, b = ctypes.c_int(), ctypes.c_int()
        self._check(self._L.trn_mesh_export_compact(self.h, _p(pts), _p(tri), _p(ten) if with_tensor else None,
                                                    ctypes.byref(a), ctypes.byref(b)))
        assert (a.value, b.value) == (nv, ne)
        return pts, tri, ten

    def set_precision(self, mode: str) -> None:
        """'fp64' (default, bit-compatible drop-in) or 'mixed' (FP32 metric
        arithmetic, FP64 coordinates and orientation)."""
        self._check(self._L.trn_set_precision(self.h, {"fp64": 0, "mixed": 1}[mode]))

    def qualities(self):
        nn, ne, _, _ = self.counts()
        q = np.empty(ne)
        self._check(self._L.trn_mesh_qualities(self.h, _p(q)))
        return q

    def quality_stats(self):
        """Mesh::computeQuality(double[3]): (min, max, mean)."""
        q = np.array([3.0, 0.0, 0.0])
        self._check(self._L.trn_mesh_quality_stats(self.h, _p(q)))
        return tuple(q.tolist())

    def set_replay(self, log) -> None:
        a = np.ascontiguousarray(log, dtype=np.int32)
        self._check(self._L.trn_set_replay(self.h, _p(a) if a.size else None, a.size))

    def set_options(self, seed: int = 0x7472696E697479, exact_sum: bool = False) -> None:
        self._check(self._L.trn_set_options(self.h, seed, 1 if exact_sum else 0))

    SWAP_MATCH = {"row_order": 0, "gain": 1, "greedy": 2}

    def set_swap_match(self, policy: str = "greedy") -> None:
        """Free-mode swap matching: "greedy" (the reference's greedy loop over
        the candidates in the order (id mod 4, id), computed exactly in
        parallel; the default), "row_order" (a handshake preferring the
        reference's row slots) or "gain" (each candidate prefers its best
        flip)."""
        if policy not in self.SWAP_MATCH:
            raise ValueError(f"swap matching policy {policy!r}: one of {sorted(self.SWAP_MATCH)}")
        self._check(self._L.trn_set_swap_match(self.h, self.SWAP_MATCH[policy]))

    def set_level_cap(self, cap: int) -> None:
        """Most coarsening / swapping levels a call runs (TRN_ERR_NO_PROGRESS past it)."""
        self._check(self._L.trn_set_level_cap(self.h, cap))

    def last_time_ms(self) -> float:
        return self._L.trn_last_time_ms(self.h)

    def stream(self) -> int:
        return self._L.trn_mesh_stream(self.h)

    TUNE_KEYS = ("smooth_threads", "filter_threads", "group_lanes", "group_max", "flip_threads", "smooth_lanes",
                 "smooth_regs")

    def get_tune(self) -> dict:
        a = np.zeros(len(self.TUNE_KEYS), dtype=np.int32)
        self._check(self._L.trn_get_tune(self.h, _p(a)))
        return dict(zip(self.TUNE_KEYS, a.tolist()))

    def set_tune(self, cfg: dict) -> None:
        a = np.array([cfg[k] for k in self.TUNE_KEYS], dtype=np.int32)
        self._check(self._L.trn_set_tune(self.h, _p(a)))

    def autotune(self, target_factor: float, Lp_norm: int = 2, depth: int = 1, rounds: int = 1,
                 h_min: float = EPSILON, h_max: float = H_MAX) -> dict:
        """Launch shapes chosen on this mesh (trn_autotune); the mesh is
        reloaded afterwards."""
        a = np.zeros(len(self.TUNE_KEYS), dtype=np.int32)
        self._check(self._L.trn_autotune(self.h, target_factor, Lp_norm, h_min, h_max, depth, rounds, _p(a)))
        return dict(zip(self.TUNE_KEYS, a.tolist()))

    def round_graph(self, depth: int, stats=None) -> None:
        """One free-mode round as the mesh's captured CUDA graph
        (trn_round_graph_run); stats: a ctypes array of 4 Stats or None."""
        self._check(self._L.trn_round_graph_run(self.h, depth, stats))

    def quality_adjoint(self, xy=None, solut=None, *, target_factor: float = 1.0, Lp_norm: int = 2,
                        h_min: float = EPSILON, h_max: float = H_MAX, precision: str = "fp64",
                        grad_xy: bool = True, grad_solut: bool | None = None):
        """J = sum of the live elements' qualities, and its adjoint
        (trn_quality_adjoint). xy: (V, 2) and solut: (V,) float64 CUDA
        tensors in the mesh's vertex numbering; xy None = the mesh's
        coordinates; solut None = the mesh's current tensors are the metric,
        else the metric is recovered from solut with (target_factor, Lp_norm,
        h_min, h_max) on the mesh's coordinates. Returns (J, dJ/dxy, dJ/dsolut),
        the gradients as CUDA tensors (None where not asked for)."""
        import torch
        nn = self.counts()[0]
        dev = torch.device("cuda", torch.cuda.current_device())

        def dptr(t, shape, name):
            if t is None:
                return None
            if (t.device.type != "cuda" or t.dtype != torch.float64 or not t.is_contiguous()
                    or tuple(t.shape) != shape):
                raise ValueError(f"{name}: want a contiguous float64 CUDA tensor of shape {shape}")
            return ctypes.c_void_p(t.data_ptr())

        if grad_solut is None:
            grad_solut = solut is not None
        if grad_solut and solut is None:
            raise ValueError("grad_solut needs solut")
        gxy = torch.empty((nn, 2), dtype=torch.float64, device=dev) if grad_xy else None
        gu = torch.empty(nn, dtype=torch.float64, device=dev) if grad_solut else None
        args = (dptr(xy, (nn, 2), "xy"), dptr(solut, (nn,), "solut"))
        torch.cuda.current_stream().synchronize()
        J = ctypes.c_double(0.0)
        self._check(self._L.trn_quality_adjoint(
            self.h, args[0], args[1], target_factor, Lp_norm, h_min, h_max,
            {"fp64": 0, "mixed": 1, "fp32": 1}[precision], ctypes.byref(J),
            dptr(gxy, (nn, 2), "grad_xy"), dptr(gu, (nn,), "grad_solut")))
        return J.value, gxy, gu


def batch_adapt(meshes, target_factor: float, Lp_norm: int = 2, rounds: int = 3, depth: int = 1,
                threads: int = 8, h_min: float = EPSILON, h_max: float = H_MAX, graph: bool = False):
    """Metric recovery + rounds for many loaded meshes at once (one stream per
    mesh, a pool of host threads). Returns (round_ms[count], tri_in[count]).
    Set CUDA_DEVICE_MAX_CONNECTIONS=32 in the environment before CUDA starts
    so that the streams do not share the default 8 hardware queues. graph:
    each round as the mesh's captured CUDA graph (free mode)."""
    L = lib()
    n = len(meshes)
    handles = (ctypes.c_void_p * n)(*[m.h.value if hasattr(m.h, "value") else m.h for m in meshes])
    ms = np.zeros(n)
    tin = np.zeros(n, dtype=np.int64)
    rc = L.trn_batch_adapt_ex(ctypes.cast(handles, ctypes.c_void_p), n, target_factor, Lp_norm, h_min, h_max,
                              rounds, depth, threads, 1 if graph else 0, _p(ms), _p(tin))
    if rc:
        raise TrinityError(rc, "batch adaptation failed: " + "; ".join(
            m._L.trn_last_error(m.h).decode() for m in meshes if m._L.trn_last_error(m.h)))
    return ms, tin


def batch_autotune(meshes, target_factor: float, Lp_norm: int = 2, rounds: int = 3, depth: int = 1,
                   threads: int = 8, graph: bool = True, candidates: dict | None = None):
    """Launch shapes for a batch adapted concurrently: coordinate descent
    over one table shared by all meshes, each candidate timed by running the
    whole batch (wall clock, best of two); shapes that suit a mesh alone need
    not suit it among many. Leaves the chosen table set on every mesh and the
    meshes reloaded. Returns (table, {trial: seconds})."""
    import time
    cand = candidates or {"group_lanes": [4, 8, 16], "group_max": [4096, 16384, 65536],
                          "smooth_threads": [64, 128, 256], "filter_threads": [128, 256, 512],
                          "flip_threads": [128, 256, 512]}
    best = meshes[0].get_tune()

    def timed(cfg):
        t = 1e300
        for _ in range(2):
            for g in meshes:
                g.set_tune(cfg)
                g.reload()
            t0 = time.perf_counter()
            batch_adapt(meshes, target_factor, Lp_norm, rounds, depth, threads=threads, graph=graph)
            t = min(t, time.perf_counter() - t0)
        return t

    trials = {}
    for key, values in cand.items():
        scores = {}
        for v in values:
            cfg = dict(best, **{key: v})
            scores[v] = timed(cfg)
            trials[f"{key}={v}"] = round(scores[v], 4)
        best[key] = min(scores, key=scores.get)
    for g in meshes:
        g.set_tune(best)
        g.reload()
    return best, trials


class Metrics:
    """Metrics(Mesh*, target_factor, Lp_norm, h_min, h_max) (metric.h:38-44)."""

    def __init__(self, mesh: Mesh, target_factor: float, Lp_norm: int, h_min: float = EPSILON,
                 h_max: float = H_MAX):
        self.mesh, self.target, self.norm, self.h_min, self.h_max = mesh, target_factor, Lp_norm, h_min, h_max

    def run(self, total: Stats | None = None) -> None:
        m = self.mesh
        m._check(m._L.trn_metric_run(m.h, self.target, self.norm, self.h_min, self.h_max,
                                     ctypes.byref(total) if total is not None else None))

    def complexity(self) -> float:
        return self.mesh._L.trn_last_complexity(self.mesh.h)


class Partit:
    """Partit(Mesh const*, max_part_size) (partition.h:46): the coloring /
    independent-set engine shared by Coarse and Smooth."""

    def __init__(self, mesh: Mesh, max_part_size: int = 8):
        self.mesh = mesh
        self.max_part = max(6, max_part_size)


class Refine:
    def __init__(self, mesh: Mesh, level: int):
        self.mesh, self.level = mesh, level

    def run(self, total: Stats | None = None) -> None:
        m = self.mesh
        m._check(m._L.trn_refine_run(m.h, self.level, ctypes.byref(total) if total is not None else None))


class Coarse:
    def __init__(self, mesh: Mesh, algo: Partit):
        self.mesh, self.algo = mesh, algo

    def run(self, total: Stats | None = None) -> None:
        m = self.mesh
        m._check(m._L.trn_coarsen_run(m.h, self.algo.max_part,
                                      ctypes.byref(total) if total is not None else None))


class Swap:
    def __init__(self, mesh: Mesh):
        self.mesh = mesh

    def run(self, total: Stats | None = None) -> None:
        m = self.mesh
        m._check(m._L.trn_swap_run(m.h, ctypes.byref(total) if total is not None else None))


class GradientSmooth:
    """Gradient-based smoothing beside Smooth (trn_smooth_gradient_run):
    `steps` passes over the color classes, each interior vertex stepping up
    the metric-preconditioned gradient of its elements' summed quality
    (objective "sum") or summed log-quality ("log"); with tensor_follows the
    moved vertex takes its neighbours' log-Euclidean mean tensor, as the smart
    Laplacian's does."""

    def __init__(self, mesh: Mesh, algo: Partit, steps: int, max_len: float = 0.1,
                 objective: str = "log", tensor_follows: bool = True):
        self.mesh, self.algo, self.steps, self.max_len = mesh, algo, steps, max_len
        self.mode = {"sum": 0, "log": 1}[objective] | (2 if tensor_follows else 0)

    def run(self, total: Stats | None = None) -> None:
        m = self.mesh
        m._check(m._L.trn_smooth_gradient_run(m.h, self.algo.max_part, self.steps, self.max_len,
                                              self.mode,
                                              ctypes.byref(total) if total is not None else None))


class Smooth:
    def __init__(self, mesh: Mesh, algo: Partit, level: int):
        self.mesh, self.algo, self.level = mesh, algo, level

    def run(self, total: Stats | None = None) -> None:
        m = self.mesh
        m._check(m._L.trn_smooth_run(m.h, self.algo.max_part, self.level,
                                     ctypes.byref(total) if total is not None else None))


def read_mesh_files(mesh_path: str, solut_path: str | None = None):
    """The .mesh (text or binary) and .bb files as ``Mesh.load`` reads them,
    on the host: (points[V,2], tris[T,3] 0-based, tags[V], solut[V] or None)."""
    L = lib()
    nv, nt = ctypes.c_int(), ctypes.c_int()
    sp = solut_path.encode() if solut_path else None
    rc = L.trn_read_mesh_files(mesh_path.encode(), sp, ctypes.byref(nv), ctypes.byref(nt),
                               None, None, None, None, 0, 0)
    if rc:
        raise TrinityError(rc, f"cannot read {mesh_path}")
    pts = np.zeros((nv.value, 2)); tri = np.zeros((nt.value, 3), np.int32)
    tags = np.zeros(nv.value, np.uint8)
    u = np.zeros(nv.value) if solut_path else None
    rc = L.trn_read_mesh_files(mesh_path.encode(), sp, ctypes.byref(nv), ctypes.byref(nt), _p(pts), _p(tri),
                               _p(tags), _p(u) if u is not None else None, nv.value, nt.value)
    if rc:
        raise TrinityError(rc, f"cannot read {mesh_path} / {solut_path}")
    return pts, tri, tags, u


def adaptive_loop(mesh: Mesh, field, cycles: int, target: float, norm: int = 2, depth: int = 1,
                  rounds: int = 3, max_part: int = 8, on_cycle=None):
    """The solver-coupled loop trinity is written for (README.md:8; the
    reference's scripts/bench_run.py:77-110 runs it through files): for each
    cycle, evaluate ``field(points) -> values`` on the current mesh, recover
    the metric, run ``rounds`` rounds of refine / coarsen / swap / smooth,
    then renumber the adapted mesh on the device for the next cycle. The
    first cycle uses the mesh as loaded. ``on_cycle(k, mesh)`` is called
    after each cycle's rounds, before the renumbering."""
    heur = Partit(mesh, max_part)
    kern = (Refine(mesh, depth), Coarse(mesh, heur), Swap(mesh), Smooth(mesh, heur, depth))
    for k in range(cycles):
        if k > 0:
            mesh.compact()
        pts = mesh.export()[0]
        mesh.set_solution(field(pts))
        Metrics(mesh, target, norm).run()
        for _ in range(rounds):
            for kk in kern:
                kk.run()
        if on_cycle is not None:
            on_cycle(k, mesh)
