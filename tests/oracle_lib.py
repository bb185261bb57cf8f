"""ctypes access to the C oracle (oracle/_build/liboracle.so) and to the
reference snapshots written by oracle/ref_harness.cpp.

Test infrastructure only: the oracle is the checker, never the product.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "_build", "liboracle.so")
REF_EXACT = os.path.join(ORACLE_DIR, "_ref", "trinity_ref_exact")
REF_TIMED = os.path.join(ORACLE_DIR, "_ref", "trinity_ref")
# trinity's own source tree (read only where it is mounted: golden fixtures,
# the C++ shim compile test and trinity's GRID4 fixture); one variable, one
# default
REF_SRC = os.environ.get("TRN_REFERENCE_DIR", "/root/reference")

LOG_MIS, LOG_MATCH, LOG_COLORING = 1, 2, 3
TAG_BOUND, TAG_CORNER = 4, 8

_lib = None


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", ORACLE_DIR, "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = ctypes.CDLL(ORACLE_SO)
        vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.orc_create.restype = vp
        L.orc_create.argtypes = [ip, ip, ip]
        L.orc_destroy.argtypes = [vp]
        L.orc_load.argtypes = [vp, ip, ip, vp, vp, vp, vp]
        L.orc_metric.argtypes = [vp, dp, ip, dp, dp]
        L.orc_refine.argtypes = [vp, ip]
        L.orc_coarsen.argtypes = [vp]
        L.orc_swap.argtypes = [vp]
        L.orc_smooth.argtypes = [vp, ip]
        L.orc_nb_nodes.argtypes = [vp]
        L.orc_nb_elems.argtypes = [vp]
        L.orc_export.argtypes = [vp, vp, vp, vp, vp, vp]
        L.orc_complexity.argtypes = [vp]
        L.orc_complexity.restype = dp
        L.orc_counters.argtypes = [vp, vp]
        L.orc_log.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t)]
        L.orc_log.restype = ctypes.POINTER(ctypes.c_int32)
        L.orc_log_clear.argtypes = [vp]
        L.orc_set_swap_rule.argtypes = [vp, ip]
        L.orc_set_swap_strict_map.argtypes = [vp, ip]
        L.orc_eigen.argtypes = [vp, vp, vp, vp]
        L.orc_interpolate.argtypes = [vp, vp, ip]
        L.orc_quality.argtypes = [vp] * 6
        L.orc_quality.restype = dp
        L.orc_length.argtypes = [vp] * 4
        L.orc_length.restype = dp
        L.orc_steiner.argtypes = [vp] * 6
        for f in ("orc_log_fn", "orc_exp_fn"):
            getattr(L, f).argtypes = [dp]
            getattr(L, f).restype = dp
        L.orc_pow_fn.argtypes = [dp, dp]
        L.orc_pow_fn.restype = dp
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def tags_of(mesh) -> np.ndarray:
    """Boundary / corner tags as trinity's loader sets them (io.cpp:80-104)."""
    t = np.zeros(mesh.nb_nodes, dtype=np.uint8)
    t[mesh.edges.ravel()] = TAG_BOUND
    t[mesh.corners] = TAG_BOUND | TAG_CORNER
    return t


class State:
    """Full-precision mesh state (same layout as the reference snapshots)."""

    def __init__(self, points, tensor, elems, alive, tags):
        self.points, self.tensor, self.elems = points, tensor, elems
        self.alive, self.tags = alive, tags

    @property
    def nb_nodes(self):
        return self.points.shape[0]

    @property
    def nb_elems(self):
        return self.elems.shape[0]

    def active_elems(self):
        return self.elems[self.elems[:, 0] >= 0]

    def diff(self, other) -> list[str]:
        out = []
        if self.nb_nodes != other.nb_nodes or self.nb_elems != other.nb_elems:
            out.append(f"counts {self.nb_nodes},{self.nb_elems} vs {other.nb_nodes},{other.nb_elems}")
            return out
        for name in ("elems", "alive", "tags"):
            a, b = getattr(self, name), getattr(other, name)
            if not np.array_equal(a, b):
                idx = np.argwhere(a != b)[:3]
                out.append(f"{name} differ at {idx.tolist()}")
        for name in ("points", "tensor"):
            a, b = getattr(self, name), getattr(other, name)
            if not np.array_equal(a.view(np.uint64), b.view(np.uint64)):
                bad = np.argwhere(a.view(np.uint64) != b.view(np.uint64))
                rel = np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))
                out.append(f"{name} differ at {len(bad)} entries (first {bad[:2].tolist()}), max rel {rel:.3e}")
        return out


def read_snapshot(path: str) -> State:
    raw = open(path, "rb").read()
    hdr = np.frombuffer(raw, dtype=np.int32, count=3)
    assert hdr[0] == 0x54524E31
    nn, ne = int(hdr[1]), int(hdr[2])
    off = 12
    pts = np.frombuffer(raw, np.float64, 2 * nn, off).reshape(nn, 2); off += 16 * nn
    ten = np.frombuffer(raw, np.float64, 3 * nn, off).reshape(nn, 3); off += 24 * nn
    el = np.frombuffer(raw, np.int32, 3 * ne, off).reshape(ne, 3); off += 12 * ne
    alive = np.frombuffer(raw, np.uint8, nn, off); off += nn
    tags = np.frombuffer(raw, np.uint8, nn, off)
    return State(pts.copy(), ten.copy(), el.copy(), alive.copy(), tags.copy())


class Oracle:
    """One mesh in the C oracle; mirrors the reference's kernel calls."""

    def __init__(self, mesh, solut, capa_scale: int = 9, bucket: int = 64, tags=None):
        L = lib()
        self.L = L
        self.h = L.orc_create(mesh.nb_nodes * capa_scale, mesh.nb_elems * capa_scale, bucket)
        if not self.h:
            raise MemoryError("oracle allocation failed")
        pts = np.ascontiguousarray(mesh.points, dtype=np.float64)
        tris = np.ascontiguousarray(mesh.tris, dtype=np.int32)
        tags = tags_of(mesh) if tags is None else np.ascontiguousarray(tags, dtype=np.uint8)
        u = np.ascontiguousarray(solut, dtype=np.float64)
        rc = L.orc_load(self.h, mesh.nb_nodes, mesh.nb_elems, _p(pts), _p(tris), _p(tags), _p(u))
        if rc:
            raise RuntimeError(f"orc_load failed: {rc}")

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def _chk(self, rc, what):
        if rc:
            raise RuntimeError(f"oracle {what} failed with {rc}")

    def metric(self, target, norm=2, h_min=1e-9, h_max=0.4):
        self._chk(self.L.orc_metric(self.h, target, norm, h_min, h_max), "metric")

    def refine(self, depth):
        self._chk(self.L.orc_refine(self.h, depth), "refine")

    def coarsen(self):
        self._chk(self.L.orc_coarsen(self.h), "coarsen")

    def swap(self):
        self._chk(self.L.orc_swap(self.h), "swap")

    def smooth(self, depth):
        self._chk(self.L.orc_smooth(self.h, depth), "smooth")

    def counters(self):
        c = np.zeros(4, dtype=np.int32)
        self.L.orc_counters(self.h, _p(c))
        return c

    def complexity(self):
        return self.L.orc_complexity(self.h)

    def state(self) -> State:
        nn, ne = self.L.orc_nb_nodes(self.h), self.L.orc_nb_elems(self.h)
        pts = np.zeros((nn, 2)); ten = np.zeros((nn, 3))
        el = np.zeros((ne, 3), np.int32)
        alive = np.zeros(nn, np.uint8); tags = np.zeros(nn, np.uint8)
        self.L.orc_export(self.h, _p(pts), _p(ten), _p(el), _p(alive), _p(tags))
        return State(pts, ten, el, alive, tags)

    SWAP_RULES = {"reference": 0, "sequential_rows": 1, "handshake_random": 2, "handshake_rowslot": 3,
                  "greedy_interleaved": 4}

    def set_swap_rule(self, rule: str) -> None:
        """Swap matching rule (analysis of the GPU free mode; "reference" is
        the reference's own)."""
        self._chk(self.L.orc_set_swap_rule(self.h, self.SWAP_RULES[rule]), "set_swap_rule")

    def set_swap_strict_map(self, on: bool) -> None:
        """Flips re-activate only rows of the current level (the GPU free mode's rule)."""
        self._chk(self.L.orc_set_swap_strict_map(self.h, 1 if on else 0), "set_swap_strict_map")

    def log(self) -> np.ndarray:
        n = ctypes.c_size_t(0)
        ptr = self.L.orc_log(self.h, ctypes.byref(n))
        if n.value == 0:
            return np.zeros(0, np.int32)
        return np.ctypeslib.as_array(ptr, shape=(n.value,)).copy()

    def clear_log(self):
        self.L.orc_log_clear(self.h)


def run_pipeline(obj, params, stages=None, log_stage=None):
    """Run metric + rounds on an Oracle-like object, calling ``log_stage(name)``
    after every kernel. Returns the list of stage names."""
    names = []
    obj.metric(params["target"], params["norm"])
    names.append("metric")
    if log_stage:
        log_stage("metric")
    for r in range(params["rounds"]):
        for k in ("refine", "coarse", "swap", "smooth"):
            if k == "refine":
                obj.refine(params["depth"])
            elif k == "coarse":
                obj.coarsen()
            elif k == "swap":
                obj.swap()
            else:
                obj.smooth(params["depth"])
            name = f"r{r}.{k}"
            names.append(name)
            if log_stage:
                log_stage(name)
    return names


def digest(st: State) -> dict:
    """SHA-256 per field of a full-precision state (bit-exact fingerprint)."""
    import hashlib
    out = {"nodes": int(st.nb_nodes), "elems": int(st.nb_elems),
           "live_elems": int((st.elems[:, 0] >= 0).sum()), "live_nodes": int(st.alive.sum())}
    for name in ("points", "tensor", "elems", "alive", "tags"):
        a = np.ascontiguousarray(getattr(st, name))
        out[name] = hashlib.sha256(a.tobytes()).hexdigest()
    return out


def compact_state(st: State):
    """Mesh::store's renumbering (io.cpp:164-255) at full precision: the live
    vertices in slot order (points, tags) and the live elements in slot
    order, renumbered; returns (points, tris, tags)."""
    keep = np.flatnonzero(st.alive)
    newid = -np.ones(st.nb_nodes, np.int64)
    newid[keep] = np.arange(keep.shape[0])
    tri = st.active_elems()
    return st.points[keep].copy(), newid[tri].astype(np.int32), st.tags[keep].copy()
