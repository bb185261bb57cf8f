"""ctypes binding of the C ABI in include/trinity_b200.h.

The shared library is built in-tree (``make -C trinity_b200``) and loaded from
the package directory; there is no CPU fallback, so a missing library is an
error.
"""
from __future__ import annotations

import ctypes
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libtrinity_b200.so")

TRN_OK = 0
ERRORS = {
    1: "TRN_ERR_CAPACITY",
    2: "TRN_ERR_IO",
    3: "TRN_ERR_INVALID",
    4: "TRN_ERR_NO_PROGRESS",
    5: "TRN_ERR_CUDA",
    6: "TRN_ERR_REPLAY",
}


class Stats(ctypes.Structure):
    """trinity::Stats (header.h:72-77)."""
    _fields_ = [("eval", ctypes.c_int), ("task", ctypes.c_int), ("elap", ctypes.c_int),
                ("step", ctypes.c_int * 5)]

    def __repr__(self):
        return f"Stats(eval={self.eval}, task={self.task}, elap={self.elap})"


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}` "
                "(the GPU path has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, dp, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t
        pmesh = ctypes.c_void_p
        sp = ctypes.POINTER(Stats)
        L.trn_mesh_create.argtypes = [vp, ip, ip, ip, ip, ctypes.POINTER(pmesh)]
        L.trn_mesh_create_ex.argtypes = [vp, ip, ip, ip, ip, ip, ctypes.POINTER(pmesh)]
        L.trn_mesh_destroy.argtypes = [pmesh]
        L.trn_mesh_load.argtypes = [pmesh, ctypes.c_char_p, ctypes.c_char_p]
        L.trn_mesh_load_arrays.argtypes = [pmesh, ip, ip, vp, vp, vp, vp]
        L.trn_mesh_store.argtypes = [pmesh, ctypes.c_char_p]
        L.trn_mesh_store_sol.argtypes = [pmesh, ctypes.c_char_p]
        L.trn_mesh_export.argtypes = [pmesh, vp, vp, vp, vp, vp]
        L.trn_mesh_counts.argtypes = [pmesh, vp, vp, vp, vp]
        L.trn_metric_run.argtypes = [pmesh, dp, ip, dp, dp, sp]
        L.trn_refine_run.argtypes = [pmesh, ip, sp]
        L.trn_coarsen_run.argtypes = [pmesh, ip, sp]
        L.trn_swap_run.argtypes = [pmesh, sp]
        L.trn_smooth_run.argtypes = [pmesh, ip, ip, sp]
        L.trn_round_run.argtypes = [pmesh, ip, sp]
        L.trn_set_replay.argtypes = [pmesh, vp, sz]
        L.trn_set_options.argtypes = [pmesh, ctypes.c_uint64, ip]
        L.trn_set_swap_match.argtypes = [pmesh, ip]
        L.trn_set_level_cap.argtypes = [pmesh, ip]
        L.trn_selftest_barrier.argtypes = [ctypes.c_longlong]
        L.trn_mesh_compact.argtypes = [pmesh]
        L.trn_mesh_capacity.argtypes = [pmesh, ctypes.POINTER(ip), ctypes.POINTER(ip)]
        L.trn_mesh_store_binary.argtypes = [pmesh, ctypes.c_char_p]
        L.trn_read_mesh_files.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ip),
                                          ctypes.POINTER(ip), vp, vp, vp, vp, ip, ip]
        L.trn_mesh_set_solution.argtypes = [pmesh, vp, ip]
        L.trn_last_complexity.argtypes = [pmesh]
        L.trn_last_complexity.restype = dp
        L.trn_last_time_ms.argtypes = [pmesh]
        L.trn_last_time_ms.restype = dp
        L.trn_mesh_stream.argtypes = [pmesh]
        L.trn_mesh_stream.restype = vp
        L.trn_last_error.argtypes = [pmesh]
        L.trn_last_error.restype = ctypes.c_char_p
        L.trn_version.restype = ctypes.c_char_p
        L.trn_mesh_reload.argtypes = [pmesh]
        L.trn_set_precision.argtypes = [pmesh, ip]
        L.trn_batch_adapt.argtypes = [vp, ip, dp, ip, dp, dp, ip, ip, ip, vp, vp]
        L.trn_batch_adapt_ex.argtypes = [vp, ip, dp, ip, dp, dp, ip, ip, ip, ip, vp, vp]
        L.trn_round_graph_run.argtypes = [pmesh, ip, sp]
        L.trn_get_tune.argtypes = [pmesh, vp]
        L.trn_set_tune.argtypes = [pmesh, vp]
        L.trn_autotune.argtypes = [pmesh, dp, ip, dp, dp, ip, ip, vp]
        L.trn_mesh_qualities.argtypes = [pmesh, vp]
        L.trn_mesh_quality_stats.argtypes = [pmesh, vp]
        L.trn_mesh_export_compact.argtypes = [pmesh, vp, vp, vp, ctypes.POINTER(ip), ctypes.POINTER(ip)]
        L.trn_profile_enable.argtypes = [ip]
        L.trn_profile_count.restype = ip
        L.trn_profile_entry.argtypes = [ip, ctypes.c_char_p, ip, ctypes.POINTER(ctypes.c_longlong),
                                        ctypes.POINTER(dp), ctypes.POINTER(dp)]
        L.trn_launch_count.restype = ctypes.c_ulonglong
        L.trn_profile_only.argtypes = [ctypes.c_char_p]
        L.trn_profile_count_bytes.argtypes = [ip, ip]
        L.trn_profile_counted.argtypes = [ip]
        L.trn_quality_adjoint.argtypes = [pmesh, vp, vp, dp, ip, dp, dp, ip, ctypes.POINTER(dp), vp, vp]
        L.trn_smooth_gradient_run.argtypes = [pmesh, ip, ip, dp, ip, sp]
        _lib = L
    return _lib


class TrinityError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


def profile_enable(on: bool) -> None:
    """Per-kernel device timing (process-wide); enabling resets the totals."""
    lib().trn_profile_enable(1 if on else 0)


def profile_only(name: str | None) -> None:
    """Time only the named kernel's launches (None = all)."""
    lib().trn_profile_only(name.encode() if name else None)


def profile_read() -> list[dict]:
    L = lib()
    out = []
    for i in range(L.trn_profile_count()):
        name = ctypes.create_string_buffer(64)
        n = ctypes.c_longlong()
        ms = ctypes.c_double()
        by = ctypes.c_double()
        L.trn_profile_entry(i, name, 64, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(by))
        out.append({"kernel": name.value.decode(), "launches": n.value, "ms": ms.value,
                    "bytes": by.value, "bytes_counted": L.trn_profile_counted(i) == n.value > 0})
    return out


def profile_count_bytes(on: bool, max_nodes: int = 0) -> None:
    """Kernels that can count their algorithmic bytes on the device do so
    (profiled runs: the counting adds atomics)."""
    rc = lib().trn_profile_count_bytes(1 if on else 0, int(max_nodes))
    if rc:
        raise TrinityError(rc, "byte counters: device allocation failed")


def launch_count() -> int:
    return int(lib().trn_launch_count())
