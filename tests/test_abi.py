"""The C-ABI library loads without a GPU and exports every function that
include/trinity_b200.h declares (no compute calls here)."""
import ctypes
import os
import re

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(REPO, "include", "trinity_b200.h")


def declared():
    src = open(HDR).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(trn_\w+)\s*\(", src)))


def test_header_declares_the_reference_boundary():
    names = declared()
    for f in ("trn_mesh_create", "trn_mesh_load", "trn_mesh_store", "trn_metric_run", "trn_refine_run",
              "trn_coarsen_run", "trn_swap_run", "trn_smooth_run", "trn_set_replay", "trn_last_error"):
        assert f in names


def test_library_exports_every_declared_symbol():
    from trinity_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [f for f in declared() if not hasattr(L, f)]
    assert not missing, missing


def test_version_string():
    from trinity_b200 import _lib
    assert b"sm_100a" in _lib.lib().trn_version()
