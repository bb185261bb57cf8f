"""Batched adaptation: many meshes adapted concurrently (one stream each, a
pool of host threads) end exactly where the same meshes adapted one at a time
end (the free mode is deterministic and the meshes share nothing)."""
import numpy as np
import pytest

from tests.helpers import check_invariants, gpu_state
from tests.oracle_lib import tags_of
from trinity_b200 import meshgen


def _load(m, u, p):
    from trinity_b200.api import Mesh
    g = Mesh((m.nb_nodes, m.nb_elems), p["bucket"], p["depth"], 0, p["rounds"],
             capa_scale=p["capa_scale"])
    g.load_arrays(m.points, m.tris, tags_of(m), u)
    g.set_swap_match(p["swap_match"])
    return g


@pytest.mark.gpu
def test_batch_equals_one_at_a_time():
    from trinity_b200.api import batch_adapt
    p = meshgen.BATCH_PARAMS
    items = list(meshgen.batch_meshes(count=10, seed=11, lo=12, hi=64))
    solo = []
    for m, u, _ in items:
        g = _load(m, u, p)
        ms, tin = batch_adapt([g], p["target"], p["norm"], p["rounds"], p["depth"], threads=1)
        solo.append(gpu_state(g))
        g.close()
    many = [_load(m, u, p) for m, u, _ in items]
    ms, tin = batch_adapt(many, p["target"], p["norm"], p["rounds"], p["depth"], threads=4)
    assert np.all(ms > 0) and np.all(tin > 0)
    for g, want in zip(many, solo):
        st = gpu_state(g)
        assert not st.diff(want)
        check_invariants(st)


@pytest.mark.gpu
def test_batch_meshes_are_valid_and_match_the_reference_build(tmp_path):
    """The first 12 meshes of the 256-mesh workload (sides 36 to 511),
    adapted concurrently with captured rounds: every one conforming, CCW and
    a disk; the ones of 50k triangles or more (sides 195 to 511) within 3 %
    of the reference build's final triangle count and 1 point of its fraction
    of metric edge lengths in [1/sqrt 2, sqrt 2] (medians of 3 reference
    runs: its OpenMP heuristics vary from run to run, 181.3k to 184.1k
    triangles on the side-301 mesh on one host, 179.5k to 181.5k on
    another), each on the same input. The workload's swap matching is the
    row-slot handshake (meshgen.BATCH_PARAMS), which ends the side-301 mesh
    at 178.9k: 2.1 % under the first host's median. (The smaller meshes,
    coarse grids under steep shocks, end far from unit lengths after 3
    rounds of depth 1 in both codes.)"""
    import os
    import subprocess
    from tests.helpers import in_range_fraction
    from tests.oracle_lib import REF_TIMED, read_snapshot
    from trinity_b200.api import batch_adapt
    p = meshgen.BATCH_PARAMS
    items = []
    for k, it in enumerate(meshgen.batch_meshes()):
        if k == 12:
            break
        items.append(it)
    meshes = [_load(m, u, p) for m, u, _ in items]
    batch_adapt(meshes, p["target"], p["norm"], p["rounds"], p["depth"], threads=4, graph=True)
    states = [gpu_state(g) for g in meshes]
    for g in meshes:
        g.close()
    for st in states:
        check_invariants(st)
    if not os.path.exists(REF_TIMED):
        pytest.skip("reference build (oracle/_ref) absent")
    big = [k for k, (m, _, _) in enumerate(items) if m.nb_elems >= 50000]
    assert len(big) >= 3
    for k in big:
        m, u, spec = items[k]
        mp, bp = str(tmp_path / f"b{k}.mesh"), str(tmp_path / f"b{k}.bb")
        meshgen.write_mesh(mp, m)
        meshgen.write_bb(bp, u)
        # the reference's OpenMP heuristics differ from run to run (up to
        # ~1.5 % in the final count on these meshes): the median of 3 runs
        counts, fracs = [], []
        for rep in range(3):
            out = str(tmp_path / f"f{k}_{rep}.bin")
            subprocess.run([REF_TIMED, mp, bp, str(p["rounds"]), str(p["depth"]), str(p["bucket"]),
                            str(p["target"]), str(p["norm"]), "--capa-depth", "4", "--final", out], check=True,
                           capture_output=True, timeout=600, env=dict(os.environ, OMP_NUM_THREADS="8"))
            ref = read_snapshot(out)
            counts.append(ref.active_elems().shape[0])
            fracs.append(in_range_fraction(ref))
        st = states[k]
        n_gpu, n_ref = st.active_elems().shape[0], float(np.median(counts))
        assert abs(n_gpu - n_ref) <= 0.03 * n_ref, (spec, n_gpu, counts)
        f_gpu, f_ref = in_range_fraction(st), float(np.median(fracs))
        assert abs(f_gpu - f_ref) <= 0.01, (spec, f_gpu, fracs)
