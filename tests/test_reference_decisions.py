"""The decisions the GPU replays are the reference's own: trinity built from
its own sources with its graph heuristics recorded as it runs
(oracle/_ref/trinity_ref_decide: Partit::extractIndepSet,
Match::computeGreedyMatching and Partit::extractColoring wrapped at link
time, oracle/ref_decisions.cpp) emits, on one thread, the same int32 stream,
word for word, as the oracle's decision log, which the replay tests feed to
the GPU (independent sets per coarsening level, matched pairs per swapping
level, color classes per smoothing call)."""
import json
import os
import subprocess

import numpy as np
import pytest

from tests.oracle_lib import ORACLE_DIR, REF_SRC, Oracle, run_pipeline
from trinity_b200 import meshgen

REF_DECIDE = os.path.join(ORACLE_DIR, "_ref", "trinity_ref_decide")
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "ref_stage_digests.json")))

needs_ref = pytest.mark.skipif(not os.path.exists(REF_DECIDE), reason="reference build (oracle/_ref) absent")


def reference_decisions(mesh_path, bb_path, params, tmp_path):
    """Run the recording reference build on one thread; its decision stream."""
    out = str(tmp_path / "decisions.bin")
    subprocess.run([REF_DECIDE, mesh_path, bb_path, str(params["rounds"]), str(params["depth"]),
                    str(params["bucket"]), str(params["target"]), str(params["norm"])],
                   check=True, capture_output=True, timeout=600,
                   env=dict(os.environ, OMP_NUM_THREADS="1", TRN_DECISIONS_OUT=out))
    return np.fromfile(out, dtype=np.int32)


def split_log(log):
    """(tag, count) of each record of a decision stream, in order."""
    recs, i = [], 0
    while i < len(log):
        tag, n = int(log[i]), int(log[i + 1])
        i += 2
        if tag == 1:
            i += n
        elif tag == 2:
            i += 2 * n
        elif tag == 3:
            for _ in range(n):
                i += 1 + int(log[i])
        else:
            raise AssertionError(f"unknown record tag {tag} at word {i - 2}")
        recs.append((tag, n))
    assert i == len(log)
    return recs


def _compare(m, u, params, tmp_path):
    mp, bp = str(tmp_path / "in.mesh"), str(tmp_path / "in.bb")
    meshgen.write_mesh(mp, m)
    meshgen.write_bb(bp, u)
    ref = reference_decisions(mp, bp, params, tmp_path)
    o = Oracle(m, u, capa_scale=9, bucket=params["bucket"])
    run_pipeline(o, params)
    log = o.log()
    recs = split_log(ref)
    # every round colors once, coarsens and swaps at least one level
    assert sum(1 for t, _ in recs if t == 3) == params["rounds"]
    assert any(t == 1 for t, _ in recs) and any(t == 2 for t, _ in recs)
    assert recs == split_log(log)
    assert np.array_equal(ref, log)


@needs_ref
@pytest.mark.parametrize("name", ["c1", "c2_n60", "c4_n50", "c2"])
def test_oracle_log_is_the_reference_decisions(oracle_built, name, tmp_path):
    g = GOLD[name]
    m, u, c = meshgen.make_config(g["config"]["name"], g["config"]["n"])
    params = dict(c)
    params.update(g["params"])
    _compare(m, u, params, tmp_path)


@needs_ref
@pytest.mark.skipif(not os.path.isdir(os.path.join(REF_SRC, "examples")),
                    reason="trinity's own GRID4 fixture is only readable where the reference is mounted")
def test_oracle_log_is_the_reference_decisions_on_grid4_fixture(oracle_built, tmp_path):
    g = GOLD["grid4_shock4"]
    m = meshgen.read_mesh(os.path.join(REF_SRC, g["fixture"]["mesh"]))
    u = meshgen.read_bb(os.path.join(REF_SRC, g["fixture"]["bb"]), m.nb_nodes)
    _compare(m, u, dict(g["params"]), tmp_path)
