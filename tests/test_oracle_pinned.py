"""The oracle is pinned to trinity itself: after the metric and after every
kernel of every round, its full-precision state hashes to the same digest as
the reference's (1 thread, built from its own sources; fixtures written by
tests/golden/make_golden.py)."""
import json
import os

import pytest

from tests.oracle_lib import REF_EXACT as REF_EXACT_BIN
from tests.oracle_lib import REF_SRC, Oracle, digest, run_pipeline
from trinity_b200 import meshgen

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "ref_stage_digests.json")))


def _check(name, m, u, params, bucket):
    want = GOLD[name]["stages"]
    o = Oracle(m, u, capa_scale=9, bucket=bucket)
    assert digest(o.state()) == want["load"], f"{name}: load"

    def check(stage):
        got = digest(o.state())
        assert got == want[stage], f"{name}: stage {stage} differs from the reference"

    run_pipeline(o, params, log_stage=check)


@pytest.mark.parametrize("name", ["c1", "c2_n60", "c4_n50", "c2"])
def test_oracle_matches_reference_digests(oracle_built, name):
    g = GOLD[name]
    m, u, c = meshgen.make_config(g["config"]["name"], g["config"]["n"])
    params = dict(c)
    params.update(g["params"])
    _check(name, m, u, params, g["params"]["bucket"])


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF_SRC, "examples")),
                    reason="trinity's own GRID4 fixture is only readable where the reference is mounted")
def test_oracle_matches_reference_on_grid4_fixture(oracle_built):
    g = GOLD["grid4_shock4"]
    m = meshgen.read_mesh(os.path.join(REF_SRC, g["fixture"]["mesh"]))
    u = meshgen.read_bb(os.path.join(REF_SRC, g["fixture"]["bb"]), m.nb_nodes)
    _check("grid4_shock4", m, u, g["params"], g["params"]["bucket"])


@pytest.mark.skipif(not os.path.exists(REF_EXACT_BIN), reason="reference build (oracle/_ref) absent")
def test_harness_final_snapshot_is_last_stage(oracle_built, tmp_path):
    """The harness's --final snapshot (read by the reference-build comparison
    of the free mode) is the state after the last kernel of the last round,
    the same as the oracle's."""
    import subprocess
    from tests.oracle_lib import read_snapshot
    m, u, c = meshgen.make_config("c2", 40)
    mp, bp = str(tmp_path / "m.mesh"), str(tmp_path / "m.bb")
    meshgen.write_mesh(mp, m)
    meshgen.write_bb(bp, u)
    pre, fin = str(tmp_path / "d"), str(tmp_path / "final.bin")
    subprocess.run([REF_EXACT_BIN, mp, bp, "2", str(c["depth"]), str(c["bucket"]), str(c["target"]),
                    str(c["norm"]), "--capa-depth", "4", "--dump", pre, "--final", fin],
                   check=True, capture_output=True, timeout=300,
                   env=dict(os.environ, OMP_NUM_THREADS="1"))
    last = read_snapshot(pre + ".r1.smooth.bin")
    final = read_snapshot(fin)
    assert not final.diff(last)
    params = dict(c)
    params["rounds"] = 2
    o = Oracle(m, u, capa_scale=9, bucket=c["bucket"])
    run_pipeline(o, params)
    assert digest(o.state()) == digest(final)
