"""The oracle is pinned to trinity itself: after the metric and after every
kernel of every round, its full-precision state hashes to the same digest as
the reference's (1 thread, built from its own sources; fixtures written by
tests/golden/make_golden.py)."""
import json
import os

import pytest

from tests.oracle_lib import Oracle, digest, run_pipeline
from trinity_b200 import meshgen

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "ref_stage_digests.json")))
REF_SRC = "/root/reference"


def _check(name, m, u, params, bucket):
    want = GOLD[name]["stages"]
    o = Oracle(m, u, capa_scale=9, bucket=bucket)
    assert digest(o.state()) == want["load"], f"{name}: load"

    def check(stage):
        got = digest(o.state())
        assert got == want[stage], f"{name}: stage {stage} differs from the reference"

    run_pipeline(o, params, log_stage=check)


@pytest.mark.parametrize("name", ["c1", "c2_n60", "c4_n50"])
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
