"""Replay parity: the GPU fed the oracle's independent sets, matchings and
colorings reproduces the reference's 1-thread run bit for bit after every
stage (metric tensors and points, element array, vertex liveness and tags)."""
import json
import os

import numpy as np
import pytest

from tests.helpers import gpu_mesh, gpu_state, oracle_run, run_gpu_stages
from tests.oracle_lib import Oracle, digest, run_pipeline
from tests.test_reference_decisions import REF_DECIDE, reference_decisions
from trinity_b200 import meshgen

CASES = [("c1", 40, 2), ("c1", None, 3), ("c2", 60, 2), ("c4", 50, 2)]
GOLD = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                   "ref_stage_digests.json")))


@pytest.mark.gpu
@pytest.mark.parametrize("name,n,rounds", CASES)
def test_replay_bit_exact(oracle_built, name, n, rounds):
    m, u, c, states, log = oracle_run(name, n, rounds)
    g = gpu_mesh(m, u, c)
    g.set_replay(log)
    seen = []

    def check(stage):
        d = gpu_state(g).diff(states[stage])
        assert not d, f"{name} n={n} stage {stage}: {d}"
        seen.append(stage)

    run_gpu_stages(g, c, check)
    assert len(seen) == 1 + 4 * c["rounds"]


@pytest.mark.gpu
@pytest.mark.parametrize("lanes,prec,regs", [(4, "fp64", 2), (8, "fp64", 2), (8, "mixed", 2), (4, "fp64", 4),
                                             (4, "mixed", 6), (2, "fp64", 5), (2, "fp64", 7), (4, "mixed", 8)])
def test_grouped_smoothing_same_results(oracle_built, lanes, prec, regs):
    """2, 4 or 8 lanes per smoothed vertex, the tries in turn or in one sweep
    (smooth_regs 4-8), give the one-lane results after every stage: FP64 in
    replay, bit-identical to the oracle too; the mixed form (free mode only)
    identical to its one-lane run."""
    m, u, c, states, log = oracle_run("c2", 60, 2)
    runs = {}
    for ln in (1, lanes):
        g = gpu_mesh(m, u, c)
        if prec == "fp64":
            g.set_replay(log)
        g.set_precision(prec)
        t = g.get_tune()
        t["smooth_lanes"] = ln
        t["smooth_regs"] = regs if ln > 1 else 2
        g.set_tune(t)
        snaps = {}
        run_gpu_stages(g, c, lambda s: snaps.__setitem__(s, gpu_state(g)))
        runs[ln] = snaps
        g.close()
    for stage, st in runs[lanes].items():
        assert not st.diff(runs[1][stage]), stage
        if prec == "fp64":
            assert not st.diff(states[stage]), stage


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF_DECIDE), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("name", ["c2_n60", "c4_n50"])
def test_replay_of_the_reference_decisions_matches_reference_digests(name, tmp_path):
    """No oracle in the loop: the GPU is fed the independent sets, matchings
    and colorings that trinity's own build records on one thread
    (oracle/_ref/trinity_ref_decide), and its state after the metric and
    after every stage hashes to the digests of the reference's run."""
    gold = GOLD[name]
    m, u, c = meshgen.make_config(gold["config"]["name"], gold["config"]["n"])
    params = dict(c)
    params.update(gold["params"])
    mp, bp = str(tmp_path / "in.mesh"), str(tmp_path / "in.bb")
    meshgen.write_mesh(mp, m)
    meshgen.write_bb(bp, u)
    log = reference_decisions(mp, bp, params, tmp_path)
    want = gold["stages"]
    g = gpu_mesh(m, u, params)
    assert digest(gpu_state(g)) == want["load"], "load"
    g.set_replay(log)
    seen = []

    def check(stage):
        got = digest(gpu_state(g))
        bad = [k for k in got if got[k] != want[stage][k]]
        assert not bad, f"{name} stage {stage}: {bad} differ from the reference"
        seen.append(stage)

    run_gpu_stages(g, params, check)
    g.close()
    assert len(seen) == 1 + 4 * params["rounds"]


@pytest.mark.gpu
def test_replay_full_size_workload_matches_reference_digests(oracle_built):
    """The full 2M-triangle workload (1000 x 1000 jittered grid, depth 2,
    bucket 128, target 0.7, L^2, 3 rounds): fed the oracle's decisions, the
    GPU's state after the metric and after every stage of every round hashes
    to the digests of the reference's own 1-thread run (written by
    tests/golden/make_golden.py), so capacity, bucket and id-ordering effects
    that only appear at this size are covered too."""
    want = GOLD["c2"]["stages"]
    m, u, c = meshgen.make_config("c2")
    o = Oracle(m, u, capa_scale=9, bucket=c["bucket"])
    run_pipeline(o, c)
    log = o.log()
    del o
    g = gpu_mesh(m, u, c)
    assert digest(gpu_state(g)) == want["load"], "load"
    g.set_replay(log)
    seen = []

    def check(stage):
        got = digest(gpu_state(g))
        bad = [k for k in got if got[k] != want[stage][k]]
        assert not bad, f"stage {stage}: {bad} differ from the reference"
        seen.append(stage)

    run_gpu_stages(g, c, check)
    g.close()
    assert len(seen) == 1 + 4 * c["rounds"]


@pytest.mark.gpu
@pytest.mark.parametrize("name,n", [("c1", None), ("c2", 120)])
def test_free_swap_matching_is_the_oracle_interleaved_greedy(oracle_built, name, n):
    """The free mode's swap matching computes the reference's greedy loop over
    the candidates in the order (id mod 4, id) exactly: from the same state
    (the oracle's decisions replayed through the metric, refinement and
    coarsening of the first round), a free-mode swap stage ends bit-identical
    to the oracle's swap stage run with that rule (ORC_SWAP_GREEDY_INTERLEAVED),
    every level's candidates, rows, matching and flips included. The oracle
    also takes the free mode's re-activation rule (a flip re-activates its
    partner's row only when that row is of the current level)."""
    from trinity_b200.api import Coarse, Metrics, Partit, Refine, Swap
    m, u, c = meshgen.make_config(name, n)
    c = dict(c, rounds=1)
    o = Oracle(m, u, capa_scale=9, bucket=c["bucket"])
    o.metric(c["target"], c["norm"])
    o.refine(c["depth"])
    o.coarsen()
    log = o.log()
    o.set_swap_rule("greedy_interleaved")
    o.set_swap_strict_map(True)
    o.swap()
    want = o.state()
    g = gpu_mesh(m, u, c)
    g.set_replay(log)
    heur = Partit(g, 8)
    Metrics(g, c["target"], c["norm"]).run()
    Refine(g, c["depth"]).run()
    Coarse(g, heur).run()
    g.set_replay(np.zeros(0, np.int32))   # free mode from here on
    g.set_swap_match("greedy")
    Swap(g).run()
    d = gpu_state(g).diff(want)
    assert not d, d
    g.close()
