"""Replay parity: the GPU fed the oracle's independent sets, matchings and
colorings reproduces the reference's 1-thread run bit for bit after every
stage (metric tensors and points, element array, vertex liveness and tags)."""
import pytest

from tests.helpers import gpu_mesh, gpu_state, oracle_run, run_gpu_stages

CASES = [("c1", 40, 2), ("c1", None, 3), ("c2", 60, 2), ("c4", 50, 2)]


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
@pytest.mark.parametrize("lanes,prec", [(4, "fp64"), (8, "fp64"), (8, "mixed")])
def test_grouped_smoothing_same_results(oracle_built, lanes, prec):
    """4 or 8 lanes per smoothed vertex give the one-lane results after every
    stage: FP64 in replay, bit-identical to the oracle too; the mixed form
    (free mode only) identical to its one-lane run."""
    m, u, c, states, log = oracle_run("c2", 60, 2)
    runs = {}
    for ln in (1, lanes):
        g = gpu_mesh(m, u, c)
        if prec == "fp64":
            g.set_replay(log)
        g.set_precision(prec)
        t = g.get_tune()
        t["smooth_lanes"] = ln
        g.set_tune(t)
        snaps = {}
        run_gpu_stages(g, c, lambda s: snaps.__setitem__(s, gpu_state(g)))
        runs[ln] = snaps
        g.close()
    for stage, st in runs[lanes].items():
        assert not st.diff(runs[1][stage]), stage
        if prec == "fp64":
            assert not st.diff(states[stage]), stage
