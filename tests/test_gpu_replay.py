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
