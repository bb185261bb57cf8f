"""The solver-coupled loop (the adaptive loop trinity is meant to run in,
README.md:8 of the reference; its scripts/bench_run.py:77-110 closes it through
Mesh::store and a fresh Mesh::load): adapt, renumber the adapted mesh as
store + load would, evaluate a new field on it, recover the metric, adapt
again. Replayed with the oracle's decisions, the GPU is bit-identical to the
oracle after every stage of both cycles and right after the renumbering; the
oracle's second cycle starts from the same renumbering done in numpy and
loaded like any input."""
from types import SimpleNamespace

import numpy as np
import pytest

from tests.helpers import check_invariants, gpu_mesh, gpu_state, run_gpu_stages
from tests.oracle_lib import Oracle, compact_state, run_pipeline
from trinity_b200 import meshgen


def _oracle_cycle(mesh, u, c, tags=None):
    o = Oracle(mesh, u, capa_scale=9, bucket=c["bucket"], tags=tags)
    load = o.state()
    states = {}
    run_pipeline(o, c, log_stage=lambda s: states.__setitem__(s, o.state()))
    return load, states, o.log(), o.state()


@pytest.mark.gpu
def test_two_cycles_replay_bit_exact(oracle_built):
    m, u, c = meshgen.make_config("c1", 40)
    c = dict(c, rounds=2)
    _, states1, log1, end1 = _oracle_cycle(m, u, c)
    pts2, tri2, tags2 = compact_state(end1)
    u2 = meshgen.field_shock(pts2, a=50.0, b=0.3)    # the front has moved
    mesh2 = SimpleNamespace(nb_nodes=pts2.shape[0], nb_elems=tri2.shape[0], points=pts2, tris=tri2)
    load2, states2, log2, _ = _oracle_cycle(mesh2, u2, c, tags=tags2)

    g = gpu_mesh(m, u, c)
    g.set_replay(log1)

    def check(states):
        def f(stage):
            d = gpu_state(g).diff(states[stage])
            assert not d, f"stage {stage}: {d}"
        return f

    run_gpu_stages(g, c, check(states1))
    g.compact()
    d = gpu_state(g).diff(load2)
    assert not d, f"after the renumbering: {d}"
    g.set_solution(u2)
    g.set_replay(log2)
    run_gpu_stages(g, c, check(states2))
    g.close()


@pytest.mark.gpu
def test_adaptive_loop_free_mode_three_cycles():
    """The library's own loop (api.adaptive_loop), free mode: every cycle ends
    with a valid mesh that follows the moving front (most metric edge lengths
    in [1/sqrt 2, sqrt 2])."""
    from tests.helpers import in_range_fraction
    from trinity_b200.api import adaptive_loop
    m, u, c = meshgen.make_config("c1", 60)
    g = gpu_mesh(m, u, c)
    fronts = [0.2, 0.25, 0.3]
    seen = []

    def on_cycle(k, mesh):
        st = gpu_state(mesh)
        check_invariants(st)
        seen.append((st.active_elems().shape[0], in_range_fraction(st)))

    adaptive_loop(g, lambda p: meshgen.field_shock(p, a=50.0, b=fronts[len(seen)]), cycles=3,
                  target=c["target"], norm=c["norm"], depth=c["depth"], rounds=2, on_cycle=on_cycle)
    assert len(seen) == 3
    for n, f in seen:
        assert n > 0 and f > 0.85, seen
    g.close()
