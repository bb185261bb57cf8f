"""A round captured as one CUDA graph (trn_round_graph_run: the coarsening,
swapping and coloring loops as device-decided loop nodes) ends exactly where
the per-stage calls end, in both arithmetic forms, and stays valid."""
import numpy as np
import pytest

from tests.helpers import check_invariants, gpu_mesh, gpu_state
from tests.oracle_lib import tags_of
from trinity_b200 import meshgen

pytestmark = pytest.mark.gpu


def _rounds(g, c, graph):
    from trinity_b200.api import Coarse, Metrics, Partit, Refine, Smooth, Stats, Swap
    Metrics(g, c["target"], c["norm"]).run()
    heur = Partit(g, 8)
    per_round = []
    for _ in range(c["rounds"]):
        st = (Stats * 4)()
        if graph:
            g.round_graph(c["depth"], st)
        else:
            for k, kern in enumerate((Refine(g, c["depth"]), Coarse(g, heur), Swap(g),
                                      Smooth(g, heur, c["depth"]))):
                kern.run(st[k])
        per_round.append([(s.eval, s.task) for s in st])
    return per_round


@pytest.mark.parametrize("name,n,prec,policy", [("c2", 120, "fp64", "row_order"), ("c2", 120, "mixed", "row_order"),
                                               ("c1", 40, "fp64", "row_order"), ("c2", 120, "fp64", "gain")])
def test_graph_round_equals_stage_calls(name, n, prec, policy):
    m, u, c = meshgen.make_config(name, n)
    out = {}
    for graph in (False, True):
        g = gpu_mesh(m, u, c)
        g.set_precision(prec)
        g.set_swap_match(policy)
        stats = _rounds(g, c, graph)
        out[graph] = (gpu_state(g), stats)
        g.close()
    (a, sa), (b, sb) = out[False], out[True]
    assert not b.diff(a)
    assert sa == sb
    check_invariants(b)


def test_graph_round_replays():
    """later calls replay the captured graph; a new seed recaptures"""
    m, u, c = meshgen.make_config("c2", 80)
    g = gpu_mesh(m, u, c)
    h = gpu_mesh(m, u, c)
    for x in (g, h):
        x.set_options(seed=1234)
    _rounds(g, c, True)
    _rounds(h, c, False)
    assert not gpu_state(g).diff(gpu_state(h))
    for x in (g, h):
        x.reload()
        x.set_options(seed=99)
    _rounds(g, c, True)
    _rounds(h, c, False)
    assert not gpu_state(g).diff(gpu_state(h))


def test_graph_round_rejects_replay_mode():
    from trinity_b200.api import Metrics, TrinityError
    m, u, c = meshgen.make_config("c1", 20)
    g = gpu_mesh(m, u, c)
    g.set_replay(np.array([1, 0], dtype=np.int32))
    Metrics(g, c["target"], c["norm"]).run()
    with pytest.raises(TrinityError):
        g.round_graph(1)


def test_graph_batch_equals_plain_batch():
    from trinity_b200.api import Mesh, batch_adapt
    p = meshgen.BATCH_PARAMS
    items = list(meshgen.batch_meshes(count=8, seed=13, lo=12, hi=48))

    def load():
        out = []
        for mm, uu, _ in items:
            g = Mesh((mm.nb_nodes, mm.nb_elems), p["bucket"], p["depth"], 0, p["rounds"],
                     capa_scale=p["capa_scale"])
            g.load_arrays(mm.points, mm.tris, tags_of(mm), uu)
            out.append(g)
        return out

    plain, graph = load(), load()
    batch_adapt(plain, p["target"], p["norm"], p["rounds"], p["depth"], threads=4)
    batch_adapt(graph, p["target"], p["norm"], p["rounds"], p["depth"], threads=4, graph=True)
    for a, b in zip(plain, graph):
        sa, sb = gpu_state(a), gpu_state(b)
        assert not sb.diff(sa)
        check_invariants(sb)


ODD_TUNE = dict(smooth_threads=64, filter_threads=512, group_lanes=4, group_max=65536, flip_threads=128,
                smooth_lanes=4, smooth_regs=0)


@pytest.mark.parametrize("graph", [False, True])
def test_launch_shapes_change_no_result(graph):
    m, u, c = meshgen.make_config("c2", 100)
    states = []
    for cfg in (None, ODD_TUNE, dict(ODD_TUNE, group_lanes=16, group_max=0, smooth_threads=256, smooth_lanes=8),
                dict(ODD_TUNE, smooth_lanes=1, smooth_regs=1),
                dict(ODD_TUNE, group_lanes=1, smooth_regs=2),
                dict(ODD_TUNE, smooth_lanes=2, smooth_regs=1),
                dict(ODD_TUNE, smooth_threads=256, smooth_regs=3),
                dict(ODD_TUNE, smooth_lanes=2, smooth_regs=3),
                dict(ODD_TUNE, smooth_threads=256, smooth_regs=4),
                dict(ODD_TUNE, smooth_lanes=8, smooth_regs=6),
                dict(ODD_TUNE, smooth_lanes=2, smooth_threads=256, smooth_regs=7),
                dict(ODD_TUNE, smooth_regs=8)):
        g = gpu_mesh(m, u, c)
        if cfg:
            g.set_tune(cfg)
            assert g.get_tune() == cfg
        _rounds(g, c, graph)
        states.append(gpu_state(g))
        g.close()
    for st in states[1:]:
        assert not st.diff(states[0])


def test_autotune_picks_valid_shapes_and_reloads():
    from trinity_b200.api import TrinityError
    m, u, c = meshgen.make_config("c2", 80)
    g = gpu_mesh(m, u, c)
    cfg = g.autotune(c["target"], c["norm"], depth=c["depth"], rounds=1)
    assert cfg["smooth_threads"] in (64, 128, 256) and cfg["group_lanes"] in (4, 8, 16)
    assert cfg["smooth_lanes"] in (1, 2, 4, 8) and cfg["smooth_regs"] in range(9)
    assert g.get_tune() == cfg
    assert g.counts()[:2] == (m.nb_nodes, m.nb_elems)
    ref = gpu_mesh(m, u, c)
    _rounds(g, c, True)
    _rounds(ref, c, False)
    assert not gpu_state(g).diff(gpu_state(ref))
    with pytest.raises(TrinityError):
        g.set_tune(dict(ODD_TUNE, group_lanes=6))
