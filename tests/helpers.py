"""Shared test helpers: oracle runs with per-stage snapshots, GPU runs through
the C ABI, and mesh invariants (conformity, orientation, metric edge lengths)."""
from __future__ import annotations

import functools

import numpy as np

from tests import oracle_lib
from tests.oracle_lib import Oracle, State, tags_of
from trinity_b200 import meshgen

STAGES = ("refine", "coarse", "swap", "smooth")


@functools.lru_cache(maxsize=8)
def oracle_run(name: str, n: int | None = None, rounds: int | None = None):
    """Run the oracle on a named workload; returns (mesh, field, params, states, log)."""
    m, u, c = meshgen.make_config(name, n)
    c = dict(c)
    if rounds is not None:
        c["rounds"] = rounds
    o = Oracle(m, u, capa_scale=9, bucket=c["bucket"])
    states = {}

    def snap(stage):
        states[stage] = o.state()

    oracle_lib.run_pipeline(o, c, log_stage=snap)
    return m, u, c, states, o.log()


def gpu_mesh(m, u, c, capa_scale=9):
    from trinity_b200.api import Mesh
    g = Mesh((m.nb_nodes, m.nb_elems), c["bucket"], c["depth"], 0, c["rounds"], capa_scale=capa_scale)
    g.load_arrays(m.points, m.tris, tags_of(m), u)
    return g


def gpu_state(g) -> State:
    pts, ten, tri, alive, tags = g.export()
    return State(pts, ten, tri, alive, tags)


def run_gpu_stages(g, c, on_stage):
    from trinity_b200.api import Coarse, Metrics, Partit, Refine, Smooth, Swap
    heur = Partit(g, 8)
    Metrics(g, c["target"], c["norm"]).run()
    on_stage("metric")
    k = {"refine": Refine(g, c["depth"]), "coarse": Coarse(g, heur), "swap": Swap(g),
         "smooth": Smooth(g, heur, c["depth"])}
    for r in range(c["rounds"]):
        for s in STAGES:
            k[s].run()
            on_stage(f"r{r}.{s}")


def signed_areas(pts, tri):
    a, b, c = pts[tri[:, 0]], pts[tri[:, 1]], pts[tri[:, 2]]
    return 0.5 * ((b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (c[:, 0] - a[:, 0]) * (b[:, 1] - a[:, 1]))


def check_invariants(st: State, bound_tag: int = 4):
    """Conforming, positively oriented, every referenced vertex alive, closed
    boundary made of boundary-tagged vertices, Euler characteristic of a disk."""
    tri = st.active_elems()
    assert tri.shape[0] > 0
    assert np.all(st.alive[tri.ravel()] == 1), "element references a deleted vertex"
    assert np.all(tri[:, 0] != tri[:, 1]) and np.all(tri[:, 1] != tri[:, 2]) and np.all(tri[:, 0] != tri[:, 2])
    ar = signed_areas(st.points, tri)
    assert np.all(ar > 1e-9), f"{int(np.sum(ar <= 1e-9))} elements not CCW"
    e = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]])
    key = e[:, 0].astype(np.int64) * (1 << 32) + e[:, 1]
    assert np.unique(key).shape[0] == key.shape[0], "a directed edge appears twice"
    rkey = e[:, 1].astype(np.int64) * (1 << 32) + e[:, 0]
    bnd = ~np.isin(rkey, key)
    be = e[bnd]
    assert np.all(st.tags[be.ravel()] & bound_tag), "open edge between interior vertices"
    used = np.unique(tri.ravel())
    n_edges = (key.shape[0] + int(bnd.sum())) // 2
    assert used.shape[0] - n_edges + tri.shape[0] == 1, "Euler characteristic is not 1"
    live = np.flatnonzero(st.alive)
    assert np.array_equal(np.sort(used), live), "alive vertex without element"


def metric_lengths(st: State):
    """Metric length of every undirected edge (numeric.cpp:469-497 formula, numpy)."""
    tri = st.active_elems()
    e = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]])
    e = np.unique(np.sort(e, axis=1), axis=0)
    pa, pb = st.points[e[:, 0]], st.points[e[:, 1]]
    ta, tb = st.tensor[e[:, 0]], st.tensor[e[:, 1]]
    w = pb - pa
    l0 = np.sqrt(w[:, 0] * (ta[:, 0] * w[:, 0] + ta[:, 1] * w[:, 1]) + w[:, 1] * (ta[:, 1] * w[:, 0] + ta[:, 2] * w[:, 1]))
    l1 = np.sqrt(w[:, 0] * (tb[:, 0] * w[:, 0] + tb[:, 1] * w[:, 1]) + w[:, 1] * (tb[:, 1] * w[:, 0] + tb[:, 2] * w[:, 1]))
    lo, hi = np.minimum(l0, l1), np.maximum(l0, l1)
    r = hi / lo
    with np.errstate(divide="ignore", invalid="ignore"):
        geo = hi * (r - 1) / (r * np.log(r))
    return np.where(np.abs(l0 - l1) < 1e-9, l0, geo)


def in_range_fraction(st: State) -> float:
    L = metric_lengths(st)
    return float(np.mean((L >= 1 / np.sqrt(2)) & (L <= np.sqrt(2))))
