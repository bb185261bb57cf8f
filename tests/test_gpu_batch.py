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
