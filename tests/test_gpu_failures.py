"""Failure paths of the C ABI, made on the host (malformed files, a capacity
set too small, a level cap set to 1): each call returns its TRN_ERR_* code
with a message, and the same mesh handle loads and adapts again afterwards.
The reference aborts or exits in these cases (src/parser.cpp:130-141,
src/io.cpp:53-161) or, for a too small capacity, writes out of bounds
(src/mesh.cpp:57-133); no kernel here writes outside its buffers or waits:
the capacity check is a device-side bound, the level cap a counter."""
import pytest

from tests.oracle_lib import tags_of
from trinity_b200 import meshgen

ERR_CAPACITY, ERR_IO, ERR_NO_PROGRESS = 1, 2, 4


def _mesh(m, capa_scale=None, depth=1):
    from trinity_b200.api import Mesh
    return Mesh((m.nb_nodes, m.nb_elems), 64, depth, 0, 1, capa_scale=capa_scale)


def _adapts(g, c):
    """metric + one round on a freshly loaded mesh, no error"""
    from trinity_b200.api import Coarse, Metrics, Partit, Refine, Smooth, Swap
    heur = Partit(g, 8)
    Metrics(g, c["target"], c["norm"]).run()
    for k in (Refine(g, 1), Coarse(g, heur), Swap(g), Smooth(g, heur, 1)):
        k.run()
    return g.counts()


@pytest.mark.gpu
def test_truncated_mesh_file_is_an_io_error(tmp_path):
    from trinity_b200.api import TrinityError
    m, u, c = meshgen.make_config("c1", 20)
    mp, bp = str(tmp_path / "a.mesh"), str(tmp_path / "a.bb")
    meshgen.write_mesh(mp, m)
    meshgen.write_bb(bp, u)
    txt = open(mp).read()
    cut = str(tmp_path / "cut.mesh")
    open(cut, "w").write(txt[: txt.index("Triangles") + len("Triangles\n") + 200])
    g = _mesh(m)
    with pytest.raises(TrinityError) as e:
        g.load(cut, bp)
    assert e.value.code == ERR_IO and "truncated" in str(e.value)
    g.load(mp, bp)
    assert _adapts(g, c)[1] > 0


@pytest.mark.gpu
def test_solution_count_differing_from_the_mesh_is_an_io_error(tmp_path):
    from trinity_b200.api import TrinityError
    m, u, c = meshgen.make_config("c1", 20)
    mp, bp = str(tmp_path / "a.mesh"), str(tmp_path / "a.bb")
    meshgen.write_mesh(mp, m)
    meshgen.write_bb(bp, u[:-5])
    g = _mesh(m)
    with pytest.raises(TrinityError) as e:
        g.load(mp, bp)
    assert e.value.code == ERR_IO and "number of vertices" in str(e.value)
    meshgen.write_bb(bp, u)
    g.load(mp, bp)
    assert _adapts(g, c)[1] > 0


@pytest.mark.gpu
def test_capacity_too_small_for_refinement_is_reported(tmp_path):
    """capacity 1x the input: the first refinement that adds vertices fails
    its device-side capacity check with TRN_ERR_CAPACITY, writes nothing past
    the slots, and a reload restores a working mesh on the same handle."""
    from trinity_b200.api import Metrics, Refine, TrinityError
    m, u, c = meshgen.make_config("c1", 30)
    g = _mesh(m, capa_scale=1)
    g.load_arrays(m.points, m.tris, tags_of(m), u)
    Metrics(g, c["target"], c["norm"]).run()
    with pytest.raises(TrinityError) as e:
        Refine(g, 1).run()
    assert e.value.code == ERR_CAPACITY and "capacity" in str(e.value)
    g.load_arrays(m.points, m.tris, tags_of(m), u)
    Metrics(g, c["target"], c["norm"]).run()   # the error word was cleared by the load
    assert g.counts()[:2] == (m.nb_nodes, m.nb_elems)


@pytest.mark.gpu
@pytest.mark.parametrize("stage", ["coarse", "swap"])
def test_level_cap_reached_is_no_progress(stage):
    from trinity_b200.api import Coarse, Metrics, Partit, Refine, Swap, TrinityError
    m, u, c = meshgen.make_config("c2", 60)
    g = _mesh(m, capa_scale=9, depth=2)
    g.load_arrays(m.points, m.tris, tags_of(m), u)
    Metrics(g, c["target"], c["norm"]).run()
    Refine(g, 2).run()
    g.set_level_cap(1)
    k = Coarse(g, Partit(g, 8)) if stage == "coarse" else Swap(g)
    with pytest.raises(TrinityError) as e:
        k.run()
    assert e.value.code == ERR_NO_PROGRESS and "level cap" in str(e.value)
    g.set_level_cap(100000)
    g.load_arrays(m.points, m.tris, tags_of(m), u)
    assert _adapts(g, c)[1] > 0


@pytest.mark.gpu
def test_level_cap_must_be_positive():
    from trinity_b200.api import TrinityError
    m, u, c = meshgen.make_config("c1", 10)
    g = _mesh(m)
    with pytest.raises(TrinityError):
        g.set_level_cap(0)


@pytest.mark.gpu
def test_grid_barrier_wait_runs_out_and_is_reported():
    """The cooperative heuristics separate their rounds by a grid barrier
    whose wait is bounded. A cooperative launch in which one block never
    arrives: the others give up after 4,096 polls and mark the failure
    (TRN_ERR_NO_PROGRESS), and the context stays usable: a mesh then adapts
    with the cooperative rounds as before (a 300x300 mesh lists more than
    1,024 collapse candidates, so its independent sets take the cooperative
    launch)."""
    from trinity_b200 import _lib
    L = _lib.lib()
    assert L.trn_selftest_barrier(4096) == ERR_NO_PROGRESS
    m, u, c = meshgen.make_config("c1", 300)
    g = _mesh(m)
    g.load_arrays(m.points, m.tris, tags_of(m), u)
    counts = _adapts(g, c)
    assert counts[3] > 0
    g.close()
