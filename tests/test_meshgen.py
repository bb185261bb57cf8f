"""Synthetic workload generator: sizes, orientation, boundary, file round trip."""
import numpy as np

from tests.helpers import signed_areas
from trinity_b200 import meshgen


def test_c1_sizes_and_orientation():
    m, u, c = meshgen.make_config("c1")
    assert (m.nb_nodes, m.nb_elems) == (10201, 20000)
    assert np.all(signed_areas(m.points, m.tris) > 0)
    assert m.edges.shape == (400, 2) and m.corners.shape == (4,)
    assert u.shape == (10201,) and np.all(np.abs(u) <= 1.0)


def test_jitter_is_bounded_and_interior_only():
    m0 = meshgen.grid_mesh(50)
    m1 = meshgen.grid_mesh(50, jitter=0.3, seed=4)
    d = np.abs(m1.points - m0.points)
    assert d.max() <= 0.3 / 50 + 1e-15
    b = np.unique(m0.edges)
    assert np.all(d[b] == 0)
    assert np.all(signed_areas(m1.points, m1.tris) > 0)


def test_mesh_and_bb_round_trip(tmp_path):
    m, u, c = meshgen.make_config("c4", 20)
    mp, bp = str(tmp_path / "x.mesh"), str(tmp_path / "x.bb")
    meshgen.write_mesh(mp, m)
    meshgen.write_bb(bp, u)
    r = meshgen.read_mesh(mp)
    assert np.array_equal(r.points, m.points) and np.array_equal(r.tris, m.tris)
    assert np.array_equal(r.edges, m.edges) and np.array_equal(r.corners, m.corners)
    assert np.array_equal(meshgen.read_bb(bp, m.nb_nodes), u)


def test_batch_specs_deterministic():
    a, b = meshgen.batch_specs(), meshgen.batch_specs()
    assert a == b and len(a) == 256
    sides = [s for s, _, _ in a]
    assert min(sides) >= 32 and max(sides) <= 512
