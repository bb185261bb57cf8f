"""Boundary I/O on the GPU path: loading the .mesh/.bb files gives the same
state as loading arrays, and after a replayed adaptation Mesh::store writes
the same bytes as the reference's Mesh::store (digest from the reference)."""
import hashlib
import json
import os
import subprocess

import pytest

from tests.helpers import gpu_state, oracle_run, run_gpu_stages
from tests.oracle_lib import tags_of
from trinity_b200 import meshgen

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "ref_stage_digests.json")))


@pytest.mark.gpu
def test_file_load_equals_array_load(tmp_path):
    from trinity_b200.api import Mesh
    m, u, c = meshgen.make_config("c4", 30)
    mp, bp = str(tmp_path / "a.mesh"), str(tmp_path / "a.bb")
    meshgen.write_mesh(mp, m)
    meshgen.write_bb(bp, u)
    a = Mesh((m.nb_nodes, m.nb_elems), 64, 1, 0, 1)
    a.load(mp, bp)
    b = Mesh((m.nb_nodes, m.nb_elems), 64, 1, 0, 1)
    b.load_arrays(m.points, m.tris, tags_of(m), u)
    assert not gpu_state(a).diff(gpu_state(b))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c1", "c2_n60"])
def test_store_after_replay_matches_reference_store(oracle_built, tmp_path, name):
    g0 = GOLD[name]
    m, u, c, states, log = oracle_run(g0["config"]["name"], g0["config"]["n"], g0["params"]["rounds"])
    from tests.helpers import gpu_mesh
    g = gpu_mesh(m, u, c)
    g.set_replay(log)
    run_gpu_stages(g, c, lambda s: None)
    out = str(tmp_path / "out.mesh")
    g.store(out)
    assert hashlib.sha256(open(out, "rb").read()).hexdigest() == g0["store_sha256"]


@pytest.mark.gpu
def test_export_compact_is_store_numbering(oracle_built):
    import numpy as np
    m, u, c, states, log = oracle_run("c1", 40, 2)
    from tests.helpers import gpu_mesh
    g = gpu_mesh(m, u, c)
    run_gpu_stages(g, c, lambda s: None)
    pts, ten, tri, alive, tags = g.export()
    newid = np.cumsum(alive.astype(np.int64)) - 1
    live = tri[tri[:, 0] >= 0]
    p2, t2, m2 = g.export_compact()
    assert np.array_equal(p2, pts[alive == 1]) and np.array_equal(m2, ten[alive == 1])
    assert np.array_equal(t2, newid[live].astype(np.int32))


@pytest.mark.gpu
def test_load_rejects_out_of_range_vertex():
    import numpy as np
    from trinity_b200.api import Mesh, TrinityError
    m, u, c = meshgen.make_config("c1", 10)
    bad = m.tris.copy()
    bad[5, 1] = m.nb_nodes + 3
    g = Mesh((m.nb_nodes, m.nb_elems), 64, 1, 0, 1)
    with pytest.raises(TrinityError):
        g.load_arrays(m.points, bad, tags_of(m), u)
    g.load_arrays(m.points, m.tris, tags_of(m), u)   # and recovers with valid input


@pytest.mark.gpu
def test_cli_runs_the_reference_command_line(tmp_path):
    exe = os.path.join(os.path.dirname(HERE), "trinity_b200", "bin", "trinity")
    mp, bp, c = meshgen.write_config("c1", str(tmp_path), 50)
    out = str(tmp_path / "adapted.mesh")
    r = subprocess.run([exe, "-i", mp, "-s", bp, "-o", out, "-b", "64", "-t", "0.9", "-p", "2",
                        "-r", "2", "-d", "1", "-v", "1"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "recap" in r.stdout
    res = meshgen.read_mesh(out) if False else None
    txt = open(out).read()
    assert txt.startswith("MeshVersionFormatted 1") and "RequiredVertices" in txt
    assert os.path.exists(str(tmp_path / "adapted.sol"))


@pytest.mark.gpu
def test_store_and_sol_give_the_in_memory_histogram(tmp_path):
    """Mesh::store's .mesh and the .sol beside it, read back by the histogram
    tool: the same tensors (17 digits) in the .mesh vertex order, and the
    in-memory mesh's metric edge-length histogram (coordinates are stored
    with 8 decimals, so bin counts may move by a few edges)."""
    import numpy as np
    from tests.helpers import gpu_mesh, in_range_fraction, run_gpu_stages
    from trinity_b200 import histogram
    m, u, c = meshgen.make_config("c2", 80)
    g = gpu_mesh(m, u, c)
    run_gpu_stages(g, c, lambda s: None)
    mp, sp = str(tmp_path / "a.mesh"), str(tmp_path / "a.sol")
    g.store(mp)
    g.store_sol(sp)
    pts, tri, ten = g.export_compact()
    sol = histogram.read_sol(sp)
    assert np.array_equal(sol.view(np.uint64), np.ascontiguousarray(ten).view(np.uint64))
    h = histogram.of_files(mp, sp)
    mem = histogram.histogram(pts, tri, ten)
    assert h["triangles"] == tri.shape[0] and h["vertices"] == pts.shape[0]
    assert np.abs(np.array(h["fractions"]) - np.array(mem["fractions"])).max() < 1e-3
    assert abs(h["in_range_fraction"] - in_range_fraction(gpu_state(g))) < 1e-3
    g.close()
