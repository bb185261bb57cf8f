"""The metric edge-length histogram tool (trinity_b200/histogram.py) on a
mesh whose lengths are known: the 20 x 20 unit-square grid under the metric
(1/h^2) I has axis edges of length 1 and diagonals of length sqrt 2."""
import json
import subprocess
import sys

import numpy as np
import pytest

from trinity_b200 import histogram, meshgen


def _write_sol(path, ten):
    with open(path, "w") as f:
        f.write(f"MeshVersionFormatted 1\nDimension 2\nSolAtVertices\n{ten.shape[0]}\n1 3\n")
        for t in ten:
            f.write("%.17g %.17g %.17g\n" % tuple(t))
        f.write("\nEnd\n")


def test_known_lengths(tmp_path):
    n = 20
    m, u, c = meshgen.make_config("c1", n)
    mp, sp = str(tmp_path / "g.mesh"), str(tmp_path / "g.sol")
    meshgen.write_mesh(mp, m)
    ten = np.tile([n * n, 0.0, n * n], (m.nb_nodes, 1)).astype(np.float64)
    _write_sol(sp, ten)
    h = histogram.of_files(mp, sp)
    axis, diag = 2 * n * (n + 1), n * n
    assert h["edges_total"] == axis + diag
    counts = dict(zip(zip(h["edges"][:-1], h["edges"][1:]), h["counts"]))
    # axis edges have length 1 up to the rounding of the coordinates i/n
    assert counts[(0.85, 1.0)] + counts[(1.0, 1.2)] == axis
    assert counts[(1.2, 2 ** 0.5)] + counts[(2 ** 0.5, 2.0)] == diag
    # every axis edge is in range; a diagonal is at sqrt 2, in or out by rounding
    assert axis / (axis + diag) <= h["in_range_fraction"] <= 1.0


def test_cli_compares_two_pairs(tmp_path):
    n = 12
    m, u, c = meshgen.make_config("c1", n)
    mp, sp, sp2 = str(tmp_path / "g.mesh"), str(tmp_path / "a.sol"), str(tmp_path / "b.sol")
    meshgen.write_mesh(mp, m)
    _write_sol(sp, np.tile([n * n, 0.0, n * n], (m.nb_nodes, 1)).astype(np.float64))
    _write_sol(sp2, np.tile([4 * n * n, 0.0, 4 * n * n], (m.nb_nodes, 1)).astype(np.float64))
    r = subprocess.run([sys.executable, "-m", "trinity_b200.histogram", mp, sp, "--against", mp, sp2],
                       capture_output=True, text=True, check=True)
    out = json.loads(r.stdout)
    assert out["max_abs_difference"] > 0.5          # every edge moved to a bin twice as long
    assert abs(sum(out["difference"])) < 1e-12


def test_wrong_sol_layout_is_refused(tmp_path):
    p = str(tmp_path / "bad.sol")
    open(p, "w").write("MeshVersionFormatted 1\nDimension 2\nSolAtVertices\n2\n1 1\n1.0\n2.0\nEnd\n")
    with pytest.raises(ValueError):
        histogram.read_sol(p)
