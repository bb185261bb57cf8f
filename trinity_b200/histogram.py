"""Edge lengths in the metric of an adapted mesh: the quality measure the
free mode is held to (most edges in [1/sqrt 2, sqrt 2], header.h:66-67 of the
reference), from the files a run leaves behind.

The reference's Mesh::store (io.cpp:164-255) writes the mesh without its
metric; ``Mesh.store_sol`` writes the tensors beside it in medit's .sol
layout (SolAtVertices, one symmetric tensor m11 m12 m22 per vertex, in the
vertex order of the .mesh). This module reads the pair and histograms the
metric length of every edge (numeric.cpp:469-497's geometric interpolation of
the lengths under the two end tensors):

    python -m trinity_b200.histogram adapted.mesh adapted.sol
    python -m trinity_b200.histogram a.mesh a.sol --against b.mesh b.sol

prints one JSON object: the bin edges, the fraction of edges per bin, the
in-range fraction, and with --against the per-bin difference to the second
pair and its largest absolute value.
"""
from __future__ import annotations

import argparse
import json
import sys

import numpy as np

from trinity_b200 import meshgen

EDGES = [0.0, 0.5, 2 ** -0.5, 0.85, 1.0, 1.2, 2 ** 0.5, 2.0, float("inf")]


def read_sol(path: str) -> np.ndarray:
    """Tensors (m11, m12, m22) per vertex from a medit .sol with one
    symmetric 2x2 tensor per vertex (type 3)."""
    toks = open(path).read().split()
    try:
        k = toks.index("SolAtVertices")
    except ValueError:
        raise ValueError(f"{path}: no SolAtVertices section") from None
    n = int(toks[k + 1])
    nfields, ftype = int(toks[k + 2]), int(toks[k + 3])
    if nfields != 1 or ftype != 3:
        raise ValueError(f"{path}: expected one symmetric tensor per vertex, got {nfields} field(s) of type {ftype}")
    vals = np.array(toks[k + 4:k + 4 + 3 * n], dtype=np.float64)
    if vals.shape[0] != 3 * n:
        raise ValueError(f"{path}: truncated, {vals.shape[0] // 3} of {n} tensors")
    return vals.reshape(n, 3)


def metric_lengths(points: np.ndarray, tris: np.ndarray, tensor: np.ndarray) -> np.ndarray:
    """Metric length of every undirected edge (numeric.cpp:469-497)."""
    e = np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]])
    e = np.unique(np.sort(e, axis=1), axis=0)
    w = points[e[:, 1]] - points[e[:, 0]]

    def under(t):
        return np.sqrt(w[:, 0] * (t[:, 0] * w[:, 0] + t[:, 1] * w[:, 1])
                       + w[:, 1] * (t[:, 1] * w[:, 0] + t[:, 2] * w[:, 1]))
    l0, l1 = under(tensor[e[:, 0]]), under(tensor[e[:, 1]])
    lo, hi = np.minimum(l0, l1), np.maximum(l0, l1)
    r = hi / lo
    with np.errstate(divide="ignore", invalid="ignore"):
        geo = hi * (r - 1) / (r * np.log(r))
    return np.where(np.abs(l0 - l1) < 1e-9, l0, geo)


def histogram(points, tris, tensor, edges=EDGES) -> dict:
    ln = metric_lengths(points, tris, tensor)
    h, _ = np.histogram(ln, np.asarray(edges))
    frac = h / max(h.sum(), 1)
    inr = float(np.mean((ln >= 2 ** -0.5) & (ln <= 2 ** 0.5))) if ln.size else 0.0
    return {"edges": [float(x) for x in edges], "fractions": [float(x) for x in frac], "counts": h.tolist(),
            "in_range_fraction": inr, "edges_total": int(ln.size), "triangles": int(tris.shape[0]),
            "vertices": int(points.shape[0])}


def of_files(mesh_path: str, sol_path: str) -> dict:
    m = meshgen.read_mesh(mesh_path)
    ten = read_sol(sol_path)
    if ten.shape[0] != m.nb_nodes:
        raise ValueError(f"{sol_path}: {ten.shape[0]} tensors for {m.nb_nodes} vertices")
    return histogram(np.asarray(m.points), np.asarray(m.tris), ten)


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("mesh")
    p.add_argument("sol")
    p.add_argument("--against", nargs=2, metavar=("MESH", "SOL"))
    a = p.parse_args(argv)
    out = of_files(a.mesh, a.sol)
    if a.against:
        other = of_files(*a.against)
        diff = [x - y for x, y in zip(out["fractions"], other["fractions"])]
        out["against"] = other
        out["difference"] = diff
        out["max_abs_difference"] = max(abs(d) for d in diff)
    json.dump(out, sys.stdout)
    sys.stdout.write("\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
