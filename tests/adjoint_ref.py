"""FP64 reference of the element-quality functional, in torch ops on the CPU,
differentiated by autograd: the independent check of the hand-written adjoint
(trn_quality_adjoint).

    J(xy, u) = sum_T q_T(xy, M(u))

q_T is numeric::computeQuality (numeric.cpp:251-306); M(u) is Metrics::run
(metric.cpp:59-238 with hessian.cpp:24-153) on the mesh's own coordinates.
Every step follows the reference's arithmetic, branch for branch: the closed
form 2x2 eigen decomposition with its diagonal shortcut (numeric.cpp:25-95),
the log-Euclidean mean (numeric.cpp:98-248), the |lambda| clamp with the local
L^p scale, the complexity, the global scale and its eigenvalue clamp.

Test infrastructure only.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import torch

EPS = 1e-9


def eig2(m0, m1, m2, m3):
    """numeric::eigenDecompose of [[m0, m1], [m2, m3]]: (l0, l1, (v0, v1, v2, v3)),
    eigenvectors in the columns (v0, v2) and (v1, v3)."""
    diag = (m1 * m2 < EPS).detach()
    one = torch.ones_like(m0)
    g1 = torch.where(diag, one, m1)   # the general branch on safe values
    g2 = torch.where(diag, one, m2)
    term = (m0 + m3) * 0.5
    det = m0 * m3 - g1 * g2
    sd = torch.sqrt(term * term - det)
    l0, l1 = term - sd, term + sd
    dm = m0 - m3
    root = torch.sqrt(torch.clamp(0.25 * dm * dm + g1 * g2, min=0.0))
    pos = (dm >= 0).detach()
    v0 = torch.where(pos, 0.5 * dm - root, g2)
    v1 = torch.where(pos, g1, 0.5 * dm + root)
    v2 = torch.where(pos, g2, -0.5 * dm - root)
    v3 = torch.where(pos, -0.5 * dm + root, g1)
    n0 = torch.sqrt(v0 * v0 + v1 * v1)
    n1 = torch.sqrt(v2 * v2 + v3 * v3)
    v0, v1, v2, v3 = v0 / n0, v1 / n0, v2 / n1, v3 / n1
    z = torch.zeros_like(m0)
    l0 = torch.where(diag, m3, l0)
    l1 = torch.where(diag, m0, l1)
    v0 = torch.where(diag, z, v0)
    v1 = torch.where(diag, one, v1)
    v2 = torch.where(diag, one, v2)
    v3 = torch.where(diag, z, v3)
    return l0, l1, (v0, v1, v2, v3)


def recompose(f0, f1, v):
    """P diag(f) P^T in the reference's operand order: (h0, h1, h2, h3)."""
    v0, v1, v2, v3 = v
    c0, c1, c2, c3 = f0 * v0, f0 * v2, f1 * v1, f1 * v3
    return (v0 * c0 + v1 * c2, v0 * c1 + v1 * c3, v2 * c0 + v3 * c2, v2 * c1 + v3 * c3)


class Topology:
    """Per-element P1 basis gradients and areas at the recovery geometry, and
    the (vertex, element) pairs of the 2-ring patches (mesh.cpp:390-434)."""

    def __init__(self, pts0: np.ndarray, tris: np.ndarray):
        V, T = len(pts0), len(tris)
        self.V, self.T = V, T
        self.tris = torch.as_tensor(tris, dtype=torch.int64)
        p = np.asarray(pts0, dtype=np.float64)
        a, b, c = p[tris[:, 0]], p[tris[:, 1]], p[tris[:, 2]]
        area = 0.5 * ((b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (c[:, 0] - a[:, 0]) * (b[:, 1] - a[:, 1]))
        norm = 2 / area
        d = np.stack([norm * (b[:, 1] - c[:, 1]), norm * (c[:, 0] - b[:, 0]),
                      norm * (c[:, 1] - a[:, 1]), norm * (a[:, 0] - c[:, 0]),
                      norm * (a[:, 1] - b[:, 1]), norm * (b[:, 0] - a[:, 0])], axis=1)
        self.area = torch.as_tensor(area)
        self.psi = torch.as_tensor(d.reshape(T, 3, 2))
        rows = np.repeat(np.arange(T), 3)
        inc = sp.csr_matrix((np.ones(3 * T), (tris.ravel(), rows)), shape=(V, T))
        edges = np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]])
        adj = sp.csr_matrix((np.ones(len(edges)), (edges[:, 0], edges[:, 1])), shape=(V, V))
        ring = ((adj + adj.T + sp.identity(V)) > 0).astype(np.float64)
        patch = (ring @ inc).tocoo()
        order = np.lexsort((patch.col, patch.row))
        self.pv = torch.as_tensor(patch.row[order], dtype=torch.int64)
        self.pt = torch.as_tensor(patch.col[order], dtype=torch.int64)
        self.atot = torch.zeros(V, dtype=torch.float64).index_add(0, self.pv, self.area[self.pt])
        self.star = torch.zeros(V, dtype=torch.float64).index_add(
            0, self.tris.reshape(-1), self.area.repeat_interleave(3))

    def patch_mean(self, per_elem):
        """area-weighted mean over each vertex's patch of a per-element field"""
        w = self.area[self.pt].reshape(-1, *([1] * (per_elem.dim() - 1)))
        out = torch.zeros((self.V,) + tuple(per_elem.shape[1:]), dtype=per_elem.dtype)
        out = out.index_add(0, self.pv, w * per_elem[self.pt])
        return out / self.atot.reshape(-1, *([1] * (per_elem.dim() - 1)))


def metric(topo: Topology, u, target_factor=1.0, p=2, h_min=1e-9, h_max=0.4):
    """Metrics::run: the stored tensors (m11, m12, m22) of every vertex."""
    tri = topo.tris
    g_t = (u[tri].unsqueeze(-1) * topo.psi).sum(1)                      # (T, 2)
    grad = topo.patch_mean(g_t)                                          # (V, 2)
    h_t = (grad[tri].unsqueeze(-1) * topo.psi.unsqueeze(2)).sum(1)       # (T, 2, 2): [a][b] = g_a psi_b
    H = topo.patch_mean(h_t)
    t0, t1, t2 = H[:, 0, 0], 0.5 * (H[:, 0, 1] + H[:, 1, 0]), H[:, 1, 1]
    l0, l1, v = eig2(t0, t1, t1, t2)
    lp0 = torch.clamp(l0.abs(), min=EPS)
    lp1 = torch.clamp(l1.abs(), min=EPS)
    e = -1.0 / (2 * p + 2) if p else 0.5
    s = (lp0 * lp1) ** e
    h = recompose(lp0 * s, lp1 * s, v)
    m0, m1, m2 = h[0], h[1], h[3]
    det = m0 * m2 - m1 * m1
    rho = torch.sqrt(det)[tri].sum(1) / 3
    complexity = (rho * topo.area).sum()
    fact = float(int(np.floor(topo.V * target_factor))) / complexity
    l0, l1, v = eig2(m0, m1, m1, m2)
    lo, hi = 1 / h_max ** 2, 1 / h_min ** 2
    f0 = torch.clamp(l0 * fact, min=lo, max=hi)
    f1 = torch.clamp(l1 * fact, min=lo, max=hi)
    h = recompose(f0, f1, v)
    return torch.stack([h[0], h[1], h[3]], 1)


def qualities(xy, tri, ten):
    """numeric::computeQuality of every element (tensor logarithms per vertex,
    their mean per element, exponentiated)."""
    l0, l1, v = eig2(ten[:, 0], ten[:, 1], ten[:, 1], ten[:, 2])
    L = torch.stack(recompose(torch.log(l0), torch.log(l1), v), 1)      # (V, 4)
    lm = (L[tri[:, 0]] + L[tri[:, 1]] + L[tri[:, 2]]) / 3
    k0, k1, w = eig2(lm[:, 0], lm[:, 1], lm[:, 2], lm[:, 3])
    j = recompose(torch.exp(k0), torch.exp(k1), w)
    j0, j1, j2 = j[0], j[1], j[3]
    det = j0 * j2 - j1 * j1
    pa, pb, pc = xy[tri[:, 0]], xy[tri[:, 1]], xy[tri[:, 2]]
    perim = 0
    for e in (pb - pa, pc - pb, pa - pc):
        uu, vv = e[:, 0], e[:, 1]
        perim = perim + torch.sqrt(uu * (j0 * uu + j1 * vv) + vv * (j1 * uu + j2 * vv))
    cross = (pb[:, 0] - pa[:, 0]) * (pc[:, 1] - pa[:, 1]) - (pc[:, 0] - pa[:, 0]) * (pb[:, 1] - pa[:, 1])
    area = 0.5 * cross.abs()
    mean = torch.minimum(perim / 3, 3 / perim)
    norm = 12 * np.sqrt(3.0) * (mean * (2 - mean)) ** 3
    return area * norm * torch.sqrt(det) / perim ** 2


def functional(topo: Topology, xy, u=None, ten=None, **metric_args):
    """J(xy, u) (metric recovered from u) or J(xy) under fixed tensors ten."""
    if u is not None:
        ten = metric(topo, u, **metric_args)
    return qualities(xy, topo.tris, ten).sum()


def gradients(topo: Topology, xy0: np.ndarray, u0: np.ndarray | None = None, ten=None, **metric_args):
    """(J, dJ/dxy, dJ/du) in FP64 by autograd."""
    xy = torch.tensor(xy0, dtype=torch.float64, requires_grad=True)
    u = torch.tensor(u0, dtype=torch.float64, requires_grad=True) if u0 is not None else None
    t = torch.as_tensor(ten, dtype=torch.float64) if ten is not None else None
    J = functional(topo, xy, u, t, **metric_args)
    J.backward()
    return float(J.detach()), xy.grad.numpy().copy(), (u.grad.numpy().copy() if u is not None else None)
