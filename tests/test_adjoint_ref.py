"""The FP64 torch reference of the quality functional, checked on the CPU:
its forward against the oracle (metric tensors and element qualities of the
reference's arithmetic), its autograd gradient against central finite
differences of itself."""
import numpy as np
import pytest
import torch

from tests import adjoint_ref as ar
from tests.oracle_lib import Oracle, _p, lib
from trinity_b200 import meshgen

PARAMS = dict(target_factor=0.7, p=2, h_min=1e-9, h_max=0.4)


def _case(n=12, jitter=0.3, seed=4):
    m = meshgen.grid_mesh(n, jitter=jitter, seed=seed)
    return m, meshgen.field_multi(m.points)


def test_metric_and_qualities_match_the_oracle(oracle_built):
    m, u = _case()
    o = Oracle(m, u, capa_scale=2, bucket=64)
    o.metric(0.7, 2)
    st = o.state()
    topo = ar.Topology(m.points, m.tris)
    ten = ar.metric(topo, torch.tensor(u), **PARAMS).numpy()
    np.testing.assert_allclose(ten, st.tensor, rtol=1e-9, atol=1e-9 * np.abs(st.tensor).max())
    L = lib()
    q_or = np.array([L.orc_quality(*[_p(np.ascontiguousarray(x)) for x in (
        st.points[a], st.points[b], st.points[c], st.tensor[a], st.tensor[b], st.tensor[c])])
        for a, b, c in m.tris])
    q = ar.qualities(torch.tensor(m.points), topo.tris, torch.tensor(st.tensor)).numpy()
    np.testing.assert_allclose(q, q_or, rtol=1e-12, atol=1e-14)
    J = float(ar.functional(topo, torch.tensor(m.points), torch.tensor(u), **PARAMS))
    assert J == pytest.approx(q_or.sum(), rel=1e-9)


def _fd(fun, x0, idx, h):
    out = []
    for i in idx:
        xp, xm = x0.copy(), x0.copy()
        xp.flat[i] += h
        xm.flat[i] -= h
        out.append((fun(xp) - fun(xm)) / (2 * h))
    return np.array(out)


def test_autograd_matches_finite_differences():
    m, u = _case(n=10)
    topo = ar.Topology(m.points, m.tris)
    J, gxy, gu = ar.gradients(topo, m.points, u, **PARAMS)
    rng = np.random.default_rng(0)
    interior = np.flatnonzero((m.points > 0).all(1) & (m.points < 1).all(1))
    verts = rng.choice(interior, 15, replace=False)
    h = 1e-6
    with torch.no_grad():
        fx = lambda x: float(ar.functional(topo, torch.tensor(x.reshape(-1, 2)), torch.tensor(u), **PARAMS))
        fu = lambda v: float(ar.functional(topo, torch.tensor(m.points), torch.tensor(v), **PARAMS))
        idx_xy = np.concatenate([2 * verts, 2 * verts + 1])
        fd_xy = _fd(fx, m.points.copy(), idx_xy, h)
        fd_u = _fd(fu, u.copy(), verts, h)
    ad_xy = gxy.ravel()[idx_xy]
    ad_u = gu[verts]
    np.testing.assert_allclose(ad_xy, fd_xy, rtol=1e-5, atol=1e-6 * np.abs(gxy).max())
    np.testing.assert_allclose(ad_u, fd_u, rtol=1e-5, atol=1e-6 * np.abs(gu).max())
    assert np.abs(gu).max() > 0 and np.abs(gxy).max() > 0


def test_fixed_metric_gradient_is_the_coordinate_part():
    """With the metric held at the recovered tensors, dJ/dxy is the same as
    with u given: the recovery runs on the mesh's own coordinates."""
    m, u = _case(n=8)
    topo = ar.Topology(m.points, m.tris)
    with torch.no_grad():
        ten = ar.metric(topo, torch.tensor(u), **PARAMS).numpy()
    J1, g1, _ = ar.gradients(topo, m.points, ten=ten)
    J2, g2, _ = ar.gradients(topo, m.points, u, **PARAMS)
    assert J1 == pytest.approx(J2, rel=1e-14)
    np.testing.assert_allclose(g1, g2, rtol=1e-12, atol=1e-12 * np.abs(g1).max())
