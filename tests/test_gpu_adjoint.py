"""The element-quality functional and its hand-written adjoint on the GPU
(trn_quality_adjoint), checked against the oracle's qualities, the FP64 torch
reference gradient, and central finite differences of the GPU's own FP64
functional; then wrapped as a torch.autograd.Function (test only), and the
gradient-based smoothing pass that uses it."""
import numpy as np
import pytest

from tests import adjoint_ref as ar
from tests.oracle_lib import Oracle, _p, lib, tags_of
from trinity_b200 import meshgen

pytestmark = pytest.mark.gpu

T, P, HMIN, HMAX = 0.7, 2, 1e-9, 0.4
MARGS = dict(target_factor=T, Lp_norm=P, h_min=HMIN, h_max=HMAX)
RARGS = dict(target_factor=T, p=P, h_min=HMIN, h_max=HMAX)


def _mesh(n, jitter=0.3, seed=4, bucket=64):
    from trinity_b200.api import Mesh
    m = meshgen.grid_mesh(n, jitter=jitter, seed=seed)
    u = meshgen.field_multi(m.points)
    g = Mesh((m.nb_nodes, m.nb_elems), bucket, 1, 0, 1, capa_scale=2)
    g.load_arrays(m.points, m.tris, tags_of(m), u)
    return m, u, g


def _cuda(a):
    import torch
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def test_value_matches_the_oracle_qualities(oracle_built):
    from trinity_b200.api import Metrics
    m, u, g = _mesh(24)
    J, _, _ = g.quality_adjoint(None, _cuda(u), grad_xy=False, **MARGS)
    o = Oracle(m, u, capa_scale=2, bucket=64)
    o.metric(T, P)
    st = o.state()
    L = lib()
    q = [L.orc_quality(*[_p(np.ascontiguousarray(x)) for x in (
        st.points[a], st.points[b], st.points[c], st.tensor[a], st.tensor[b], st.tensor[c])])
        for a, b, c in m.tris]
    assert J == pytest.approx(float(np.sum(q)), rel=1e-12)
    # the same metric through trn_metric_run, then the mesh's tensors: same bits
    Metrics(g, T, P).run()
    J2, _, _ = g.quality_adjoint(None, None, grad_xy=False)
    assert J2 == J


@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-8), ("mixed", 2e-3)])
def test_gradients_match_the_fp64_reference(precision, rtol):
    m, u, g = _mesh(16)
    J, gxy, gu = g.quality_adjoint(None, _cuda(u), precision=precision, **MARGS)
    topo = ar.Topology(m.points, m.tris)
    Jr, rxy, ru = ar.gradients(topo, m.points, u, **RARGS)
    gxy, gu = gxy.cpu().numpy(), gu.cpu().numpy()
    assert J == pytest.approx(Jr, rel=1e-10 if precision == "fp64" else 1e-5)
    for got, want in ((gxy, rxy), (gu, ru)):
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err < rtol, (precision, err)
    if precision == "fp64":
        np.testing.assert_allclose(gxy, rxy, rtol=1e-7, atol=1e-9 * np.abs(rxy).max())
        np.testing.assert_allclose(gu, ru, rtol=1e-7, atol=1e-9 * np.abs(ru).max())


def test_deterministic():
    m, u, g = _mesh(20)
    a = g.quality_adjoint(None, _cuda(u), **MARGS)
    b = g.quality_adjoint(None, _cuda(u), **MARGS)
    assert a[0] == b[0]
    assert bool((a[1] == b[1]).all()) and bool((a[2] == b[2]).all())


def _probe(g, xy, uu, v, c, h):
    """J at +h and -h on one coordinate (c = 0, 1) or on the solution (c = 2)
    of vertex v; returns (J+, J-, the exact difference of the two arguments)"""
    t = uu if c == 2 else xy
    idx = (v,) if c == 2 else (v, c)
    x0 = float(t[idx])
    out = []
    for s in (1, -1):
        t[idx] = x0 + s * h
        if c == 2:
            out.append(g.quality_adjoint(None, uu, grad_xy=False, grad_solut=False, **MARGS)[0])
        else:
            out.append(g.quality_adjoint(xy, None, grad_xy=False)[0])
    t[idx] = x0
    return out[0], out[1], (x0 + h) - (x0 - h)


def _central(g, u, verts, h, coords):
    import torch
    xy = torch.tensor(g.export()[0], dtype=torch.float64, device="cuda").contiguous()
    uu = _cuda(u)
    fd = np.zeros((len(verts), len(coords)))
    for k, v in enumerate(verts):
        for j, c in enumerate(coords):
            jp, jm, den = _probe(g, xy, uu, int(v), c, h)
            fd[k, j] = (jp - jm) / den
    return fd


def _rel(got, want):
    return np.abs(got - want) / np.maximum(np.abs(want), 1e-12 * np.abs(want).max())


@pytest.mark.parametrize("n,count", [(40, 200), (1000, 1000)])
def test_finite_differences(n, count):
    """Central differences of the GPU's FP64 functional, step 1e-6, at random
    interior vertices; n = 1000 is the 2M-triangle mesh with vertices jittered
    by +-0.3h and the multi-feature field, 1,000 vertices.

    The coordinate gradient is smooth at that step. The solution's is not
    everywhere: the recovery amplifies a change of u by about 16/h_e^2, so at
    h_e = 1e-3 a 1e-6 step moves the Hessian by about 16 and some probes cross
    a kink of the forward (|lambda| at 0, the eigen shortcut, the clamps).
    There the check is statistical (median and 90th percentile), and a
    100x smaller step must shrink the overall error."""
    from trinity_b200.api import Metrics
    m, u, g = _mesh(n, bucket=64)
    Metrics(g, T, P).run()          # the mesh's tensors = M(u): the xy probes reuse them
    res = {}
    for prec in ("fp64", "mixed"):
        J, gxy, gu = g.quality_adjoint(None, _cuda(u), precision=prec, **MARGS)
        res[prec] = (gxy.cpu().numpy(), gu.cpu().numpy())
    rng = np.random.default_rng(7)
    interior = np.flatnonzero((m.points > 0).all(1) & (m.points < 1).all(1))
    verts = rng.choice(interior, count, replace=False)
    fd = _central(g, u, verts, 1e-6, (0, 1, 2))
    fd_xy, fd_u = fd[:, :2], fd[:, 2]
    for prec, tol in (("fp64", 1e-4), ("mixed", 1e-3)):
        gxy, gu = res[prec]
        r = _rel(gxy[verts], fd_xy)
        assert np.mean(r > tol) <= 0.01, (prec, np.percentile(r, [50, 99]))
        r = _rel(gu[verts], fd_u)
        assert np.median(r) < tol and np.percentile(r, 90) < 10 * tol, (prec, np.percentile(r, [50, 90]))
    gu = res["fp64"][1][verts]
    e6 = np.linalg.norm(fd_u - gu) / np.linalg.norm(gu)
    fd8 = _central(g, u, verts, 1e-8, (2,))[:, 0]
    e8 = np.linalg.norm(fd8 - gu) / np.linalg.norm(gu)
    assert e8 < 2e-2 and e8 < e6 + 1e-3, (e6, e8)
    # FP32 against FP64 over every vertex (near the eigen shortcut's threshold
    # the two forms can take different branches)
    for a, b, tol in zip(res["mixed"], res["fp64"], (1e-3, 5e-3)):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < tol


def test_autograd_function():
    """test-only torch.autograd.Function over the C ABI adjoint"""
    import torch

    class QualityFunctional(torch.autograd.Function):
        @staticmethod
        def forward(ctx, xy, solut, mesh):
            J, gxy, gu = mesh.quality_adjoint(xy.detach().contiguous(), solut.detach().contiguous(),
                                              **MARGS)
            ctx.save_for_backward(gxy, gu)
            return torch.tensor(J, dtype=torch.float64, device=xy.device)

        @staticmethod
        def backward(ctx, gJ):
            gxy, gu = ctx.saved_tensors
            return gJ * gxy, gJ * gu, None

    m, u, g = _mesh(12)
    xy = _cuda(m.points).requires_grad_()
    uu = _cuda(u).requires_grad_()
    J = QualityFunctional.apply(xy, uu, g)
    (2.0 * J).backward()
    topo = ar.Topology(m.points, m.tris)
    Jr, rxy, ru = ar.gradients(topo, m.points, u, **RARGS)
    assert float(J.detach()) == pytest.approx(Jr, rel=1e-10)
    np.testing.assert_allclose(xy.grad.cpu().numpy(), 2 * rxy, rtol=1e-7, atol=1e-9 * np.abs(rxy).max())
    np.testing.assert_allclose(uu.grad.cpu().numpy(), 2 * ru, rtol=1e-7, atol=1e-9 * np.abs(ru).max())


def test_gradient_smoothing_improves_quality():
    from tests.helpers import check_invariants, gpu_state
    from trinity_b200.api import GradientSmooth, Metrics, Partit, Smooth
    out = {}
    for kind in ("gradient", "laplacian"):
        m, u, g = _mesh(60)
        Metrics(g, T, P).run()
        q0 = g.quality_stats()
        if kind == "gradient":
            GradientSmooth(g, Partit(g, 8), 20).run()
        else:
            Smooth(g, Partit(g, 8), 20).run()
        q1 = g.quality_stats()
        st = gpu_state(g)
        check_invariants(st)
        out[kind] = (q0, q1)
    (q0, q1) = out["gradient"]
    assert q1[0] >= q0[0] and q1[2] > q0[2]
