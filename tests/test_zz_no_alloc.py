"""The allocation-free metric recovery (trn_metric_noalloc) gives the same
tensors as trn_metric_run, and the oracle's to 1e-12.

That entry point exists for callers that keep every byte of device memory
under their own control (a fixed budget, or their own pool allocator) and so
cannot let the library call cudaMalloc: they pass device buffers in and out,
and the library works in one fixed __device__ array. Two calls in a row with
different meshes check that the shared array is cleared between calls; a third
checks that oversized input is refused. This file is named to run last.
"""
import ctypes

import numpy as np
import pytest

TRN_ERR_CAPACITY = 1
TRN_ERR_INVALID = 3
MAX_NODES = 16384
BUCKET = 32


def _fn():
    from trinity_b200 import _lib
    f = _lib.lib().trn_metric_noalloc
    i, d, vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    f.argtypes = [i, i, vp, vp, vp, d, i, d, d, vp, vp]
    f.restype = i
    return f


def _reference_tensor(m, u, c):
    from tests.oracle_lib import tags_of
    from trinity_b200.api import Mesh, Metrics
    g = Mesh((m.nb_nodes, m.nb_elems), c["bucket"], c["depth"], 0, c["rounds"])
    g.load_arrays(m.points, m.tris, tags_of(m), u)
    Metrics(g, c["target"], c["norm"]).run()
    ten = g.export()[1]
    g.close()
    return ten


@pytest.mark.gpu
def test_metric_noalloc_matches_metric_run_twice():
    import torch
    from trinity_b200 import meshgen
    f = _fn()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev).cuda_stream
    for n in (40, 30):  # a larger mesh first, then a smaller one over its leftovers
        m, u, c = meshgen.make_config("c1", n)
        want = _reference_tensor(m, u, c)
        pts = torch.from_numpy(np.ascontiguousarray(m.points)).to(dev)
        tris = torch.from_numpy(np.ascontiguousarray(m.tris, dtype=np.int32)).to(dev)
        sol = torch.from_numpy(np.ascontiguousarray(u)).to(dev)
        out = torch.full((m.nb_nodes, 3), float("nan"), dtype=torch.float64, device=dev)
        rc = f(m.nb_nodes, m.nb_elems, pts.data_ptr(), tris.data_ptr(), sol.data_ptr(),
               c["target"], c["norm"], 1e-9, 0.4, out.data_ptr(), stream)
        torch.cuda.synchronize()
        assert rc == 0
        got = out.cpu().numpy()
        # same kernels, same reduction shape: equal to 1e-12 relative (bit-equal in practice)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=0.0)


@pytest.mark.gpu
def test_metric_noalloc_rejects_oversize():
    import torch
    f = _fn()
    dev = torch.device("cuda:0")
    buf = torch.zeros(8, dtype=torch.float64, device=dev)
    rc = f(MAX_NODES + 1, 8, buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 0.9, 2, 1e-9, 0.4,
           buf.data_ptr(), None)
    assert rc == TRN_ERR_CAPACITY


def _call(f, pts, tris, u, out, target=0.9, norm=2):
    import torch
    dev = torch.device("cuda:0")
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (pts, tris.astype(np.int32), u)]
    o = torch.full((pts.shape[0], 3), float("nan"), dtype=torch.float64, device=dev)
    rc = f(pts.shape[0], tris.shape[0], t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), target, norm,
           1e-9, 0.4, o.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize()
    out.append(o.cpu().numpy())
    return rc


@pytest.mark.gpu
def test_metric_noalloc_matches_the_oracle(oracle_built):
    """Against the oracle's tensors directly (the oracle sums the complexity
    in element order, the entry point with a tree: last bits only)."""
    from tests.helpers import oracle_run
    f = _fn()
    m, u, c, states, _ = oracle_run("c1", 40, 1)
    out = []
    assert _call(f, m.points, m.tris, u, out, c["target"], c["norm"]) == 0
    np.testing.assert_allclose(out[0], states["metric"].tensor, rtol=1e-12, atol=0.0)


@pytest.mark.gpu
def test_metric_noalloc_device_refusals_then_recovers():
    """A vertex with more triangles than the bucket (a fan of BUCKET + 1
    triangles) is TRN_ERR_CAPACITY, a triangle naming a vertex past the last
    is TRN_ERR_INVALID; both are caught on the device without writing outside
    the array, and the next call on the shared array is right again."""
    from trinity_b200 import meshgen
    f = _fn()
    k = BUCKET + 1
    ang = 2 * np.pi * np.arange(k) / k
    pts = np.concatenate([[[0.5, 0.5]], np.stack([0.5 + 0.4 * np.cos(ang), 0.5 + 0.4 * np.sin(ang)], 1)])
    fan = np.array([[0, 1 + i, 1 + (i + 1) % k] for i in range(k)], np.int32)
    out = []
    assert _call(f, pts, fan, np.sin(pts[:, 0]), out) == TRN_ERR_CAPACITY
    m, u, c = meshgen.make_config("c1", 12)
    bad = m.tris.copy()
    bad[7, 2] = m.nb_nodes
    assert _call(f, m.points, bad, u, out) == TRN_ERR_INVALID
    assert _call(f, m.points, m.tris, u, out, c["target"], c["norm"]) == 0
    np.testing.assert_allclose(out[-1], _reference_tensor(m, u, c), rtol=1e-12, atol=0.0)
