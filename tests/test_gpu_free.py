"""Free mode (GPU heuristics: Jones-Plassmann MIS and coloring, handshake
matching): every stage keeps the mesh conforming and positively oriented, and
the final mesh matches the reference's size and metric-length quality."""
import numpy as np
import pytest

from tests.helpers import check_invariants, gpu_mesh, gpu_state, in_range_fraction, oracle_run, run_gpu_stages


@pytest.mark.gpu
@pytest.mark.parametrize("name,n,rounds", [("c1", None, 3), ("c2", 120, 3)])
def test_free_mode_invariants_and_quality(oracle_built, name, n, rounds):
    m, u, c, states, _ = oracle_run(name, n, rounds)
    g = gpu_mesh(m, u, c)

    def check(stage):
        check_invariants(gpu_state(g))

    run_gpu_stages(g, c, check)
    st = gpu_state(g)
    ref = states[f"r{c['rounds'] - 1}.smooth"]
    n_gpu, n_ref = st.active_elems().shape[0], ref.active_elems().shape[0]
    assert abs(n_gpu - n_ref) <= 0.03 * n_ref, (n_gpu, n_ref)
    f_gpu, f_ref = in_range_fraction(st), in_range_fraction(ref)
    assert f_gpu >= f_ref - 0.02, (f_gpu, f_ref)


@pytest.mark.gpu
def test_free_mode_deterministic(oracle_built):
    m, u, c, _, _ = oracle_run("c1", 40, 2)
    outs = []
    for _ in range(2):
        g = gpu_mesh(m, u, c)
        run_gpu_stages(g, c, lambda s: None)
        outs.append(gpu_state(g))
    assert not outs[0].diff(outs[1])
