"""Failures injected from the host, reported as statuses (none traps the GPU):
element-node ids outside [1, numNodes] gather zeros instead of reading out of
bounds, PCG at maxIT reports NOT_CONVERGED (the reference's warning,
TOP_GPU.m:656-659), a non-finite right-hand side reports TOP_ERR_NAN."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("u32", [False, True])
def test_gather_out_of_range_ids_read_zero(u32):
    from top_gpu_on_matlab_b200 import mex
    L = O.Model(np.ones((4, 8, 4), bool)).level(0)
    u = np.random.default_rng(0).standard_normal((L.numNodes, 3))
    eN = L.eNodMat.astype(np.int64)
    bad = [0, L.numNodes + 5, (2 ** 32 - 1) if u32 else -3]
    eN[0, 0], eN[1, 3], eN[2, 7] = bad
    eN = eN.astype(np.uint32 if u32 else np.int32)
    g = mex.zeros((L.numElements, 24))
    mex.Gathering_inplace(g, mex.gpu_array(u), mex.gpu_array(eN))
    out = mex.gather(g)
    for e, n in ((0, 0), (1, 3), (2, 7)):
        assert not out[e, 3 * n:3 * n + 3].any()
    ok = eN.astype(np.int64).copy()
    ok[0, 0], ok[1, 3], ok[2, 7] = 1, 1, 1
    ref = O.gather(u, ok)
    ref[0, 0:3] = ref[1, 9:12] = ref[2, 21:24] = 0.0
    assert np.array_equal(out, ref)


def _solver(maxIT, tol):
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    m = Mesh(np.ones((8, 16, 8), bool))
    m.apply_optcase(1)
    s = Solver(m, E0=1.0, Emin=1e-9, tol=tol, maxIT=maxIT, omega=0.6)
    s.set_density(torch.full((m.info()[0]["numElements"],), 0.5, dtype=torch.float64, device="cuda"))
    s.assemble()
    return s


def test_pcg_at_maxit_reports_not_converged(capsys):
    from top_gpu_on_matlab_b200._lib import TOP_ERR_NOT_CONVERGED, TopGpuError
    s = _solver(maxIT=1, tol=1e-12)
    with pytest.raises(TopGpuError) as e:
        s.pcg(0, raise_on_maxit=True)
    assert e.value.status == TOP_ERR_NOT_CONVERGED
    U, its, res = s.pcg(0)
    assert its == 1 and res > 1e-12 and torch.isfinite(U).all()
    assert "Exceed the maximum iterate numbers" in capsys.readouterr().out


def test_pcg_non_finite_rhs_reports_nan():
    from top_gpu_on_matlab_b200._lib import TOP_ERR_NAN, TopGpuError
    s = _solver(maxIT=50, tol=1e-8)
    b = torch.zeros(s.numDOFs, dtype=torch.float64, device="cuda")
    b[5] = float("nan")
    with pytest.raises(TopGpuError) as e:
        s.pcg(b=b)
    assert e.value.status == TOP_ERR_NAN and "non-finite" in str(e.value)
