"""Failures injected from the host, reported as statuses (none traps the GPU):
element-node ids outside [1, numNodes] gather zeros instead of reading out of
bounds, PCG at maxIT reports NOT_CONVERGED (the reference's warning,
TOP_GPU.m:656-659), a non-finite right-hand side reports TOP_ERR_NAN, and a
withheld packed-tile copy makes the coarse product's bounded wait give up and
report TOP_ERR_CUDA."""
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


@pytest.mark.parametrize("mixed", [False, True])
def test_coarse_tile_copy_wait_gives_up_and_reports(mixed):
    """A packed-tile copy withheld by the test hook: the two-pass coarse
    product's bounded wait for it runs out (one second), the kernel raises its
    error flag and skips the rest of its tiles, and the V-cycle call reports
    TOP_ERR_CUDA; the next calls on the same solver give the V-cycle and PCG
    of a solver that never failed, bit for bit."""
    from top_gpu_on_matlab_b200._lib import TOP_ERR_CUDA, TopGpuError
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    m = Mesh(np.ones((24, 48, 24), bool), control=50)
    m.apply_optcase(1)
    ne = m.info()[0]["numElements"]
    x = torch.from_numpy(0.2 + 0.7 * np.random.default_rng(4).random(ne)).cuda()
    r = torch.from_numpy(np.random.default_rng(5).standard_normal(3 * m.info()[0]["numNodes"])).cuda()
    solvers = []
    for _ in range(2):
        s = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-8, maxIT=400, omega=0.6, mixed=mixed)
        s.set_density(x)
        s.assemble()
        s.set_tail_operator(False)               # the coarse products run in the V-cycle
        solvers.append(s)
    ref = solvers[0].vcycle(r)
    s = solvers[1]
    s.test_withhold_tile()
    with pytest.raises(TopGpuError) as e:
        s.vcycle(r)
    assert e.value.status == TOP_ERR_CUDA and "tile copy did not complete" in str(e.value)
    assert torch.equal(s.vcycle(r), ref)
    U0, its0, _ = solvers[0].pcg(0)
    U1, its1, _ = s.pcg(0)
    assert its0 == its1 and torch.equal(U0, U1)
