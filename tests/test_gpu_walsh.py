"""Level-0 stiffness product in the Walsh basis of the voxel element: every
tile shape and z-chunk of the kernel against the oracle's K*u
(Solving_KbyU_MatrixFree, TOP_GPU.m:669-765) and against the node-centric
dense-Ke kernel, on full, irregular and roller-supported domains."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHAPES = [(16, 16), (16, 8)]


def _rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _model(mask, opt, seed):
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    o = O.Model(mask, control=20000)
    o.apply_optcase(opt)
    o.set_material(1.0, 1e-9, 3.0)
    o.set_solver(1e-6, 800, 0.6)
    m = Mesh(mask, control=20000)
    m.apply_optcase(opt)
    s = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-6, maxIT=800, omega=0.6)
    x = 0.05 + 0.95 * np.random.default_rng(seed).random(o.level(0).numElements)
    o.set_density(x)
    s.set_density(torch.from_numpy(x).cuda())
    return o, s


def _irregular(shape, seed):
    mk = np.random.default_rng(seed).random(shape) < 0.7
    mk[:, 0, :] = True
    mk[:, -1, :] = True
    return mk


CASES = {
    "cantilever_17x33x9": (np.ones((17, 33, 9), bool), 1),
    "irregular_20x30x14": (_irregular((20, 30, 14), 0), 1),
    "mbb_10x40x6": (np.ones((10, 40, 6), bool), 2),
}


@pytest.fixture(scope="module", params=list(CASES))
def model(request):
    mask, opt = CASES[request.param]
    return _model(mask, opt, 3)


def test_walsh_is_default(model):
    _, s = model
    assert s.l0_kernel(False)[0] == 1 and s.l0_kernel(True)[0] == 1


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("ctas", [0, 1, 7, 100000])
def test_walsh_matvec_matches_oracle(model, shape, ctas):
    """ctas = 1: one CTA walks every tile; 7: ranges straddle tiles;
    100000: clamped to one CTA per (tile, layer)."""
    o, s = model
    keep = s.l0_kernel(False), s.l0_kernel(True)
    u = np.random.default_rng(ctas).standard_normal(o.level(0).numDOFs)
    ref = o.matvec(0, u)
    ud = torch.from_numpy(u).cuda()
    for fp32 in (False, True):
        s.set_l0_kernel(fp32, 1, shape[0], shape[1], ctas)
        y = s.matvec(0, ud, fp32=fp32)
        assert _rel(y, ref) < (2e-6 if fp32 else 1e-13), (shape, ctas, fp32)
    for fp32, k in ((False, keep[0]), (True, keep[1])):
        s.set_l0_kernel(fp32, *k)


def test_walsh_and_dense_kernels_agree(model):
    o, s = model
    u = torch.from_numpy(np.random.default_rng(9).standard_normal(o.level(0).numDOFs)).cuda()
    keep = s.l0_kernel(False)
    yw = s.matvec(0, u)
    s.set_l0_kernel(False, 0)
    yd = s.matvec(0, u)
    s.set_l0_kernel(False, *keep)
    assert _rel(yw, yd.cpu().numpy()) < 1e-13


def test_walsh_rejects_bad_shape(model):
    from top_gpu_on_matlab_b200._lib import TopGpuError
    _, s = model
    with pytest.raises(TopGpuError):
        s.set_l0_kernel(False, 1, 12, 12, 4)
    with pytest.raises(TopGpuError):
        s.set_l0_kernel(False, 1, 16, 16, -1)
    assert s.l0_kernel(False)[0] == 1


def test_vcycle_and_pcg_with_walsh_match_oracle():
    o, s = _model(np.ones((12, 24, 12), bool), 1, 5)
    o.assemble()
    s.assemble()
    r = np.random.default_rng(6).standard_normal(o.level(0).numDOFs)
    assert _rel(s.vcycle(torch.from_numpy(r).cuda()), o.vcycle(r)) < 1e-11
