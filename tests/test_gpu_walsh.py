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
    assert s.l0_kernel(False)[0] == 3 and s.l0_kernel(True)[0] == 3


def test_autotune_picks_a_working_kernel(model):
    o, s = model
    keep = s.l0_kernel(False), s.l0_kernel(True)
    res = s.autotune(nrep=2, flush_bytes=0)
    assert res["fp64"][0] > 0 and res["fp32"][0] > 0
    assert s.l0_kernel(False) == res["fp64"][1] and s.l0_kernel(True) == res["fp32"][1]
    u = np.random.default_rng(5).standard_normal(o.level(0).numDOFs)
    ref = o.matvec(0, u)
    ud = torch.from_numpy(u).cuda()
    assert _rel(s.matvec(0, ud), ref) < 1e-13
    assert _rel(s.matvec(0, ud, fp32=True), ref) < 2e-6
    for fp32, k in ((False, keep[0]), (True, keep[1])):
        s.set_l0_kernel(fp32, *k)


@pytest.mark.parametrize("mixed", [False, True])
def test_autotune_on_the_pcg_products(mixed):
    """the autotuner times the products a PCG iteration makes (outer product
    with its dot, V-cycle residual and post-smoothing products); a solver
    tuned that way solves to the FP64 oracle's compliance"""
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    mask = np.ones((12, 24, 12), bool)
    o = O.Model(mask, control=20000)
    o.apply_optcase(1)
    o.set_material(1.0, 1e-9, 3.0)
    o.set_solver(1e-8, 800, 0.6)
    m = Mesh(mask, control=20000)
    m.apply_optcase(1)
    s = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-8, maxIT=800, omega=0.6, mixed=mixed)
    x = np.full(o.level(0).numElements, 0.3)
    o.set_density(x)
    o.assemble()
    s.set_density(torch.from_numpy(x).cuda())
    s.assemble()
    res = s.autotune(nrep=2, flush_bytes=0)
    assert res["fp64"][0] > 0 and res["fp32"][0] > 0
    assert s.l0_kernel(False) == res["fp64"][1] and s.l0_kernel(True) == res["fp32"][1]
    b = o.F()[:, 0]
    xo, _, _ = o.pcg(b)
    U, its, r = s.pcg(0)
    assert r < 1e-8
    c_o, c = b @ xo, float(torch.from_numpy(b).cuda() @ U)
    assert abs(c - c_o) <= 1e-7 * abs(c_o)


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
    for fp32, kind in ((False, 1), (True, 1), (True, 2), (False, 3), (True, 3), (True, 4), (True, 5), (True, 6)):
        if kind == 5 and shape != (16, 8):    # the tensor-core kind: 16 x 8 element columns only
            continue
        s.set_l0_kernel(fp32, kind, shape[0], shape[1], ctas)
        y = s.matvec(0, ud, fp32=fp32)
        assert _rel(y, ref) < (2e-6 if fp32 else 1e-13), (shape, ctas, fp32, kind)
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
    keep = s.l0_kernel(False)
    with pytest.raises(TopGpuError):
        s.set_l0_kernel(False, 1, 12, 12, 4)
    with pytest.raises(TopGpuError):
        s.set_l0_kernel(False, 1, 16, 16, -1)
    with pytest.raises(TopGpuError):          # paired-element kernels: FP32 only
        s.set_l0_kernel(False, 2, 16, 8, 0)
    with pytest.raises(TopGpuError):
        s.set_l0_kernel(False, 4, 16, 8, 0)
    with pytest.raises(TopGpuError):          # tensor-core kind: FP32, 16 x 8 only
        s.set_l0_kernel(False, 5, 16, 8, 0)
    with pytest.raises(TopGpuError):
        s.set_l0_kernel(True, 5, 16, 16, 0)
    with pytest.raises(TopGpuError):          # TMA-staged kind: FP32 only
        s.set_l0_kernel(False, 6, 16, 8, 0)
    assert s.l0_kernel(False) == keep        # a rejected configuration changes nothing


def test_vcycle_and_pcg_with_walsh_match_oracle():
    o, s = _model(np.ones((12, 24, 12), bool), 1, 5)
    o.assemble()
    s.assemble()
    r = np.random.default_rng(6).standard_normal(o.level(0).numDOFs)
    assert _rel(s.vcycle(torch.from_numpy(r).cuda()), o.vcycle(r)) < 1e-11


@pytest.mark.parametrize("kind", [1, 2, 3, 4, 5, 6])
def test_mixed_vcycle_kinds_agree(kind):
    """The FP32 V-cycle with either Walsh kernel stays within FP32 rounding
    of the FP64 V-cycle."""
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    mask = np.ones((12, 24, 12), bool)
    m = Mesh(mask, control=20000)
    m.apply_optcase(1)
    s64 = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-6, maxIT=800, omega=0.6)
    s32 = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-6, maxIT=800, omega=0.6, mixed=True)
    x = torch.from_numpy(0.3 + 0.6 * np.random.default_rng(1).random(m.info()[0]["numElements"])).cuda()
    for s in (s64, s32):
        s.set_density(x)
        s.assemble()
    s32.set_l0_kernel(True, kind, 16, 8, 0)
    r = torch.from_numpy(np.random.default_rng(2).standard_normal(s64.numDOFs)).cuda()
    z64, z32 = s64.vcycle(r), s32.vcycle(r)
    assert float((z32 - z64).abs().max() / z64.abs().max()) < 1e-5
