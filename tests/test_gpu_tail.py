"""The V-cycle's condensed tail: the levels from the highest one with at most
2500 DOFs (above the coarsest) down, as one operator formed at assembly
(M = 2J - J K J + Q M' Q^T, Q = (I - J K) P, J = omega D^-1; TOP_GPU.m:766-816
in matrix form) and applied by one GEMV.  Checked against the launched steps
it replaces (smoothing products, transfers, coarsest solve), against the
oracle's V-cycle, and for batched right-hand sides."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = b.detach().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _cavity(shape):
    """a box with an internal cavity and a corner notch: void regions on every
    level, no one-voxel bridges (random-fill masks have weakly held voxels on
    which the FP32 V-cycle stalls PCG with or without the tail)"""
    mk = np.ones(shape, bool)
    mk[8:32, 16:48, 8:24] = False
    mk[28:, 20:44, 24:] = False
    return mk


# mask, coarsest-resolution control, optCase, the tail's first level
MODELS = {
    "cantilever_48x96x48": (np.ones((48, 96, 48), bool), 400, 1, 2),       # 4 levels, tail 1911 DOFs
    "cavity_40x64x32": (_cavity((40, 64, 32)), 100, 1, 2),                 # 4 levels, tail 789 DOFs
    "mbb_16x96x16": (np.ones((16, 96, 16), bool), 60, 2, 1),               # 3 levels, tail from level 1
    "cantilever_24x48x24_4lvl": (np.ones((24, 48, 24), bool), 50, 1, 1),   # tail over two levels
}


def _smooth(m):
    """smooth density field in [0.1, 0.95] on the mesh's elements"""
    L0 = m.info()[0]
    eb = m.get(0, "eleMapBack").astype(np.int64) - 1
    y, x, z = eb % L0["resY"], (eb // L0["resY"]) % L0["resX"], eb // (L0["resY"] * L0["resX"])
    return torch.from_numpy(0.1 + 0.85 * np.sin(x / 3.0) ** 2 * np.cos(z / 4.0 + y / 5.0) ** 2).cuda()


def _load(m, s, k=0):
    """load case k's right-hand side (the mesh's F, 3 Nn x nLoads)"""
    return torch.from_numpy(m.get(0, "F")[k * s.numDOFs:(k + 1) * s.numDOFs].copy()).cuda()


def _solver(m, mixed, tol=1e-8):
    from top_gpu_on_matlab_b200.fea import Solver
    s = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=tol, maxIT=2000, omega=0.6, mixed=mixed)
    s.set_density(_smooth(m))
    s.assemble()
    return s


@pytest.fixture(scope="module", params=list(MODELS))
def model(request):
    from top_gpu_on_matlab_b200.fea import Mesh
    mask, control, opt, lvl = MODELS[request.param]
    m = Mesh(mask, control=control)
    m.apply_optcase(opt)
    return m, lvl


def test_tail_fp64_equals_the_launched_steps(model):
    """FP64: the V-cycle with the tail operator equals the launched steps to
    FP64 rounding, and PCG with it reaches the same solution"""
    m, lvl = model
    s = _solver(m, False)
    r = torch.from_numpy(np.random.default_rng(13).standard_normal(s.numDOFs)).cuda()
    assert s.set_tail_operator(None) == 0          # FP64 default: the launched steps
    z0 = s.vcycle(r)
    U0, its0, res0 = s.pcg(0)
    assert s.set_tail_operator(True) == lvl
    z1 = s.vcycle(r)
    U1, its1, res1 = s.pcg(0)
    assert s.set_tail_operator(None) == 0
    assert _rel(z1, z0) < 1e-12
    assert res0 < 1e-8 and res1 < 1e-8
    b = _load(m, s)
    c0, c1 = float(b @ U0), float(b @ U1)
    assert abs(c1 - c0) <= 1e-9 * abs(c0) and _rel(U1, U0) < 1e-6


def test_tail_is_the_mixed_default(model):
    """mixed precision uses the tail by default (M held in FP32, sums in FP64):
    its V-cycle stays within FP32 rounding of the FP64 V-cycle, like the
    launched FP32 steps, and its PCG reaches the FP64 solution"""
    m, lvl = model
    s64 = _solver(m, False)
    s32 = _solver(m, True)
    r = torch.from_numpy(np.random.default_rng(14).standard_normal(s64.numDOFs)).cuda()
    z64 = s64.vcycle(r)
    assert s32.set_tail_operator(None) == lvl
    zt = s32.vcycle(r)
    Ut, _, rest = s32.pcg(0)
    assert s32.set_tail_operator(False) == 0
    zl = s32.vcycle(r)
    assert s32.set_tail_operator(None) == lvl
    assert _rel(zt, z64) < 1e-5 and _rel(zl, z64) < 1e-5
    U64, _, _ = s64.pcg(0)
    b = _load(m, s64)
    c64, ct = float(b @ U64), float(b @ Ut)
    assert rest < 1e-8 and abs(ct - c64) <= 1e-7 * abs(c64)


def test_tail_vcycle_matches_oracle():
    """the tail over two levels (24x48x24, control 50: levels 1 and 2 above the
    coarsest) against the oracle's step-by-step V-cycle"""
    from top_gpu_on_matlab_b200.fea import Mesh
    mask = np.ones((24, 48, 24), bool)
    o = O.Model(mask, control=50)
    o.apply_optcase(1)
    o.set_material(1.0, 1e-9, 3.0)
    o.set_solver(1e-6, 800, 0.6)
    m = Mesh(mask, control=50)
    m.apply_optcase(1)
    s = _solver(m, False)
    x = _smooth(m).cpu().numpy()
    assert x.size == o.level(0).numElements
    o.set_density(x)
    o.assemble()
    assert s.set_tail_operator(True) == 1
    r = np.random.default_rng(6).standard_normal(o.level(0).numDOFs)
    assert _rel(s.vcycle(torch.from_numpy(r).cuda()), o.vcycle(r)) < 1e-11


@pytest.mark.parametrize("mixed", [False, True])
def test_tail_batched_rhs_equal_per_load(mixed):
    """several load cases in one batched PCG pass through the tail GEMV
    together (four right-hand sides per pass of the GEMV): every load case's
    iterates equal its own PCG bit for bit"""
    from top_gpu_on_matlab_b200.fea import Mesh
    ny, nx, nz = 16, 32, 16
    rng = np.random.default_rng(0)

    def node(y, x, z):
        return 1 + y + (ny + 1) * (x + (nx + 1) * z)
    fix = np.array([[node(y, 0, z), 1, 1, 1] for z in range(nz + 1) for y in range(ny + 1)], float)
    dirs = [(0, -1, 0), (0, 0, 1), (0, 0, -1), (0, 1, 0), (1, 0, 0)]
    loads = []
    for k in range(5):
        pts = rng.choice((ny + 1) * (nz + 1), 6, replace=False)
        d = dirs[k]
        loads.append(np.array([[node(int(p % (ny + 1)), nx, int(p // (ny + 1))), *d] for p in pts], float))
    m = Mesh(np.ones((ny, nx, nz), bool), control=20)
    m.apply_bc(fix, loads)
    s = _solver(m, mixed)
    assert s.set_tail_operator(True) == 1
    nd = s.numDOFs
    Ub, its_b, res_b = s.pcg_all()
    for k in range(5):
        Uk, its_k, res_k = s.pcg(k)
        assert its_b[k] == its_k and res_b[k] == res_k, k
        assert torch.equal(Ub[k * nd:(k + 1) * nd], Uk), k


@pytest.mark.parametrize("case", ["no_level", "super_element"])
def test_tail_not_used_where_it_does_not_apply(case):
    """no level between level 1 and the coarsest with at most 2500 DOFs
    (40x80x40, control 3000: level 1 has 7623), or super-element mode (the
    level-0 operator is per-element): the tail reports level 0 and the
    V-cycle is the launched steps', bit for bit"""
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    if case == "no_level":
        m = Mesh(np.ones((40, 80, 40), bool), control=3000)
    else:
        m = Mesh(np.ones((10, 60, 10), bool), control=20000, super_element=1)
    m.apply_optcase(1)
    s = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-6, maxIT=800, omega=0.6, mixed=True)
    s.set_density(torch.full((s.num_design,), 0.5, dtype=torch.float64, device="cuda"))
    s.assemble()
    r = torch.from_numpy(np.random.default_rng(15).standard_normal(s.numDOFs)).cuda()
    assert s.set_tail_operator(None) == 0
    z0 = s.vcycle(r)
    assert s.set_tail_operator(True) == 0
    z1 = s.vcycle(r)
    assert torch.equal(z0, z1)
