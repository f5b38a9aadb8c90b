"""Super-element mode in the fused solver (TOP_GPU.m:721-741 K·u with
K_mat = I_mat·E_sub, 1101-1104; level-2 Galerkin with the super-element
children, assembleKs_level2_superEle_inplace.cu:70-173) against the oracle:
element matrices, coarse Ks, diagonals, products on every level, V-cycle, PCG."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _smooth_sub(ny, nx, nz):
    """smooth sub-voxel densities in [0.15, 0.95], element-major [64 x Ne]"""
    fy, fx, fz = 4 * ny, 4 * nx, 4 * nz
    y, x, z = np.meshgrid(np.arange(fy), np.arange(fx), np.arange(fz), indexing="ij")
    f = 0.15 + 0.8 * np.sin(x / 7.0) ** 2 * np.cos(z / 5.0 + y / 9.0) ** 2
    out = np.zeros(fy * fx * fz)
    # element-major order: q = ly + 4 (lx + 4 lz), element = ey + ny (ex + nx ez)
    for lz in range(4):
        for lx in range(4):
            for ly in range(4):
                q = ly + 4 * (lx + 4 * lz)
                blk = f[ly::4, lx::4, lz::4]             # [ny, nx, nz]
                out[q::64] = blk.ravel(order="F")
    return out


@pytest.fixture(scope="module", params=[(10, 60, 10, 2), (6, 16, 6, 1)])
def super_pair(request):
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    ny, nx, nz, opt = request.param
    mask = np.ones((ny, nx, nz), bool)
    o = O.Model(mask, control=20000, super_element=1)
    o.apply_optcase(opt)
    o.set_material(1.0, 1e-9, 3.0)
    o.set_solver(1e-8, 800, 0.6)
    m = Mesh(mask, control=20000, super_element=1)
    m.apply_optcase(opt)
    s = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-8, maxIT=800, omega=0.6)
    x = _smooth_sub(ny, nx, nz)
    o.set_density(x)
    o.assemble()
    s.set_density(torch.from_numpy(x).cuda())
    s.assemble()
    return o, s, m


def test_super_element_matrices(super_pair):
    o, s, m = super_pair
    K = s.Ks(0).cpu().numpy().reshape(576, -1, order="F")
    Kref = o.K_mat()
    free = o.mapUniqueKes() == 0            # elements without fixed DOFs: K_mat = I_mat E_sub
    assert _rel(K[:, free], Kref[:, free]) < 1e-13


def test_super_coarse_ks_and_diagonals(super_pair):
    o, s, _ = super_pair
    for l in range(1, o.numLevels):
        assert _rel(s.Ks(l), o.level(l).Ks().ravel(order="F")) < 1e-12, l
    for l in range(o.numLevels - 1):
        assert _rel(s.diag(l), o.level(l).diagK()) < 1e-12, l


@pytest.mark.parametrize("fp32", [False, True])
def test_super_matvec_every_level(super_pair, fp32):
    o, s, _ = super_pair
    rng = np.random.default_rng(3)
    for l in range(o.numLevels - 1):
        u = rng.standard_normal(o.level(l).numDOFs)
        y = s.matvec(l, torch.from_numpy(u).cuda(), fp32=fp32)
        assert _rel(y, o.matvec(l, u)) < (2e-6 if fp32 else 1e-12), (l, fp32)


def test_super_vcycle_and_pcg(super_pair):
    o, s, _ = super_pair
    r = np.random.default_rng(6).standard_normal(o.level(0).numDOFs)
    assert _rel(s.vcycle(torch.from_numpy(r).cuda()), o.vcycle(r)) < 1e-10
    b = o.F()[:, 0]
    xo, its_o, _ = o.pcg(b)
    U, its, res = s.pcg(0)
    # several hundred iterations: rounding differences move the stopping
    # iteration by a few percent; the solution agrees to the tolerance
    assert abs(its - its_o) <= max(1, 0.1 * its_o) and res < 1e-8
    c_o, c = b @ xo, float(torch.from_numpy(b).cuda() @ U)
    assert abs(c - c_o) <= 1e-7 * abs(c_o)


def test_super_optimisation_loop_matches_oracle():
    """cfg1-like MBB beam in super-element mode: true(10,60,10), 4x4x4
    sub-voxels, optCase 2, ft = 2 (the super-element density filter), V0 0.2."""
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    mask = np.ones((10, 60, 10), bool)
    o = O.Model(mask, control=20000, super_element=1)
    o.apply_optcase(2)
    o.set_material(1.0, 1e-9, 3.0)
    o.set_solver(1e-9, 800, 0.6)
    m = Mesh(mask, control=20000, super_element=1)
    m.apply_optcase(2)
    s = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-9, maxIT=800, omega=0.6)
    nloop = 4
    xo, ho, cso = o.top_opt(V0=0.2, rMin=np.sqrt(3), nLoop=nloop, ft=2)
    xg, hg, csg = s.optimize(V0=0.2, rMin=np.sqrt(3), nLoop=nloop, ft=2)
    assert abs(csg - cso) <= 1e-9 * abs(cso)
    assert len(hg) == len(ho)
    for k, (a, b) in enumerate(zip(hg, ho)):
        assert abs(a["c"] - b[0]) <= 1e-6 * abs(b[0]), k
        assert abs(a["vol"] - b[1]) <= 1e-9, k
    assert np.abs(xg.cpu().numpy() - xo).max() <= 1e-6


def _to_fine(v, ny, nx, nz):
    f = np.zeros((4 * ny, 4 * nx, 4 * nz))
    for lz in range(4):
        for lx in range(4):
            for ly in range(4):
                q = ly + 4 * (lx + 4 * lz)
                f[ly::4, lx::4, lz::4] = v[q::64].reshape((ny, nx, nz), order="F")
    return f


@pytest.mark.parametrize("mode", [0, 1])
def test_super_density_filter_matches_imfilter(mode):
    """imfilter(A, h) with zero padding (scipy.ndimage.correlate, mode
    'constant'), h = max(0, 4 rMin - dist), Hs = imfilter(ones, h)."""
    from scipy import ndimage
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    ny, nx, nz = 6, 16, 6
    m = Mesh(np.ones((ny, nx, nz), bool), control=20000, super_element=1)
    m.apply_optcase(1)
    s = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-8, maxIT=800, omega=0.6)
    rmin = np.sqrt(3)
    s.super_filter_setup(rmin)
    v = np.random.default_rng(mode).random(64 * ny * nx * nz)
    out = s.super_filter(torch.from_numpy(v).cuda(), mode).cpu().numpy()
    r = 4 * rmin
    R = int(np.ceil(r)) - 1
    d = np.arange(-R, R + 1)
    DY, DX, DZ = np.meshgrid(d, d, d, indexing="ij")
    h = np.maximum(0, r - np.sqrt(DY ** 2 + DX ** 2 + DZ ** 2))
    Hs = ndimage.correlate(np.ones((4 * ny, 4 * nx, 4 * nz)), h, mode="constant")
    g = _to_fine(v, ny, nx, nz)
    ref = ndimage.correlate(g / Hs, h, mode="constant") if mode == 0 else ndimage.correlate(g, h, mode="constant") / Hs
    assert np.abs(_to_fine(out, ny, nx, nz) - ref).max() <= 1e-12 * np.abs(ref).max()
