"""Adjoint sensitivities on the device (top_solver_sensitivity): compliance
against the reference's element-energy sensitivity (TOP_GPU.m:191-198,
580-600, restated by the oracle), a nodal displacement objective against
central finite differences of full solves, and the chain through the
sensitivity filter (formula, as the reference applies it) and the PDE
density filter (finite differences on the design variables)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

E0, EMIN, P = 1.0, 1e-9, 3.0


def _models(shape, omega=0.4, mixed=False, oracle=True):
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    mask = np.ones(shape, bool)
    m = Mesh(mask, control=20000)
    m.apply_optcase(1)
    s = Solver(m, E0=E0, Emin=EMIN, penal=P, tol=1e-10, maxIT=2000, omega=omega, mixed=mixed)
    o = None
    if oracle:
        o = O.Model(mask, control=20000)
        o.apply_optcase(1)
        o.set_material(E0, EMIN, P)
        o.set_solver(1e-12, 2000, omega)
    return o, s, m


def _iid(ne, seed=7):
    """densities i.i.d. uniform in [0.05, 1] from a fixed seed"""
    return 0.05 + 0.95 * np.random.default_rng(seed).random(ne)


def _load_dof(m):
    """the load-parallel DOF at the middle loaded node (the loaded DOFs are the
    nonzero entries of F; the middle one is the load-edge midpoint)"""
    F = m.get(0, "F")
    nz = np.flatnonzero(F)
    return int(nz[len(nz) // 2])


def test_compliance_sensitivity_matches_reference_formula():
    o, s, _ = _models((8, 16, 8))
    ne = o.level(0).numElements
    x = _iid(ne)
    xt = torch.from_numpy(x).cuda()
    g, J, its = s.sensitivity(xt, "compliance", tol=1e-11)
    o.set_density(x)
    o.assemble()
    U, _ = o.solve_state()
    ce = o.unit_compliance(U)
    dc_ref = -P * (E0 - EMIN) * x ** (P - 1) * ce
    E = EMIN + x ** P * (E0 - EMIN)
    assert abs(J - E @ ce) <= 1e-9 * abs(E @ ce)
    gg = g.cpu().numpy()
    assert np.abs(gg - dc_ref).max() <= 1e-8 * np.abs(dc_ref).max()
    assert (gg < 0).all()


def test_displacement_adjoint_matches_central_differences():
    _, s, m = _models((8, 16, 8), oracle=False)
    ne = m.info()[0]["numElements"]
    x = _iid(ne, 3)
    dof = _load_dof(m)
    xt = torch.from_numpy(x).cuda()
    g, J, _ = s.sensitivity(xt, "displacement", dof=dof, tol=1e-12)
    gg = g.cpu().numpy()
    h = 1e-5
    for e in np.random.default_rng(1).choice(ne, 8, replace=False):
        xp, xm = x.copy(), x.copy()
        xp[e] += h
        xm[e] -= h
        _, Jp, _ = s.sensitivity(torch.from_numpy(xp).cuda(), "displacement", dof=dof, tol=1e-12)
        _, Jm, _ = s.sensitivity(torch.from_numpy(xm).cuda(), "displacement", dof=dof, tol=1e-12)
        fd = (Jp - Jm) / (2 * h)
        assert abs(fd - gg[e]) <= 1e-5 * np.abs(gg).max(), (e, fd, gg[e])


def test_displacement_value_matches_oracle_solve():
    o, s, m = _models((8, 16, 8))
    ne = o.level(0).numElements
    x = _iid(ne, 5)
    dof = _load_dof(m)
    _, J, _ = s.sensitivity(torch.from_numpy(x).cuda(), "displacement", dof=dof, tol=1e-12)
    o.set_density(x)
    o.assemble()
    U, _ = o.solve_state()
    assert abs(J - U[dof, 0]) <= 1e-9 * abs(U[dof, 0])


def test_pde_filter_chain_matches_central_differences():
    _, s, m = _models((8, 16, 8), oracle=False)
    ne = m.info()[0]["numElements"]
    s.filter_setup(2.5)
    x = _iid(ne, 9)
    dof = _load_dof(m)

    def J_of(xd):
        xp, _ = s.filter(torch.from_numpy(xd).cuda())
        return s.sensitivity(xp, "displacement", dof=dof, ft=2, tol=1e-12)

    g, _, _ = J_of(x)
    gg = g.cpu().numpy()
    h = 1e-5
    for e in np.random.default_rng(2).choice(ne, 6, replace=False):
        xp, xm = x.copy(), x.copy()
        xp[e] += h
        xm[e] -= h
        fd = (J_of(xp)[1] - J_of(xm)[1]) / (2 * h)
        assert abs(fd - gg[e]) <= 1e-5 * np.abs(gg).max(), (e, fd, gg[e])


def test_sensitivity_filter_chain_matches_reference_formula():
    o, s, _ = _models((8, 16, 8))
    ne = o.level(0).numElements
    x = _iid(ne, 4)
    s.filter_setup(np.sqrt(3))
    o.pde_filter_setup(np.sqrt(3))
    xt = torch.from_numpy(x).cuda()
    g0, _, _ = s.sensitivity(xt, "compliance", tol=1e-11)
    g1, _, _ = s.sensitivity(xt, "compliance", ft=1, tol=1e-11)
    ref = o.pde_filter(x * g0.cpu().numpy()) / np.maximum(1e-3, x)
    assert np.abs(g1.cpu().numpy() - ref).max() <= 1e-8 * np.abs(ref).max()


def test_mixed_precision_sensitivity_tracks_fp64():
    _, s64, m = _models((8, 16, 8), oracle=False)
    _, s32, _ = _models((8, 16, 8), mixed=True, oracle=False)
    ne = m.info()[0]["numElements"]
    xt = torch.from_numpy(_iid(ne, 8)).cuda()
    dof = _load_dof(m)
    for obj in ("compliance", "displacement"):
        g64, J64, _ = s64.sensitivity(xt, obj, dof=dof, tol=1e-10)
        g32, J32, _ = s32.sensitivity(xt, obj, dof=dof, tol=1e-10)
        assert abs(J32 - J64) <= 1e-8 * abs(J64)
        assert float((g32 - g64).abs().max()) <= 1e-6 * float(g64.abs().max())


def test_displacement_adjoint_at_64x128x64():
    """64x128x64 cantilever (524,288 elements) with i.i.d. densities: the
    adjoint displacement gradient against central differences on a few
    seeded elements (damped Jacobi omega 0.4: the reference's 0.6 stalls on
    i.i.d. densities)."""
    _, s, m = _models((64, 128, 64), oracle=False)
    ne = m.info()[0]["numElements"]
    x = _iid(ne, 12)
    dof = _load_dof(m)
    g, J, its = s.sensitivity(torch.from_numpy(x).cuda(), "displacement", dof=dof, tol=1e-11)
    gg = g.cpu().numpy()
    assert np.isfinite(gg).all() and J != 0
    h = 1e-4
    for e in np.random.default_rng(3).choice(ne, 3, replace=False):
        xp, xm = x.copy(), x.copy()
        xp[e] += h
        xm[e] -= h
        Jp = s.sensitivity(torch.from_numpy(xp).cuda(), "displacement", dof=dof, tol=1e-11)[1]
        Jm = s.sensitivity(torch.from_numpy(xm).cuda(), "displacement", dof=dof, tol=1e-11)[1]
        fd = (Jp - Jm) / (2 * h)
        assert abs(fd - gg[e]) <= 1e-4 * np.abs(gg).max(), (e, fd, gg[e])


def test_sensitivity_argument_errors():
    from top_gpu_on_matlab_b200._lib import TopGpuError
    _, s, m = _models((4, 8, 4), oracle=False)
    xt = torch.full((m.info()[0]["numElements"],), 0.5, dtype=torch.float64, device="cuda")
    with pytest.raises(TopGpuError):
        s.sensitivity(xt, "displacement", dof=10 ** 9)
    with pytest.raises(TopGpuError):
        s.sensitivity(xt, "compliance", ft=2)          # no filter set up
