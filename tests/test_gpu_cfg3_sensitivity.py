"""Differentiation workload at full size: cantilever true(64,128,64) (524,288
elements, 1,635,075 DOFs), densities i.i.d. uniform in [0.05, 1] from a fixed
seed, FP64, PCG and filter tolerances 1e-12 (the filter solves at a tenth of
the state tolerance, as TOP_GPU.m:1001 does), rMin 2.5.

Checked on the device's adjoint sensitivities (top_solver_sensitivity):
  * compliance (self-adjoint) and the load-parallel displacement at the
    load-edge midpoint node (true adjoint solve), each
      - unfiltered, against central differences (step 1e-5) on 64 seeded
        elements,
      - through the PDE density filter (ft = 2), against central differences
        of J(filter(x)) on the same elements,
      - through the sensitivity filter (ft = 1), against the reference's
        formula filter(x .* dc) ./ max(1e-3, x) (TOP_GPU.m:213-217) with the
        oracle's filter;
  * the compliance gradient against the reference's sensitivity kernel
    (element energies, TOP_GPU.m:191-198, 580-600) evaluated by the oracle on
    the device's displacement field.
Damped Jacobi omega 0.4: the reference's 0.6 makes the V-cycle indefinite on
i.i.d. densities (in the oracle as on the device).

Central differences: J at x +- h e_k is computed from the state U0 at x as
J(U0 + d), where K(x +- h e_k) d = F - K(x +- h e_k) U0 is solved to a relative
residual of 1e-12 of its own right-hand side -- the same solution as a full
solve, with a solver error that scales with the perturbation instead of with
F, so that differences of two solves resolve the 1e-5 step.  Through the PDE
filter the perturbed design is filter(x) +- h filter(e_k) (the filter is
linear).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHAPE = (64, 128, 64)
E0, EMIN, P, RMIN, TOL, OMEGA = 1.0, 1e-9, 3.0, 2.5, 1e-12, 0.4
H = 1e-5
NFD = 64


@pytest.fixture(scope="module")
def cfg3():
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    m = Mesh(np.ones(SHAPE, bool), control=20000)
    m.apply_optcase(1)
    s = Solver(m, E0=E0, Emin=EMIN, penal=P, tol=TOL, maxIT=4000, omega=OMEGA)
    ne = m.info()[0]["numElements"]
    x = 0.05 + 0.95 * np.random.default_rng(12).random(ne)
    F = m.get(0, "F")
    nz = np.flatnonzero(F)
    dof = int(nz[len(nz) // 2])          # load-parallel DOF of the load-edge midpoint node
    s.filter_setup(RMIN)
    elems = np.random.default_rng(13).choice(ne, NFD, replace=False)
    return m, s, x, torch.from_numpy(F).cuda(), dof, elems


def _state(s, xphys):
    s.set_density(xphys)
    s.assemble()
    U, its, res = s.pcg(0)
    assert res < TOL
    return U


def _J_pert(s, xphys, U0, F, dof):
    """(compliance, U[dof]) at design xphys from a correction solve around U0"""
    s.set_density(xphys)
    s.assemble()
    r0 = F - s.matvec(0, U0)
    d, its, res = s.pcg(b=r0)
    assert res < TOL
    U = U0 + d
    return float(F @ U), float(U[dof])


def _fd_check(s, g, xphys0, dirs, U0, F, dof, which):
    gg = g.cpu().numpy()
    scale = np.abs(gg).max()
    worst = 0.0
    for k, dk in dirs:
        Jp = _J_pert(s, xphys0 + H * dk, U0, F, dof)[which]
        Jm = _J_pert(s, xphys0 - H * dk, U0, F, dof)[which]
        fd = (Jp - Jm) / (2 * H)
        worst = max(worst, abs(fd - gg[k]) / scale)
    return worst


@pytest.mark.parametrize("objective", ["compliance", "displacement"])
def test_unfiltered_gradient_matches_central_differences(cfg3, objective):
    m, s, x, F, dof, elems = cfg3
    xt = torch.from_numpy(x).cuda()
    g, J, _ = s.sensitivity(xt, objective, dof=dof, tol=TOL)
    U0 = _state(s, xt)
    which = 0 if objective == "compliance" else 1
    assert abs(J - (float(F @ U0), float(U0[dof]))[which]) <= 1e-9 * abs(J)
    dirs = []
    for k in elems:
        e = torch.zeros_like(xt)
        e[int(k)] = 1.0
        dirs.append((int(k), e))
    worst = _fd_check(s, g, xt, dirs, U0, F, dof, which)
    print("cfg3 %s unfiltered: max |fd - g| / max|g| = %.2e over %d elements" % (objective, worst, len(dirs)))
    assert worst <= 1e-5


@pytest.mark.parametrize("objective", ["compliance", "displacement"])
def test_density_filter_chain_matches_central_differences(cfg3, objective):
    m, s, x, F, dof, elems = cfg3
    xt = torch.from_numpy(x).cuda()
    xphys, _ = s.filter(xt)
    g, J, _ = s.sensitivity(xphys, objective, dof=dof, ft=2, tol=TOL)
    U0 = _state(s, xphys)
    which = 0 if objective == "compliance" else 1
    dirs = []
    for k in elems:
        e = torch.zeros_like(xt)
        e[int(k)] = 1.0
        fe, _ = s.filter(e)
        dirs.append((int(k), fe))
    worst = _fd_check(s, g, xphys, dirs, U0, F, dof, which)
    print("cfg3 %s through the PDE filter: max |fd - g| / max|g| = %.2e over %d elements" % (objective, worst, len(dirs)))
    assert worst <= 1e-5


@pytest.fixture(scope="module")
def oracle3():
    o = O.Model(np.ones(SHAPE, bool), control=20000)
    o.apply_optcase(1)
    o.set_material(E0, EMIN, P)
    o.set_solver(TOL, 4000, OMEGA)
    o.pde_filter_setup(RMIN)
    yield o
    o.close()


@pytest.mark.parametrize("objective", ["compliance", "displacement"])
def test_sensitivity_filter_chain_matches_reference_formula(cfg3, oracle3, objective):
    m, s, x, F, dof, _ = cfg3
    xt = torch.from_numpy(x).cuda()
    g0, _, _ = s.sensitivity(xt, objective, dof=dof, tol=TOL)
    g1, _, _ = s.sensitivity(xt, objective, dof=dof, ft=1, tol=TOL)
    ref = oracle3.pde_filter(x * g0.cpu().numpy()) / np.maximum(1e-3, x)
    err = np.abs(g1.cpu().numpy() - ref).max() / np.abs(ref).max()
    print("cfg3 %s through the sensitivity filter: %.2e vs the reference formula" % (objective, err))
    assert err <= 1e-8


def test_compliance_gradient_matches_reference_sensitivity_kernel(cfg3, oracle3):
    m, s, x, F, dof, _ = cfg3
    xt = torch.from_numpy(x).cuda()
    g, J, _ = s.sensitivity(xt, "compliance", tol=TOL)
    U = _state(s, xt)
    ce = oracle3.unit_compliance(U.cpu().numpy()[:, None])
    dc_ref = -P * (E0 - EMIN) * x ** (P - 1) * ce
    err = np.abs(g.cpu().numpy() - dc_ref).max() / np.abs(dc_ref).max()
    print("cfg3 compliance gradient vs the reference's sensitivity kernel: %.2e" % err)
    assert err <= 1e-8
