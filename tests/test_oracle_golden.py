"""The FP64 oracle against the reference's own tables and the identities of its algebra."""
import numpy as np
import pytest

from oracle import oracle as O


def test_ke_matches_reference_closed_form(golden):
    # FEA_VoxelBasedElementStiffnessMatrix (TOP_GPU.m:1465-1503), nu = 0.3, cell 1
    Ke = O.element_stiffness(0.3, 1.0)
    assert np.abs(Ke - golden["Ke"]).max() <= 4 * np.finfo(float).eps * np.abs(golden["Ke"]).max()


@pytest.mark.parametrize("span", [2, 4])
def test_ri_tables_match_reference(golden, span):
    assert np.array_equal(O.ri_table(span), golden["RI%d" % span])


@pytest.mark.parametrize("span", [2, 4])
def test_subele_nodmat_matches_reference(golden, span):
    assert np.array_equal(O.subele_nodmat(span), golden["SUB%d" % span])


def _rigid_modes():
    pos = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    modes = []
    for c in range(3):
        v = np.zeros(24); v[c::3] = 1; modes.append(v)
    for a, b in ((0, 1), (1, 2), (0, 2)):
        v = np.zeros(24)
        v[a::3] = -pos[:, b]; v[b::3] = pos[:, a]
        modes.append(v)
    return modes


def test_kat1_ke_symmetric_rigid_body_null():
    Ke = O.element_stiffness(0.3, 0.25)
    assert np.abs(Ke - Ke.T).max() < 1e-15
    for v in _rigid_modes():
        assert np.abs(Ke @ v).max() < 1e-14
    assert np.abs(Ke.sum(axis=1)).max() < 1e-14
    assert np.all(np.linalg.eigvalsh(Ke)[6:] > 1e-3)


def test_super_imat_consistent_with_ke():
    I = O.super_imat(1.0)
    S = I.sum(axis=1).reshape(24, 24, order="F")
    Ke = O.element_stiffness(0.3, 1.0)
    # the 4x4x4 midpoint rule is exact for the constant and bilinear parts:
    # symmetric, same rigid-body null space, close to the exact matrix
    assert np.abs(S - S.T).max() < 1e-14
    for v in _rigid_modes():
        assert np.abs(S @ v).max() < 1e-13
    assert np.abs(S - Ke).max() < 0.05 * np.abs(Ke).max()


@pytest.mark.parametrize("span", [2, 4])
def test_kat3_ri_partition_of_unity(span):
    RI = O.ri_table(span)
    assert np.allclose(RI.sum(axis=1), 1.0, atol=0, rtol=0)


def _assemble_global(m):
    import scipy.sparse as sp
    L0 = m.level(0)
    eN = L0.eNodMat - 1
    dof = np.concatenate([3 * eN[:, [a]] + c for a in range(8) for c in range(3)], axis=1)
    mu = m.mapUniqueKes(); fr, fx = m.uniqueKes()
    E = O._arr(m.m.eleModulus, L0.numElements, np.float64)
    I, J, V = [], [], []
    for e in range(L0.numElements):
        if mu[e] > 0:
            K = fr[:, mu[e] - 1].reshape(24, 24, order="F") * E[e] + fx[:, mu[e] - 1].reshape(24, 24, order="F")
        else:
            K = L0.Ke * E[e]
        I.append(np.repeat(dof[e], 24)); J.append(np.tile(dof[e], 24)); V.append(K.ravel(order="F"))
    n = L0.numDOFs
    return sp.csr_matrix((np.concatenate(V), (np.concatenate(J), np.concatenate(I))), shape=(n, n))


@pytest.fixture(scope="module")
def small_model():
    m = O.Model(np.ones((8, 16, 8), bool))
    m.apply_optcase(1)
    m.set_material(1.0, 1e-9, 3.0)
    m.set_solver(1e-8, 400, 0.6)
    rng = np.random.default_rng(3)
    m.set_modulus(0.05 + rng.random(m.level(0).numElements))
    m.assemble()
    return m


def test_kat4_transfer_multiplicities(small_model):
    for ii in range(1, small_model.numLevels):
        L = small_model.level(ii)
        cnt = np.bincount(L.transferMat.ravel() - 1, minlength=L.intermediateNumNodes)
        assert np.array_equal(cnt.astype(float), L.transferMatCoeffi)


def test_kat5_diag_equals_assembled_diag(small_model):
    K = _assemble_global(small_model)
    assert np.allclose(small_model.level(0).diagK(), K.diagonal(), rtol=1e-14, atol=0)


def test_matvec_equals_assembled_operator(small_model):
    K = _assemble_global(small_model)
    u = np.random.default_rng(1).standard_normal(K.shape[0])
    y = small_model.matvec(0, u)
    assert np.linalg.norm(y - K @ u) <= 1e-13 * np.linalg.norm(K @ u)


def test_kat6_pcg_matches_direct_solve(small_model):
    import scipy.sparse.linalg as spl
    K = _assemble_global(small_model)
    b = small_model.F()[:, 0]
    x, its, res = small_model.pcg(b, tol=1e-10)
    xs = spl.spsolve(K.tocsc(), b)
    assert res < 1e-10 and its < 200
    assert np.linalg.norm(x - xs) <= 1e-8 * np.linalg.norm(xs)


def test_kat2_galerkin_consistency():
    # a solid, unconstrained coarse cell with all children at E = 1:
    # sum_s P_s' K0 P_s == Ke * span  (TOP_GPU.m:1066 relies on this)
    for span in (2, 4):
        Ke = O.element_stiffness(0.3, 1.0)
        nch = span ** 3
        RI = O.ri_table(span)
        SUB = O.subele_nodmat(span)
        P = np.zeros((24, 24, nch))
        for s in range(nch):
            for i in range(8):
                for c in range(3):
                    P[3 * i + c, c::3, s] = RI[SUB[s, i] - 1, :]
        up = np.arange(1, nch + 1, dtype=np.int32).reshape(1, nch)
        Ks = O.assemble_ks_level2(up, np.ones(nch), Ke, P, np.zeros(nch, np.int32), None, None)
        assert np.abs(Ks[:, :, 0] - Ke * span).max() < 1e-13


def test_coarse_operator_is_galerkin_of_fine(small_model):
    # level-2 Ks equals the Galerkin product R K1 P when children pair with their
    # own interpolation block; for span 2 the reference pairs child slots with
    # the listed sub-element order (TOP_GPU.m:1941-1948 vs 1330-1336)
    m = small_model
    L1 = m.level(1)
    Ks = L1.Ks()
    assert np.abs(Ks - np.transpose(Ks, (1, 0, 2))).max() < 1e-12 * np.abs(Ks).max()
    for e in range(Ks.shape[2]):
        w = np.linalg.eigvalsh(Ks[:, :, e])
        assert w.min() > -1e-10 * w.max()


def test_vcycle_is_symmetric_positive(small_model):
    rng = np.random.default_rng(5)
    n = small_model.level(0).numDOFs
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    Ma, Mb = small_model.vcycle(a), small_model.vcycle(b)
    assert abs(b @ Ma - a @ Mb) <= 1e-10 * abs(b @ Ma)
    assert a @ Ma > 0


def test_restrict_is_transpose_of_interpolate(small_model):
    rng = np.random.default_rng(9)
    for ii in range(1, small_model.numLevels):
        nf, nc = small_model.level(ii - 1).numDOFs, small_model.level(ii).numDOFs
        a, b = rng.standard_normal(nf), rng.standard_normal(nc)
        lhs = small_model.restrict(ii, a) @ b
        rhs = a @ small_model.interpolate(ii, b)
        assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_kat7_compliance_sensitivity_fd():
    # unfiltered dc/dE_e = -u_e' Ke u_e for compliance b'u, central differences
    m = O.Model(np.ones((6, 12, 6), bool))
    m.apply_optcase(1)
    m.set_material(1.0, 1e-9, 3.0)
    m.set_solver(1e-12, 500, 0.6)
    ne = m.level(0).numElements
    E = 0.3 + 0.7 * np.random.default_rng(2).random(ne)
    m.set_modulus(E); m.assemble()
    b = m.F()[:, 0]
    U, _ = m.solve_state()
    ce = m.unit_compliance(U)
    for e in (5, 77, ne - 3):
        h = 1e-3
        Ep, Em = E.copy(), E.copy(); Ep[e] += h; Em[e] -= h
        m.set_modulus(Ep); m.assemble(); up, _ = m.solve_state()
        m.set_modulus(Em); m.assemble(); um, _ = m.solve_state()
        fd = (b @ up[:, 0] - b @ um[:, 0]) / (2 * h)
        assert abs(fd + ce[e]) <= 5e-6 * abs(ce[e])
