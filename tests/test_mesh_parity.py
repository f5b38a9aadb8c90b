"""Host mesh model of libtopgpu.so vs the oracle: index maps are bit-exact.

Covers FEA_VoxelBasedDiscretization (TOP_GPU.m:2019-2119), the hierarchy
(1276-1442), the BC generators (505-534), FEA_ApplyBoundaryCondition
(1505-1546) and Solving_SetupKeWithFixedDOFs (1548-1727).
"""
import numpy as np
import pytest

from oracle import oracle as O
from top_gpu_on_matlab_b200.fea import Mesh
from top_gpu_on_matlab_b200._lib import TopGpuError


def _irregular(shape, seed, fill=0.7):
    mk = np.random.default_rng(seed).random(shape) < fill
    mk[:, 0, :] = True
    mk[:, -1, :] = True
    return mk


CASES = [
    ("cantilever 24x48x24 (3 levels)", np.ones((24, 48, 24), bool), 20000, 1, 0),
    ("cantilever 24x48x24, control 50 (4 levels, padded)", np.ones((24, 48, 24), bool), 50, 1, 0),
    ("MBB 10x60x10 (padded)", np.ones((10, 60, 10), bool), 20000, 2, 0),
    ("MBB 10x60x10 super-element", np.ones((10, 60, 10), bool), 20000, 2, 1),
    ("irregular 20x30x14", _irregular((20, 30, 14), 0), 20000, 1, 0),
    ("irregular 12x40x12, control 100", _irregular((12, 40, 12), 4, 0.55), 100, 1, 0),
    ("minimal 3x3x3", np.ones((3, 3, 3), bool), 20000, 1, 0),
]


@pytest.mark.parametrize("name,mask,control,opt,sup", CASES, ids=[c[0] for c in CASES])
def test_maps_bit_exact(name, mask, control, opt, sup):
    o = O.Model(mask, control=control, super_element=sup)
    o.apply_optcase(opt)
    m = Mesh(mask, control=control, super_element=sup)
    m.apply_optcase(opt)
    assert o.numLevels == m.numLevels
    for l in range(o.numLevels):
        L = o.level(l)
        names = ["eleMapBack", "eleMapForward", "eNodMat", "nodMapBack", "nodMapForward", "nodesOnBoundary"]
        names += ["elementsOnBoundary"] if l == 0 else ["elementUpwardMap", "transferMat", "transferMatCoeffi", "RI"]
        for n in names:
            a = getattr(L, n).ravel(order="F")
            b = m.get(l, n)
            assert a.shape == b.shape and np.array_equal(a, b), (l, n)
        if l > 0:
            sm = O._arr(o.m.L[l].solidNodeMapCoarser2Finer, o.m.L[l - 1].numNodes, np.int32)
            assert np.array_equal(sm, m.get(l, "solidNodeMapCoarser2Finer"))
        # element stiffness: closed form (oracle) vs Gauss quadrature (library)
        assert np.abs(m.get(l, "Ke") - L.Ke.ravel(order="F")).max() < 1e-15 * max(1, 2 ** l)
    fr, fx = o.uniqueKes()
    assert np.array_equal(o.mapUniqueKes(), m.get(0, "mapUniqueKes"))
    assert np.array_equal(o.eleWithFixedDOFs(), m.get(0, "eleWithFixedDOFs"))
    assert np.array_equal(o.fixingCond().ravel(order="F"), m.get(0, "fixingCond"))
    assert np.array_equal(o.F().ravel(order="F"), m.get(0, "F"))
    assert np.abs(fr.ravel(order="F") - m.get(0, "uniqueKesFree")).max() < 1e-15
    assert np.array_equal(fx.ravel(order="F"), m.get(0, "uniqueKesFixed"))
    if sup:
        assert np.abs(o.I_mat().ravel(order="F") - m.get(0, "I_mat")).max() < 1e-15


def test_level_counts_match_reference_rule():
    # numLevels = max(3, #halvings while nnz >= control); the 96x192x96 cantilever
    # gets 5 levels with control 400 (6x3x3 coarsest, 336 DOFs)
    m = Mesh(np.ones((96, 192, 96), bool), control=400)
    info = m.info()
    assert [(l["resX"], l["resY"], l["resZ"]) for l in info] == [(192, 96, 96), (48, 24, 24), (24, 12, 12), (12, 6, 6), (6, 3, 3)]
    assert 3 * info[-1]["numNodes"] == 336


def test_generic_bc_multi_load_weights():
    mask = np.ones((6, 10, 6), bool)
    o = O.Model(mask); m = Mesh(mask)
    nodes = O.Model(mask).level(0).nodMapForward
    fix = np.array([[n, 1, 0, 1] for n in range(1, 20)] + [[3, 1, 1, 1]], float)
    loads = [np.array([[200, 0, 0, -1.0], [201, 0, 1.0, 0], [200, 1, 0, 0]]), np.array([[5, 0, 0, 1.0], [210, 0, 0.5, 0]])]
    o.apply_bc(fix, loads); m.apply_bc(fix, loads)
    assert np.array_equal(o.fixingCond().ravel(order="F"), m.get(0, "fixingCond"))
    assert np.array_equal(o.F().ravel(order="F"), m.get(0, "F"))
    assert np.allclose(m.get(0, "objWeights"), [0.5, 0.5])
    assert np.array_equal(o.mapUniqueKes(), m.get(0, "mapUniqueKes"))
    fr, fx = o.uniqueKes()
    assert np.abs(fr.ravel(order="F") - m.get(0, "uniqueKesFree")).max() < 1e-15
    assert np.array_equal(fx.ravel(order="F"), m.get(0, "uniqueKesFixed"))
    del nodes


def test_rejects_small_and_bad_input():
    with pytest.raises(TopGpuError) as ei:
        Mesh(np.ones((2, 8, 8), bool))
    assert "Shape" in ei.value.identifier
    m = Mesh(np.ones((4, 8, 4), bool))
    with pytest.raises(TopGpuError):
        m.apply_bc(np.array([[10 ** 7, 1, 1, 1]], float), [np.array([[2, 0, 0, 1.0]])])
    with pytest.raises(TopGpuError):
        m.apply_optcase(3)
