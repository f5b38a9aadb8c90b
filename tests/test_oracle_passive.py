"""Passive elements in the oracle's optimisation loop (CPU), the checker for
the device loop: design 1 on them inside the OC bisection and after the
filter (TOP_GPU.m:239, 270), in super-element mode on sub-voxel row Num_ = 4
only (247, 273, as the reference indexes it)."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import topvoxel as OT
from top_gpu_on_matlab_b200.topvoxel import node_index, write_topvoxel


def _model(shape=(8, 16, 8), super_element=0):
    o = O.Model(np.ones(shape, bool), control=500, super_element=super_element)
    o.apply_optcase(1)
    o.set_material(1.0, 1e-9, 3.0)
    o.set_solver(1e-8, 400, 0.6)
    return o


def _slab(o, shape):
    """elements of the first x layer next to the load (x = end) as passive"""
    ny, nx, nz = shape
    emb = o.level(0).eleMapBack - 1
    L0 = o.level(0)
    x = (emb // L0.resY) % L0.resX
    return np.flatnonzero(x == nx - 1) + 1


@pytest.mark.parametrize("ft", [1, 2])
def test_passive_elements_end_at_one(ft):
    shape = (8, 16, 8)
    o = _model(shape)
    ids = _slab(o, shape)
    o.set_passive(ids)
    xp, hist, _ = o.top_opt(V0=0.12, rMin=1.5, nLoop=4, ft=ft)
    assert np.all(xp[ids - 1] == 1.0)
    assert not np.all(xp == 1.0)
    if ft == 1:     # xPhys = xnew: the bisection met the volume with the passive elements counted
        assert abs(xp.mean() - 0.12) < 1e-4


def test_empty_passive_list_changes_nothing():
    a, b = _model(), _model()
    b.set_passive(np.zeros(0, np.int32))
    xa, ha, ca = a.top_opt(V0=0.12, rMin=1.5, nLoop=3, ft=1)
    xb, hb, cb = b.top_opt(V0=0.12, rMin=1.5, nLoop=3, ft=1)
    assert np.array_equal(xa, xb) and np.array_equal(ha, hb) and ca == cb


def test_passive_changes_the_design():
    shape = (8, 16, 8)
    a, b = _model(shape), _model(shape)
    b.set_passive(_slab(b, shape))
    xa, _, _ = a.top_opt(V0=0.12, rMin=1.5, nLoop=3, ft=1)
    xb, _, _ = b.top_opt(V0=0.12, rMin=1.5, nLoop=3, ft=1)
    assert np.abs(xa - xb).max() > 1e-3


def test_super_element_pins_row_num():
    shape = (4, 8, 4)
    o = _model(shape, super_element=1)
    ids = np.array([1, 5, 9])
    o.set_passive(ids)
    xp, _, _ = o.top_opt(V0=0.2, rMin=1.5, nLoop=2, ft=2)
    X = xp.reshape(64, -1, order="F")
    assert np.all(X[3, ids - 1] == 1.0)
    assert not np.all(X[:, ids - 1] == 1.0)


def test_passive_from_a_model_file(tmp_path):
    """the passive list of a .TopVoxel file drives the oracle loop"""
    shape = (6, 12, 6)
    mask = np.ones(shape, bool)
    ys, zs = np.meshgrid(np.arange(shape[0] + 1), np.arange(shape[2] + 1), indexing="ij")
    fix = np.column_stack([node_index(ys.ravel(), 0, zs.ravel(), shape), np.ones((ys.size, 3), int)])
    load = np.array([[node_index(3, shape[1], 0, shape), 0.0, 0.0, -1.0]])
    passive = np.arange(1, shape[0] + 1) + shape[0] * (shape[1] - 1)      # the x = end, z = 0 voxel column
    path = tmp_path / "m.TopVoxel"
    write_topvoxel(path, mask, fix, [load], passive=passive)
    o, pas, _ = OT.create_model(path, control=500)
    o.set_material(1.0, 1e-9, 3.0)
    o.set_solver(1e-8, 400, 0.6)
    o.set_passive(pas)
    xp, _, _ = o.top_opt(V0=0.2, rMin=1.5, nLoop=2, ft=1)
    assert pas.size == shape[0] and np.all(xp[pas - 1] == 1.0)
    with pytest.raises(ValueError):
        o.set_passive([o.level(0).numElements + 1])
