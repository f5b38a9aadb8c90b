"""Passive elements in the device optimisation loop against the oracle
(TOP_GPU.m:239, 270: design 1 on them in the OC bisection and after the
filter), same tolerances as the loop without them."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pair(mask, opt, tol):
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    o = O.Model(mask)
    o.apply_optcase(opt)
    o.set_material(1.0, 1e-9, 3.0)
    o.set_solver(tol, 800, 0.6)
    m = Mesh(mask)
    m.apply_optcase(opt)
    s = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=tol, maxIT=800, omega=0.6)
    return o, s


def _last_x_layer(o):
    """elements of the last x layer (next to the cantilever's load)"""
    L0 = o.level(0)
    emb = L0.eleMapBack - 1
    x = (emb // L0.resY) % L0.resX
    return (np.flatnonzero(x == x.max()) + 1).astype(np.int32)


@pytest.mark.parametrize("ft,opt,shape", [(1, 1, (12, 24, 12)), (2, 2, (10, 20, 10))])
def test_passive_loop_matches_oracle(ft, opt, shape):
    o, s = _pair(np.ones(shape, bool), opt, 1e-9)
    ids = _last_x_layer(o)
    o.set_passive(ids)
    s.set_passive(ids)
    nloop = 6
    xo, ho, cso = o.top_opt(V0=0.12, rMin=np.sqrt(3), nLoop=nloop, ft=ft)
    xg, hg, csg = s.optimize(V0=0.12, rMin=np.sqrt(3), nLoop=nloop, ft=ft)
    assert abs(csg - cso) <= 1e-9 * abs(cso)
    assert len(hg) == len(ho)
    for k, (a, b) in enumerate(zip(hg, ho)):
        assert abs(a["c"] - b[0]) <= 1e-6 * abs(b[0]), k
        assert abs(a["vol"] - b[1]) <= 1e-9, k
        assert abs(a["change"] - b[4]) <= 1e-6, k
    x = xg.cpu().numpy()
    assert np.all(x[ids - 1] == 1.0)
    assert np.abs(x - xo).max() <= 1e-6
    s.set_passive([])                          # cleared: the next run has none
    xg2, _, _ = s.optimize(V0=0.12, rMin=np.sqrt(3), nLoop=2, ft=ft)
    assert not np.all(xg2.cpu().numpy()[ids - 1] == 1.0)
