"""Device optimisation loop vs the oracle: PDE filter (TOP_GPU.m:880-1031),
sensitivities, OC bisection and the full loop (141-292)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _pair(mask, opt, tol, control=20000, omega=0.6):
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    o = O.Model(mask, control=control)
    o.apply_optcase(opt)
    o.set_material(1.0, 1e-9, 3.0)
    o.set_solver(tol, 800, omega)
    m = Mesh(mask, control=control)
    m.apply_optcase(opt)
    s = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=tol, maxIT=800, omega=omega)
    return o, s


@pytest.mark.parametrize("shape", [(24, 48, 24), (12, 30, 10)])
def test_pde_filter_matches_oracle(shape):
    o, s = _pair(np.ones(shape, bool), 1, 1e-6)
    rmin = np.sqrt(3)
    o.pde_filter_setup(rmin)
    s.filter_setup(rmin)
    src = np.random.default_rng(4).random(o.level(0).numElements)
    ref = o.pde_filter(src)
    out, its = s.filter(torch.from_numpy(src).cuda())
    assert _rel(out, ref) < 1e-10


def test_filter_preserves_constants():
    _, s = _pair(np.ones((8, 16, 8), bool), 1, 1e-8)
    s.filter_setup(2.5)
    one = torch.ones(s.levels[0]["numElements"], dtype=torch.float64, device="cuda")
    out, _ = s.filter(one)
    # a constant field is a fixed point of the Helmholtz filter (zero-flux boundary)
    assert float((out - 1).abs().max()) < 1e-6


@pytest.mark.parametrize("ft,opt,shape", [(1, 1, (12, 24, 12)), (2, 2, (10, 20, 10))])
def test_optimisation_loop_matches_oracle(ft, opt, shape):
    o, s = _pair(np.ones(shape, bool), opt, 1e-9)
    nloop = 8
    xo, ho, cso = o.top_opt(V0=0.12, rMin=np.sqrt(3), nLoop=nloop, ft=ft)
    xg, hg, csg = s.optimize(V0=0.12, rMin=np.sqrt(3), nLoop=nloop, ft=ft)
    assert abs(csg - cso) <= 1e-9 * abs(cso)
    assert len(hg) == len(ho)
    for k, (a, b) in enumerate(zip(hg, ho)):
        assert abs(a["c"] - b[0]) <= 1e-6 * abs(b[0]), k
        assert abs(a["vol"] - b[1]) <= 1e-9, k
        assert abs(a["change"] - b[4]) <= 1e-6, k
    assert np.abs(xg.cpu().numpy() - xo).max() <= 1e-6


def test_mixed_precision_loop_tracks_fp64():
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    mask = np.ones((12, 24, 12), bool)
    res = {}
    for mixed in (False, True):
        m = Mesh(mask); m.apply_optcase(1)
        s = Solver(m, Emin=1e-9, tol=1e-6, maxIT=800, mixed=mixed)
        xp, hist, cs = s.optimize(V0=0.12, nLoop=6, ft=1)
        res[mixed] = (xp.cpu().numpy(), [h["c"] for h in hist])
    c64, c32 = np.array(res[False][1]), np.array(res[True][1])
    assert np.abs(c32 - c64).max() <= 1e-6 * np.abs(c64).max()
    assert np.abs(res[True][0] - res[False][0]).max() <= 1e-4


def test_design_host_round_trip_and_launch_count():
    """set_design / get_design through pinned host memory: an iteration
    started from a design that went down and up again equals one started
    from the device state; every step launches kernels."""
    _, a = _pair(np.ones((8, 16, 8), bool), 1, 1e-9)
    _, b = _pair(np.ones((8, 16, 8), bool), 1, 1e-9)
    a.opt_begin(V0=0.12, rMin=np.sqrt(3), nLoop=50, ft=1)
    b.opt_begin(V0=0.12, rMin=np.sqrt(3), nLoop=50, ft=1)
    ra, rb = a.opt_step(), b.opt_step()
    ne = a.levels[0]["numElements"]
    xp = torch.empty(ne, dtype=torch.float64).pin_memory()
    x = torch.empty(ne, dtype=torch.float64).pin_memory()
    b.get_design_into(xp, x)
    b.set_design(xp, x)
    n0 = b.launches
    ra, rb = a.opt_step(), b.opt_step()
    assert b.launches > n0
    assert ra["c"] == rb["c"]
    xa, _ = a.design()
    xb, _ = b.design()
    assert torch.equal(xa, xb)
