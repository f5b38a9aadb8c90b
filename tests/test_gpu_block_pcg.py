"""Several load cases solved as one batched PCG (top_solver_pcg_all): every
operator launched once per iteration for all right-hand sides, one
recurrence and stopping test per right-hand side.  The iterates are those of
the per-load-case PCG (the reference solves load cases one after the other,
TOP_GPU.m:181-187), checked bit for bit, and the solutions against the oracle."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _multi_load(shape, nload, seed=0):
    """x = 0 face fixed; nload unit loads on seeded nodes of the x = max face"""
    ny, nx, nz = shape
    rng = np.random.default_rng(seed)
    # compact node numbers of a full box: y fastest, then x, then z (1-based)
    def node(y, x, z):
        return 1 + y + (ny + 1) * (x + (nx + 1) * z)
    fix = np.array([[node(y, 0, z), 1, 1, 1] for z in range(nz + 1) for y in range(ny + 1)], float)
    dirs = [(0, -1, 0), (0, 0, 1), (0, 0, -1), (0, 1, 0), (1, 0, 0)]
    loads = []
    for k in range(nload):
        pts = rng.choice((ny + 1) * (nz + 1), 6, replace=False)
        d = dirs[k % len(dirs)]
        rows = [[node(int(p % (ny + 1)), nx, int(p // (ny + 1))), d[0], d[1], d[2]] for p in pts]
        loads.append(np.array(rows, float))
    return fix, loads


def _pair(shape, nload, mixed=False):
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    mask = np.ones(shape, bool)
    fix, loads = _multi_load(shape, nload)
    o = O.Model(mask, control=20000)
    o.apply_bc(fix, loads)
    o.set_material(1.0, 1e-9, 3.0)
    o.set_solver(1e-8, 800, 0.6)
    m = Mesh(mask, control=20000)
    m.apply_bc(fix, loads)
    s = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-8, maxIT=800, omega=0.6, mixed=mixed)
    L0 = o.level(0)
    eb = L0.eleMapBack - 1
    y, x, z = eb % L0.resY, (eb // L0.resY) % L0.resX, eb // (L0.resY * L0.resX)
    xd = 0.1 + 0.85 * np.sin(x / 3.0) ** 2 * np.cos(z / 4.0 + y / 5.0) ** 2
    o.set_density(xd)
    o.assemble()
    s.set_density(torch.from_numpy(xd).cuda())
    s.assemble()
    return o, s


@pytest.mark.parametrize("mixed", [False, True])
def test_batched_pcg_equals_per_load_pcg(mixed):
    o, s = _pair((12, 24, 12), 4, mixed)
    nd = s.numDOFs
    Ub, its_b, res_b = s.pcg_all()
    for k in range(4):
        Uk, its_k, res_k = s.pcg(k)
        assert its_b[k] == its_k and res_b[k] == res_k, k
        assert torch.equal(Ub[k * nd:(k + 1) * nd], Uk), k


def test_batched_pcg_matches_oracle():
    o, s = _pair((12, 24, 12), 3)
    nd = s.numDOFs
    Ub, its_b, res_b = s.pcg_all()
    U_o, _ = o.solve_state()
    F = o.F()
    for k in range(3):
        u = Ub[k * nd:(k + 1) * nd].cpu().numpy()
        c, c_o = F[:, k] @ u, F[:, k] @ U_o[:, k]
        assert abs(c - c_o) <= 1e-7 * abs(c_o), k
        assert res_b[k] < 1e-8


def test_batched_pcg_warm_start():
    _, s = _pair((8, 16, 8), 2)
    U, its, _ = s.pcg_all()
    U2, its2, res2 = s.pcg_all(U)
    assert max(its2) <= 2 and max(res2) < 1e-8


def test_optimisation_loop_with_four_load_cases_matches_oracle():
    """the loop's state solves run as one batched PCG over the load cases;
    summed (weighted) compliance per iteration against the oracle"""
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    shape = (10, 20, 10)
    mask = np.ones(shape, bool)
    fix, loads = _multi_load(shape, 4, seed=3)
    o = O.Model(mask, control=20000)
    o.apply_bc(fix, loads)
    o.set_material(1.0, 1e-9, 3.0)
    o.set_solver(1e-9, 800, 0.6)
    m = Mesh(mask, control=20000)
    m.apply_bc(fix, loads)
    s = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-9, maxIT=800, omega=0.6)
    xo, ho, cso = o.top_opt(V0=0.3, rMin=np.sqrt(3), nLoop=4, ft=2)
    xg, hg, csg = s.optimize(V0=0.3, rMin=np.sqrt(3), nLoop=4, ft=2)
    assert abs(csg - cso) <= 1e-9 * abs(cso)
    for k, (a, b) in enumerate(zip(hg, ho)):
        assert abs(a["c"] - b[0]) <= 1e-6 * abs(b[0]), k
    assert np.abs(xg.cpu().numpy() - xo).max() <= 1e-6
