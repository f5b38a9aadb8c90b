"""Fused B200 solver vs the FP64 oracle: operators level by level, V-cycle, PCG."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def smooth_design(level0, resY, resX):
    """Smooth density field in [0.1, 0.95] (optimisation-like, moderate contrast)."""
    eb = level0.eleMapBack - 1
    y, x, z = eb % resY, (eb // resY) % resX, eb // (resY * resX)
    return 0.1 + 0.85 * (np.sin(x / 3.0) ** 2) * (np.cos(z / 4.0 + y / 5.0) ** 2)


def _irregular(shape, seed, fill=0.7):
    mk = np.random.default_rng(seed).random(shape) < fill
    mk[:, 0, :] = True
    mk[:, -1, :] = True
    return mk


MODELS = {
    "cantilever_24x48x24": (np.ones((24, 48, 24), bool), 20000, 1),
    "cantilever_24x48x24_smooth": (np.ones((24, 48, 24), bool), 20000, 1),
    "cantilever_24x48x24_4lvl": (np.ones((24, 48, 24), bool), 50, 1),
    "irregular_20x30x14": (_irregular((20, 30, 14), 0), 20000, 1),
    "mbb_10x60x10": (np.ones((10, 60, 10), bool), 20000, 2),
}


@pytest.fixture(scope="module", params=list(MODELS))
def pair(request):
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    mask, control, opt = MODELS[request.param]
    o = O.Model(mask, control=control)
    o.apply_optcase(opt)
    o.set_material(1.0, 1e-9, 3.0)
    o.set_solver(1e-6, 800, 0.6)
    m = Mesh(mask, control=control)
    m.apply_optcase(opt)
    s = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-6, maxIT=800, omega=0.6)
    ne = o.level(0).numElements
    x = 0.05 + 0.95 * np.random.default_rng(11).random(ne)
    if request.param.endswith("_smooth"):
        L0 = o.level(0)
        x = smooth_design(L0, L0.resY, L0.resX)
    o.set_density(x)
    o.assemble()
    s.set_density(torch.from_numpy(x).cuda())
    s.assemble()
    return o, s, m, ("smooth" if request.param.endswith("_smooth") else "random")


def test_coarse_ks_match(pair):
    o, s, _, _ = pair
    for l in range(1, o.numLevels):
        ref = o.level(l).Ks().ravel(order="F")
        assert _rel(s.Ks(l), ref) < 1e-13, l


def test_diagonals_match(pair):
    o, s, _, _ = pair
    for l in range(o.numLevels - 1):
        assert _rel(s.diag(l), o.level(l).diagK()) < 1e-13, l


@pytest.mark.parametrize("fp32", [False, True])
def test_matvec_every_level(pair, fp32):
    o, s, _, _ = pair
    rng = np.random.default_rng(2)
    for l in range(o.numLevels - 1):
        u = rng.standard_normal(o.level(l).numDOFs)
        ref = o.matvec(l, u)
        y = s.matvec(l, torch.from_numpy(u).cuda(), fp32=fp32)
        assert _rel(y, ref) < (2e-6 if fp32 else 1e-13), (l, fp32)


def test_transfers(pair):
    o, s, _, _ = pair
    rng = np.random.default_rng(4)
    for ii in range(1, o.numLevels):
        rf = rng.standard_normal(o.level(ii - 1).numDOFs)
        xc = rng.standard_normal(o.level(ii).numDOFs)
        assert _rel(s.restrict(ii, torch.from_numpy(rf).cuda()), o.restrict(ii, rf)) < 1e-14
        assert _rel(s.interpolate(ii, torch.from_numpy(xc).cuda()), o.interpolate(ii, xc)) < 1e-14


def test_vcycle_fp64(pair):
    o, s, _, _ = pair
    r = np.random.default_rng(6).standard_normal(o.level(0).numDOFs)
    assert _rel(s.vcycle(torch.from_numpy(r).cuda()), o.vcycle(r)) < 1e-11


_SMOOTHED = set()


def _smooth_only(pair):
    """PCG parity runs on a smooth design on every model: i.i.d. random moduli
    (contrast 8000) make the reference's damped-Jacobi V-cycle (omega 0.6)
    indefinite, in the oracle as on the device.  A model set up with the
    i.i.d. design is switched (oracle and device alike) to the smooth one."""
    o, s, _, kind = pair
    if kind == "smooth" or id(s) in _SMOOTHED:
        return
    L0 = o.level(0)
    x = smooth_design(L0, L0.resY, L0.resX)
    o.set_density(x)
    o.assemble()
    s.set_density(torch.from_numpy(x).cuda())
    s.assemble()
    _SMOOTHED.add(id(s))


def _oracle_spread(o, b, seeds=(1, 2, 3, 4, 5), eps=1e-15):
    """The oracle's own sensitivity to rounding: PCG on b and on b perturbed
    by eps (relative, seeded) -- (min, max) iterations and the compliance
    spread.  On slowly converging models (the irregular mask needs 630-680
    iterations) a 1e-15 perturbation already moves the oracle's iteration
    count by tens and its compliance by ~1e-9; parity is asked for within
    that band."""
    xo, it, _ = o.pcg(b)
    its, cs = [it], [b @ xo]
    for sd in seeds:
        bb = b * (1 + eps * np.random.default_rng(sd).standard_normal(b.size))
        xo, it, _ = o.pcg(bb)
        its.append(it)
        cs.append(b @ xo)
    return min(its), max(its), max(cs) - min(cs)


def test_pcg_fp64_matches_oracle(pair):
    _smooth_only(pair)
    o, s, _, _ = pair
    b = o.F()[:, 0]
    xo, its_o, res_o = o.pcg(b)
    U, its, res = s.pcg(0)
    assert res < 1e-6 and res_o < 1e-6
    c_o, c = b @ xo, float(torch.from_numpy(b).cuda() @ U)      # compliance F'U
    lo, hi, dc = _oracle_spread(o, b)
    print("PCG its device %d, oracle %d (oracle under 1e-15 perturbations: %d..%d); compliance rel diff %.2e "
          "(oracle spread %.2e)" % (its, its_o, lo, hi, abs(c - c_o) / abs(c_o), dc / abs(c_o)))
    # iterations within +-1 of the oracle, or within the oracle's own rounding band
    band = max(1, 2 * (hi - lo))
    assert min(its_o, lo) - band <= its <= max(its_o, hi) + band, (its, its_o, lo, hi)
    # compliance within 1e-9, or within twice the oracle's own spread
    assert abs(c - c_o) <= max(1e-9 * abs(c_o), 2 * dc)


def test_pcg_graphs_match_launches(pair):
    """The CUDA-graph PCG (chunks of four iterations) runs the same kernels in
    the same order as launch-by-launch PCG: identical iterates."""
    _smooth_only(pair)
    _, s, _, _ = pair
    n0 = s.launches
    Ug, its_g, res_g = s.pcg(0)
    n1 = s.launches
    s.set_graphs(False)
    try:
        Ul, its_l, res_l = s.pcg(0)
    finally:
        s.set_graphs(True)
    n2 = s.launches
    assert its_g == its_l and res_g == res_l
    assert torch.equal(Ug, Ul)
    # graph launches count their kernels; whole chunks may run a few extra
    # (early-exiting) iterations
    assert n1 - n0 >= n2 - n1 > 0


@pytest.mark.parametrize("mixed", [False, True])
def test_persistent_coarse_vcycle_matches_per_level_launches(pair, mixed):
    """levels below 0 in one cooperative launch give the per-level launches'
    results bit for bit (same device code, same summation order; the
    condensed tail off, as the persistent kernel runs every level)"""
    o, s, m, _ = pair
    from top_gpu_on_matlab_b200.fea import Solver
    s2 = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-6, maxIT=800, omega=0.6, mixed=mixed)
    x = torch.from_numpy(0.2 + 0.7 * np.random.default_rng(3).random(o.level(0).numElements)).cuda()
    s2.set_density(x)
    s2.assemble()
    s2.set_tail_operator(False)                 # the persistent kernel runs every level
    r = torch.from_numpy(np.random.default_rng(8).standard_normal(o.level(0).numDOFs)).cuda()
    s2.set_coarse_persistent(True)
    za = s2.vcycle(r)
    s2.set_coarse_persistent(2)                 # from level 2 down (level 1 launched per step)
    zc = s2.vcycle(r)
    s2.set_coarse_persistent(False)
    zb = s2.vcycle(r)
    assert torch.equal(za, zb) and torch.equal(zc, zb)


@pytest.mark.parametrize("mixed", [False, True])
def test_dependent_launch_changes_no_result(pair, mixed, monkeypatch):
    """programmatic dependent launch only lets a kernel be scheduled early; it
    waits for its predecessor before reading anything: identical solutions"""
    o, s, m, _ = pair
    from top_gpu_on_matlab_b200.fea import Solver
    x = torch.from_numpy(0.2 + 0.7 * np.random.default_rng(4).random(o.level(0).numElements)).cuda()
    out = []
    for off in (False, True):
        if off:
            monkeypatch.setenv("TOPGPU_NO_PDL", "1")
        s2 = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-8, maxIT=800, omega=0.6, mixed=mixed)
        s2.set_density(x)
        s2.assemble()
        U, its, _ = s2.pcg(0)
        r = torch.from_numpy(np.random.default_rng(8).standard_normal(o.level(0).numDOFs)).cuda()
        out.append((U, its, s2.vcycle(r)))
    assert out[0][1] == out[1][1] and torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][2], out[1][2])


@pytest.mark.parametrize("mixed", [False, True])
def test_vector_transfers_change_no_result(pair, mixed, monkeypatch):
    """span-4 restriction / prolongation with four fine y slots per aligned
    vector access give the per-slot kernels' results bit for bit (every model
    here coarsens by 4 first, with a ragged last y group)"""
    o, s, m, _ = pair
    from top_gpu_on_matlab_b200.fea import Solver
    assert o.level(1).spanWidth == 4
    x = torch.from_numpy(0.2 + 0.7 * np.random.default_rng(5).random(o.level(0).numElements)).cuda()
    out = []
    for off in (False, True):
        if off:
            monkeypatch.setenv("TOPGPU_NO_VEC4", "1")
        s2 = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-8, maxIT=800, omega=0.6, mixed=mixed)
        s2.set_density(x)
        s2.assemble()
        U, its, _ = s2.pcg(0)
        r = torch.from_numpy(np.random.default_rng(9).standard_normal(o.level(0).numDOFs)).cuda()
        out.append((U, its, s2.vcycle(r)))
    assert out[0][1] == out[1][1] and torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][2], out[1][2])


@pytest.mark.parametrize("mixed", [False, True])
def test_two_pass_coarse_product_changes_no_result(pair, mixed, monkeypatch):
    """the two-pass coarse product (packed tiles staged in shared memory,
    element outputs, then node sums) gives the one-pass tile kernel's results
    bit for bit: coarse products in both precisions, V-cycle and PCG"""
    o, s, m, _ = pair
    from top_gpu_on_matlab_b200.fea import Solver
    x = torch.from_numpy(0.2 + 0.7 * np.random.default_rng(5).random(o.level(0).numElements)).cuda()
    rng = np.random.default_rng(8)
    us = [torch.from_numpy(rng.standard_normal(3 * o.level(l).numNodes)).cuda() for l in range(o.numLevels)]
    r = torch.from_numpy(np.random.default_rng(9).standard_normal(o.level(0).numDOFs)).cuda()
    out = []
    for minTiles in ("0", "1000000000"):          # every coarse level two-pass / none
        monkeypatch.setenv("TOPGPU_COARSE_TWOPASS_MIN", minTiles)
        s2 = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-8, maxIT=800, omega=0.6, mixed=mixed)
        s2.set_density(x)
        s2.assemble()
        prods = [s2.matvec(l, us[l], fp32=f) for l in range(1, o.numLevels - 1) for f in (False, True)]
        U, its, _ = s2.pcg(0)
        out.append((prods, U, its, s2.vcycle(r)))
    (pa, Ua, ia, za), (pb, Ub, ib, zb) = out
    assert len(pa) == 2 * (o.numLevels - 2) and all(torch.equal(a, b) for a, b in zip(pa, pb))
    assert ia == ib and torch.equal(Ua, Ub) and torch.equal(za, zb)


def test_filter_graph_matches_launches(pair):
    """the PDE filter's PCG chunks as CUDA graphs give the launch-by-launch result bit for bit"""
    o, s, m, _ = pair
    from top_gpu_on_matlab_b200.fea import Solver
    s2 = Solver(m, E0=1.0, Emin=1e-9, penal=3.0, tol=1e-6, maxIT=800, omega=0.6)
    s2.filter_setup(2.0)
    src = torch.from_numpy(np.random.default_rng(6).random(o.level(0).numElements)).cuda()
    ya, ia = s2.filter(src)
    yb, ib = s2.filter(src)                   # the graph built by the first call, replayed
    s2.set_graphs(False)
    yc, ic = s2.filter(src)
    assert ia == ib == ic and torch.equal(ya, yb) and torch.equal(ya, yc)


def test_pcg_warm_start_and_unit_compliance(pair):
    _smooth_only(pair)
    o, s, _, _ = pair
    U1, its1, _ = s.pcg(0)
    U2, its2, res2 = s.pcg(0, U=U1)
    assert its2 <= 2 and res2 < 1e-6
    ce = s.unit_compliance(U1)
    ce_o = o.unit_compliance(U1.cpu().numpy()[:, None])
    assert _rel(ce, ce_o) < 1e-12


def test_mixed_precision_compliance_within_1e6():
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    mask = np.ones((24, 48, 24), bool)
    o = O.Model(mask); o.apply_optcase(1); o.set_material(1.0, 1e-9, 3.0); o.set_solver(1e-12, 2000, 0.6)
    m = Mesh(mask); m.apply_optcase(1)
    s = Solver(m, E0=1.0, Emin=1e-9, tol=1e-6, maxIT=800, mixed=True)
    L0 = o.level(0)
    x = smooth_design(L0, L0.resY, L0.resX)
    o.set_density(x); o.assemble()
    s.set_density(torch.from_numpy(x).cuda()); s.assemble()
    b = o.F()[:, 0]
    xo, _, _ = o.pcg(b)
    U, its, res = s.pcg(0)
    assert res < 1e-6
    c_o, c = b @ xo, float(torch.from_numpy(b).cuda() @ U)
    assert abs(c - c_o) <= 1e-6 * abs(c_o)


def test_maxit_status():
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    from top_gpu_on_matlab_b200 import TopGpuError
    m = Mesh(np.ones((8, 16, 8), bool)); m.apply_optcase(1)
    s = Solver(m, tol=1e-14, maxIT=3)
    s.set_density(torch.full((m.info()[0]["numElements"],), 0.5, dtype=torch.float64, device="cuda"))
    s.assemble()
    U, its, res = s.pcg(0)
    assert its == 3 and res > 1e-14
    with pytest.raises(TopGpuError) as ei:
        s.pcg(0, raise_on_maxit=True)
    assert ei.value.status == -5


def test_iid_densities_converge_with_smaller_omega():
    # i.i.d. U[0.05,1] densities: omega 0.6 stalls (as in the oracle), 0.4 converges
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    mask = np.ones((8, 16, 8), bool)
    o = O.Model(mask); o.apply_optcase(1); o.set_material(1.0, 1e-9, 3.0); o.set_solver(1e-6, 400, 0.4)
    m = Mesh(mask); m.apply_optcase(1)
    s = Solver(m, Emin=1e-9, tol=1e-6, maxIT=400, omega=0.4)
    x = 0.05 + 0.95 * np.random.default_rng(11).random(mask.size)
    o.set_density(x); o.assemble()
    s.set_density(torch.from_numpy(x).cuda()); s.assemble()
    b = o.F()[:, 0]
    xo, its_o, _ = o.pcg(b)
    U, its, res = s.pcg(0)
    assert res < 1e-6 and abs(its - its_o) <= 1
