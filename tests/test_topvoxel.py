""".TopVoxel model files (CPU): the library's reader (top_mesh_create_from_topvoxel)
against the oracle's restatement of CreateVoxelFEAmodel's file branch
(TOP_GPU.m:416-496, AdaptBCExternalMdl 1743-1793, AdaptPassiveElementsExternalMdl
1795-1813) on synthetic files, the writer's round trip, and the format errors."""
import numpy as np
import pytest

from oracle import topvoxel as OT
from top_gpu_on_matlab_b200._lib import TopGpuError
from top_gpu_on_matlab_b200.fea import Mesh
from top_gpu_on_matlab_b200.topvoxel import node_index, voxel_index, write_topvoxel


def synthetic(shape, seed, n_cases=2, density=False, duplicates=True):
    """Irregular domain with solid x = 0 and x = end faces; fixations on the
    x = 0 face (mixed per-component flags), loads on the x = end face, passive
    voxels scattered over the solid ones."""
    rng = np.random.default_rng(seed)
    ny, nx, nz = shape
    mask = rng.random(shape) < 0.7
    mask[:, 0, :] = True
    mask[:, -1, :] = True
    ys, zs = np.meshgrid(np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    fnodes = node_index(ys.ravel(), 0, zs.ravel(), shape)
    flags = rng.integers(0, 2, size=(fnodes.size, 3))
    flags[:, 0] = 1
    fix = np.column_stack([fnodes, flags])
    loads = []
    for _ in range(n_cases):
        pick = rng.choice(fnodes.size, size=max(2, fnodes.size // 5), replace=False)
        lnodes = node_index(ys.ravel()[pick], nx, zs.ravel()[pick], shape)
        loads.append(np.column_stack([lnodes, rng.standard_normal((lnodes.size, 3))]))
    if duplicates:        # repeated nodes: the first row of a node counts
        fix = np.vstack([fix, np.column_stack([fnodes[:5], np.zeros((5, 3), int)])])
        loads[0] = np.vstack([loads[0], np.column_stack([loads[0][:3, 0], 9.0 * np.ones((3, 3))])])
    solid = np.flatnonzero(mask.ravel(order="F")) + 1
    passive = rng.choice(solid, size=max(1, solid.size // 50), replace=False)
    if duplicates:
        passive = np.concatenate([passive, passive[:2]])
    dens = rng.random(solid.size) if density else None
    return mask, fix, loads, passive, dens


CASES = [((20, 30, 14), 0, 2, False), ((12, 24, 12), 1, 1, True), ((9, 17, 7), 2, 3, True)]


@pytest.mark.parametrize("shape,seed,n_cases,density", CASES)
def test_reader_matches_oracle(tmp_path, shape, seed, n_cases, density):
    mask, fix, loads, passive, dens = synthetic(shape, seed, n_cases, density)
    path = tmp_path / "model.TopVoxel"
    write_topvoxel(path, mask, fix, loads, passive=passive, density=dens)
    m = Mesh.from_topvoxel(path, control=500)
    o, passive_o, dens_o = OT.create_model(path, control=500)
    assert m.shape == shape
    assert m.numLevels == o.numLevels
    assert np.array_equal(m.get(0, "eleMapBack"), o.level(0).eleMapBack)
    assert np.array_equal(m.get(0, "fixingCond").reshape(-1, 4, order="F"), o.fixingCond())
    assert np.array_equal(m.get(0, "F"), o.F().ravel(order="F"))
    assert np.array_equal(m.get(0, "objWeights"), o.objWeights())
    assert np.allclose(o.objWeights(), 1.0 / n_cases)
    assert np.array_equal(m.passive_elements, passive_o)
    assert np.array_equal(m.density_layout, dens_o)
    if dens is not None:
        assert np.array_equal(m.density_layout, dens)


def test_padding_moves_bc_nodes(tmp_path):
    """a resolution that the hierarchy pads (20 x 30 x 14 -> multiples of 8): the
    compact fixed nodes are those of the same (y, x, z) positions"""
    mask, fix, loads, passive, _ = synthetic((20, 30, 14), 3, duplicates=False)
    path = tmp_path / "model.TopVoxel"
    write_topvoxel(path, mask, fix, loads, passive=passive)
    m = Mesh.from_topvoxel(path, control=500)
    info = m.info()[0]
    assert (info["resY"], info["resX"], info["resZ"]) != (20, 30, 14)
    back = m.get(0, "nodMapBack")            # compact node -> padded grid node (1-based)
    py, px = info["resY"] + 1, info["resX"] + 1
    g = back[m.get(0, "fixingCond").reshape(-1, 4, order="F")[:, 0] - 1] - 1
    y, x, z = g % py, (g // py) % px, g // (py * px)
    assert np.all(x == 0) and y.max() == 20 and z.max() == 14


def test_writer_round_trip_and_empty_case(tmp_path):
    mask, fix, loads, passive, dens = synthetic((9, 17, 7), 4, n_cases=3, density=True)
    loads[1] = np.zeros((0, 4))                # an empty case between two others
    path = tmp_path / "model.TopVoxel"
    write_topvoxel(path, mask, fix, loads, passive=passive, density=dens)
    d = OT.read(path)
    assert (d["nely"], d["nelx"], d["nelz"]) == mask.shape
    assert np.array_equal(d["solid"], np.flatnonzero(mask.ravel(order="F")) + 1)
    assert np.array_equal(d["density"], dens)
    assert np.array_equal(d["passive"], passive)
    assert np.array_equal(d["fixing"], fix)
    assert len(d["loads"]) == 3 and len(d["loads"][1]) == 0
    assert np.array_equal(d["loads"][0], loads[0]) and np.array_equal(d["loads"][2], loads[2])
    # an empty load case stops the BC set-up, as FEA_ApplyBoundaryCondition's
    # 'No Loads!' does (TOP_GPU.m:1519)
    _expect_error(path, "No Loads!")
    with pytest.raises(ValueError):
        OT.create_model(path, control=500)


def _expect_error(path, text):
    with pytest.raises(TopGpuError) as e:
        Mesh.from_topvoxel(path, control=500)
    assert text in str(e.value)


def _base_file(tmp_path):
    mask, fix, loads, passive, _ = synthetic((6, 8, 5), 5, n_cases=1, duplicates=False)
    path = tmp_path / "base.TopVoxel"
    write_topvoxel(path, mask, fix, loads, passive=passive)
    return path, path.read_text()


def test_format_errors(tmp_path):
    path, text = _base_file(tmp_path)
    bad = tmp_path / "bad.TopVoxel"
    bad.write_text(text.replace("Version: 1.0", "Version: 2.0"))
    _expect_error(bad, "Unsupported Data!")
    with pytest.raises(OT.FormatError, match="Unsupported"):
        OT.read(bad)
    bad.write_text(text.replace("Resolution:", "Resolutions:"))
    _expect_error(bad, "Incompatible Mesh Data Format!")
    bad.write_text(text.replace("Fixations:", "Fixings:"))
    _expect_error(bad, "Incompatible Mesh Data Format!")
    bad.write_text(text[: len(text) // 2])
    _expect_error(bad, "Incompatible Mesh Data Format!")
    bad.write_text(text.replace("Passive elements: ", "Passive elements: 999999999999 "))
    _expect_error(bad, "Incompatible Mesh Data Format!")
    _expect_error(tmp_path / "missing.TopVoxel", "cannot open")


def test_bc_on_void_is_rejected(tmp_path):
    shape = (8, 8, 8)
    mask = np.ones(shape, bool)
    mask[2:6, 2:6, 2:6] = False              # a void pocket; node (4, 4, 4) touches no solid voxel
    fix = np.array([[node_index(0, 0, 0, shape), 1, 1, 1], [node_index(4, 4, 4, shape), 1, 1, 1]])
    loads = [np.array([[node_index(0, 7, 0, shape), 0.0, 0.0, -1.0]])]
    path = tmp_path / "void.TopVoxel"
    write_topvoxel(path, mask, fix, loads)
    _expect_error(path, "touches no solid voxel")
    with pytest.raises(OT.FormatError):
        OT.create_model(path, control=500)
    write_topvoxel(path, mask, fix[:1], loads, passive=[voxel_index(3, 3, 3, shape)])
    _expect_error(path, "is not a solid voxel")


def test_corrupted_files_fail_cleanly(tmp_path):
    """seeded token corruption (dropped, duplicated, replaced, huge or negative
    numbers): every file either loads or fails with a status, never crashes"""
    path, text = _base_file(tmp_path)
    toks = text.split()
    rng = np.random.default_rng(7)
    bad = tmp_path / "fuzz.TopVoxel"
    outcomes = {"ok": 0, "error": 0}
    for _ in range(200):
        t = list(toks)
        for _ in range(int(rng.integers(1, 4))):
            k = int(rng.integers(0, len(t)))
            op = int(rng.integers(0, 4))
            if op == 0:
                del t[k]
            elif op == 1:
                t.insert(k, t[k])
            elif op == 2:
                t[k] = str(int(rng.choice([-1, 0, 2 ** 31, 2 ** 62, 10 ** 30])))
            else:
                t[k] = rng.choice(["x", "1e400", "nan", "-0", "Loads:"])
        bad.write_text(" ".join(t))
        try:
            Mesh.from_topvoxel(bad, control=500).close()
            outcomes["ok"] += 1
        except TopGpuError:
            outcomes["error"] += 1
    assert outcomes["error"] > 0 and sum(outcomes.values()) == 200
