"""Per-load-case PCG iteration counts of an optimisation step (the reference's
lssIts, TOP_GPU.m:186): one count per case, summing to the record's count."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_case_iterations_sum_to_record(tmp_path):
    from top_gpu_on_matlab_b200.fea import Mesh, Solver
    from top_gpu_on_matlab_b200.topvoxel import node_index, write_topvoxel
    shape = (8, 16, 8)
    ys, zs = np.meshgrid(np.arange(shape[0] + 1), np.arange(shape[2] + 1), indexing="ij")
    fix = np.column_stack([node_index(ys.ravel(), 0, zs.ravel(), shape), np.ones((ys.size, 3), int)])
    loads = [np.array([[node_index(4, shape[1], 0, shape), 0.0, 0.0, -1.0]]),
             np.array([[node_index(0, shape[1], 4, shape), 0.0, -1.0, 0.0],
                       [node_index(8, shape[1], 4, shape), 0.0, 1.0, 0.0]])]
    path = tmp_path / "two_loads.TopVoxel"
    write_topvoxel(path, np.ones(shape, bool), fix, loads)
    m = Mesh.from_topvoxel(path)
    s = Solver(m, E0=1.0, Emin=1e-9, tol=1e-6, maxIT=800, omega=0.6)
    assert s.nLoads == 2
    s.opt_begin(V0=0.3, nLoop=3, ft=1)
    for _ in range(2):
        rec = s.opt_step()
        its = s.opt_case_its()
        assert len(its) == 2 and all(k > 0 for k in its) and sum(its) == rec["pcgIts"]
