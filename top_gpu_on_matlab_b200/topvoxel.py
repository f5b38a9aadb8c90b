"""Synthetic .TopVoxel model files, format version 1.0 -- the token layout the
file branch of CreateVoxelFEAmodel reads (TOP_GPU.m:416-496) and
top_mesh_create_from_topvoxel parses:

    # TopVoxel model file
    Version: 1.0
    Resolution: nelx nely nelz
    Density values: 0|1
    Solid voxels: N
    voxel [density]                 (N lines)
    Passive elements: P
    voxel ...
    Fixations: F
    node fixX fixY fixZ             (F lines)
    Loads: L
    node fx fy fz                   (load case 1)
    Additional loads: A
    Loads: L case                   (then L lines of load case `case`)

Voxels are 1-based linear indices of the nely x nelx x nelz grid and nodes of
the (nely+1) x (nelx+1) x (nelz+1) node grid, y fastest (MATLAB order).
"""
import numpy as np


def voxel_index(y, x, z, shape):
    """1-based linear index of voxel (y, x, z) of a nely x nelx x nelz grid."""
    ny, nx, _ = shape
    return 1 + np.asarray(y) + ny * (np.asarray(x) + nx * np.asarray(z))


def node_index(y, x, z, shape):
    """1-based linear index of node (y, x, z) of the voxel grid's node grid."""
    ny, nx, _ = shape
    return 1 + np.asarray(y) + (ny + 1) * (np.asarray(x) + (nx + 1) * np.asarray(z))


def _rows(f, rows, fmt):
    if len(rows):
        f.write("\n".join(fmt % tuple(r) for r in rows) + "\n")


def _load_rows(f, rows):
    if len(rows):
        f.write("\n".join("%d %.17g %.17g %.17g" % (int(r[0]), r[1], r[2], r[3]) for r in rows) + "\n")


def write_topvoxel(path, mask, fixations, loads, passive=(), density=None):
    """Write a model file.

    mask: [nely, nelx, nelz] bool; fixations: rows (node, fixX, fixY, fixZ);
    loads: a list of load cases, each rows (node, fx, fy, fz) -- case 1 goes in
    the Loads block, case k > 1 in an additional block numbered k (an empty
    case gets no block: between others it reads back as an empty case, at the
    end it is dropped, since a file holds the cases up to its highest block
    number); passive: 1-based voxel indices; density:
    one value per solid voxel, in ascending voxel order (the file then carries
    densities).  Values are written with 17 significant digits, so they read
    back exactly."""
    mask = np.asarray(mask, dtype=bool)
    ny, nx, nz = mask.shape
    solid = np.flatnonzero(mask.ravel(order="F")) + 1
    if density is not None:
        density = np.asarray(density, dtype=np.float64)
        if density.shape != solid.shape:
            raise ValueError("density needs one value per solid voxel")
    fixations = np.asarray(fixations, dtype=np.int64).reshape(-1, 4)
    loads = [np.asarray(l, dtype=np.float64).reshape(-1, 4) for l in loads]
    if not loads:
        raise ValueError("at least one load case")
    more = [(case, l) for case, l in enumerate(loads, start=1) if case > 1 and len(l)]
    with open(path, "w") as f:
        f.write("# TopVoxel model file\n")
        f.write("Version: 1.0\n")
        f.write("Resolution: %d %d %d\n" % (nx, ny, nz))
        f.write("Density values: %d\n" % (density is not None))
        f.write("Solid voxels: %d\n" % solid.size)
        if density is None:
            if solid.size:
                f.write("\n".join(map(str, solid.tolist())) + "\n")
        elif solid.size:
            f.write("\n".join("%d %.17g" % vd for vd in zip(solid.tolist(), density.tolist())) + "\n")
        passive = np.asarray(passive, dtype=np.int64).ravel()
        f.write("Passive elements: %d\n" % passive.size)
        if passive.size:
            f.write(" ".join("%d" % p for p in passive) + "\n")
        f.write("Fixations: %d\n" % len(fixations))
        _rows(f, fixations, "%d %d %d %d")
        f.write("Loads: %d\n" % len(loads[0]))
        _load_rows(f, loads[0])
        f.write("Additional loads: %d\n" % len(more))
        for case, l in more:
            f.write("Loads: %d %d\n" % (len(l), case))
            _load_rows(f, l)
