"""numpy restatement of the .TopVoxel branch of CreateVoxelFEAmodel
(TOP_GPU.m:416-496) with AdaptBCExternalMdl (1743-1793) and
AdaptPassiveElementsExternalMdl (1795-1813).

TEST INFRASTRUCTURE ONLY: the checker of top_mesh_create_from_topvoxel.  It
follows the MATLAB statements one by one -- token reads in fscanf order, the
node / voxel volumes filled, padded with zeros at the end of each axis and
read back with find -- rather than the library's index arithmetic.  Parity
unpinned: the reference's tree holds no model file and its MATLAB driver
cannot run here, so the files come from the synthetic writer.
"""
import numpy as np

from . import oracle as O


class FormatError(ValueError):
    pass


def read(path):
    """Token reads of TOP_GPU.m:418-460; returns the raw file contents."""
    toks = open(path).read().split()
    pos = [0]

    def tok():
        if pos[0] >= len(toks):
            raise FormatError("Incompatible Mesh Data Format!")
        pos[0] += 1
        return toks[pos[0] - 1]

    def expect(w):
        if tok() != w:
            raise FormatError("Incompatible Mesh Data Format!")

    toks4 = [tok() for _ in range(4)]                         # fileHead (418)
    tok()                                                     # versionHead (419)
    version = float(tok())                                    # versionID (420)
    if version != 1.0:
        raise FormatError("Unsupported Data!")
    expect("Resolution:")                                     # 423
    nelx, nely, nelz = int(tok()), int(tok()), int(tok())     # 424-425
    tok(); tok()
    with_density = int(tok())                                 # 426-427
    tok(); tok()
    n_solid = int(tok())                                      # 428-429
    if with_density:                                          # 430-433
        pairs = [(int(tok()), float(tok())) for _ in range(n_solid)]
        solid = np.array([p[0] for p in pairs], dtype=np.int64)
        density = np.array([p[1] for p in pairs])
    else:
        solid = np.array([int(tok()) for _ in range(n_solid)], dtype=np.int64)
        density = np.zeros(0)
    expect("Passive"); expect("elements:")                    # 436-437
    n_passive = int(tok())
    passive = np.array([int(tok()) for _ in range(n_passive)], dtype=np.int64)
    expect("Fixations:")                                      # 441
    n_fix = int(tok())
    fixing = np.array([[int(tok()) for _ in range(4)] for _ in range(n_fix)], dtype=np.int64).reshape(-1, 4)
    expect("Loads:")                                          # 446
    loads = [None]                                            # loadingCond_ = cell(1,1)
    n = int(tok())
    loads[0] = np.array([[int(tok()), float(tok()), float(tok()), float(tok())] for _ in range(n)]).reshape(-1, 4)
    tok(); tok()
    n_more = int(tok())                                       # 451-452
    for _ in range(n_more):                                   # 453-460
        expect("Loads:")
        n, idx = int(tok()), int(tok())
        rows = np.array([[int(tok()), float(tok()), float(tok()), float(tok())] for _ in range(n)]).reshape(-1, 4)
        while len(loads) < idx:
            loads.append(np.zeros((0, 4)))
        loads[idx - 1] = rows
    return dict(header=toks4, nelx=nelx, nely=nely, nelz=nelz, solid=solid, density=density,
                passive=passive, fixing=fixing, loads=loads)


def _pad_volume(vol, shape_to):
    """MATLAB's vol(:, end+1:n, :) = zeros(...) growth along x, then y, then z."""
    out = np.zeros(shape_to, dtype=vol.dtype)
    out[: vol.shape[0], : vol.shape[1], : vol.shape[2]] = vol
    return out


def adapt_bc(src, nel, adjusted_nodes):
    """AdaptBCExternalMdl (TOP_GPU.m:1743-1793): src rows (node, v1, v2, v3) in
    the file's node grid -> the padded node grid adjusted_nodes = (nx, ny, nz)."""
    nelx, nely, nelz = nel
    anx, any_, anz = adjusted_nodes
    null = np.zeros((nelx + 1) * (nely + 1) * (nelz + 1))
    src = np.asarray(src, dtype=np.float64)
    src = src[np.argsort(src[:, 0], kind="stable")]
    idx = src[:, 0].astype(np.int64) - 1
    tmp = np.zeros_like(src)

    def volume(values):
        vol = null.copy()
        vol[idx] = values
        vol = vol.reshape((nely + 1, nelx + 1, nelz + 1), order="F")
        return _pad_volume(vol, (any_, anx, anz)).ravel(order="F")

    new = np.flatnonzero(volume(1.0)) + 1
    tmp[:, 0] = new
    for c in (1, 2, 3):
        tmp[:, c] = volume(src[:, c])[new - 1]
    return tmp


def adapt_passive(src, nel, adjusted_res):
    """AdaptPassiveElementsExternalMdl (TOP_GPU.m:1795-1813)."""
    nelx, nely, nelz = nel
    ax, ay, az = adjusted_res
    vol = np.zeros(nelx * nely * nelz)
    vol[np.sort(np.asarray(src, dtype=np.int64)) - 1] = 1
    vol = vol.reshape((nely, nelx, nelz), order="F")
    return np.flatnonzero(_pad_volume(vol, (ay, ax, az)).ravel(order="F")) + 1


def _unique_first(rows):
    """[~, ia] = unique(rows(:,1)); rows(ia,:) -- first occurrence, ascending"""
    _, ia = np.unique(rows[:, 0], return_index=True)
    return rows[ia]


def create_model(path, control=20000, nu=0.3):
    """The oracle model of a file (TOP_GPU.m:462-496): (Model, passive elements
    in compact numbering, file densities).  Every non-empty load case is moved
    to the compact numbering; the reference does so only when case 1 is not
    empty (TOP_GPU.m:483), leaving other cases in file numbering otherwise."""
    d = read(path)
    nel = (d["nelx"], d["nely"], d["nelz"])
    vox = np.zeros(d["nelx"] * d["nely"] * d["nelz"], dtype=bool)
    vox[d["solid"] - 1] = True
    mask = vox.reshape((d["nely"], d["nelx"], d["nelz"]), order="F")
    o = O.Model(mask, control=control, nu=nu, cell=1.0)
    L0 = o.level(0)
    adj_nodes = (L0.resX + 1, L0.resY + 1, L0.resZ + 1)
    fixing = np.zeros((0, 4))
    if len(d["fixing"]):
        fixing = adapt_bc(_unique_first(d["fixing"].astype(np.float64)), nel, adj_nodes)
        fixing[:, 0] = L0.nodMapForward[fixing[:, 0].astype(np.int64) - 1]
        if np.any(fixing[:, 0] == 0):
            raise FormatError("fixed node touches no solid voxel")
    loads = []
    for rows in d["loads"]:
        if len(rows):
            rows = adapt_bc(_unique_first(rows), nel, adj_nodes)
            rows[:, 0] = L0.nodMapForward[rows[:, 0].astype(np.int64) - 1]
            if np.any(rows[:, 0] == 0):
                raise FormatError("loaded node touches no solid voxel")
        loads.append(rows)
    o.apply_bc(fixing, loads)
    passive = np.zeros(0, dtype=np.int64)
    if len(d["passive"]):
        passive = adapt_passive(d["passive"], nel, (L0.resX, L0.resY, L0.resZ))
        passive = L0.eleMapForward[passive - 1].astype(np.int64)
        if np.any(passive == 0):
            raise FormatError("passive element is not a solid voxel")
    return o, passive, d["density"]
