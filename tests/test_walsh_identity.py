"""The identity the Walsh-basis level-0 kernel is built on, checked on the
oracle's element matrix (CPU): Ke = W B W / 64 with W the 8-point
Walsh-Hadamard transform per displacement component and B block diagonal
over the characters t = s ^ e(c), with the fixed 45-entry sparsity pattern
of the isotropic cube, for any Poisson ratio."""
import numpy as np
import pytest

from oracle import oracle as O

# corner offsets (dy, dx, dz) of the element node map
OFF = [(1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 0), (1, 0, 1), (1, 1, 1), (0, 1, 1), (0, 0, 1)]
AXIS_BIT = [2, 1, 4]                       # component x -> s_x, y -> s_y, z -> s_z
PATTERN = [0x1FF, 0x145, 0x1B0, 0x11B, 0x01B, 0x1B1, 0x155, 0x1FF]


def _w(s, a):
    dy, dx, dz = OFF[a]
    return -1 if ((s & 1) * dy + ((s >> 1) & 1) * dx + ((s >> 2) & 1) * dz) & 1 else 1


def _walsh_matrix():
    W = np.zeros((24, 24))                 # column (s, c) -> DOF (a, c)
    for s in range(8):
        for c in range(3):
            for a in range(8):
                W[3 * a + c, 3 * s + c] = _w(s, a)
    return W


@pytest.mark.parametrize("nu", [0.3, 0.2, 0.45, 0.1])
def test_ke_block_diagonal_in_walsh_basis(nu):
    Ke = O.element_stiffness(nu, 1.0)
    W = _walsh_matrix()
    M = W.T @ Ke @ W / 64.0
    kmax = np.abs(Ke).max()
    Bmask = np.zeros((24, 24), bool)
    for s in range(8):
        for c in range(3):
            for s2 in range(8):
                for d in range(3):
                    t = s ^ AXIS_BIT[c]
                    if (s2 ^ AXIS_BIT[d]) == t and (PATTERN[t] >> (3 * c + d)) & 1:
                        Bmask[3 * s + c, 3 * s2 + d] = True
    assert Bmask.sum() == 45
    assert np.abs(M[~Bmask]).max() <= 1e-13 * kmax
    B = np.where(Bmask, M, 0.0)
    assert np.abs(W @ B @ W.T - Ke).max() <= 1e-13 * kmax


def test_walsh_product_equals_dense_product():
    Ke = O.element_stiffness(0.3, 1.0)
    u = np.random.default_rng(0).standard_normal(24)
    W = _walsh_matrix()
    B = W.T @ Ke @ W / 64.0
    # (y, x) butterflies on each layer, then the z butterfly, as the kernel does
    U = W.T @ u
    assert np.allclose(W @ (B @ U), Ke @ u, rtol=0, atol=1e-13 * np.abs(Ke @ u).max())
