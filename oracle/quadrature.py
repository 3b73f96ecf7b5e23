"""Quadrature rules and P1 reference-element data (oracle copy).

The decimals are the reference's literal constants: src/numerics/gauss.py:31-37
(3-point triangle rule, weights 0.166666666666667 -- not exactly 1/6) and
src/numerics/gauss_3D.py:29-39 (4-point tetrahedron rule whose weights sum
to 1, not 1/6).  Basis: gauss.py:154-180, gauss_3D.py:163-199.
"""
import numpy as np

TRI3_POINTS = np.array([[0.166666666666667, 0.166666666666667],
                        [0.166666666666667, 0.666666666666667],
                        [0.666666666666667, 0.166666666666667]])
TRI3_WEIGHTS = np.array([0.166666666666667, 0.166666666666667, 0.166666666666667])

_A, _B = 0.585410196624969, 0.138196601125011
TET4_POINTS = np.array([[_A, _B, _B], [_B, _A, _B], [_B, _B, _A], [_B, _B, _B]])
TET4_WEIGHTS = np.array([0.25, 0.25, 0.25, 0.25])

# d N / d (ksi, eta[, zeta]) on the reference element (gauss.py:154-167, gauss_3D.py:163-180)
TRI_DREF = np.array([[-1.0, 1.0, 0.0], [-1.0, 0.0, 1.0]])
TET_DREF = np.array([[-1.0, 1.0, 0.0, 0.0], [-1.0, 0.0, 1.0, 0.0], [-1.0, 0.0, 0.0, 1.0]])

# 2-point Gauss rule on [-1, 1] used for boundary edges (richards_solver_v2.py:65-66)
EDGE_POINTS = np.array([-1 / np.sqrt(3), 1 / np.sqrt(3)])
EDGE_WEIGHTS = np.array([1.0, 1.0])


def tri_shape(ksi, eta):
    """P1 triangle shape functions (gauss.py:169-180)."""
    return np.array([1 - ksi - eta, ksi, eta])


def tet_shape(ksi, eta, zeta):
    """P1 tetrahedron shape functions (gauss_3D.py:182-199)."""
    return np.array([1.0 - ksi - eta - zeta, ksi, eta, zeta])


def edge_shape(ksi):
    """1D linear shape functions (boundary.py:100-104): rows = nodes, cols = points."""
    return np.stack([(1 - ksi) / 2, (1 + ksi) / 2])
