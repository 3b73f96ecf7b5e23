"""Tetrahedron quadrature and P1 basis (drop-in for src/numerics/gauss_3D.py:10-199).

The 4-point rule's weights are the reference's 0.25 each (they sum to 1, not
1/6, so every element integral is 6x the true value; mass, stiffness and
gravity scale together, so the solution is unaffected).
"""
import numpy as np


def gauss_tetrahedron(n: int):
    if n == 1:
        return np.array([[0.25, 0.25, 0.25]]), np.array([1.0])
    if n == 4:
        a, b = 0.585410196624969, 0.138196601125011
        return (np.array([[a, b, b], [b, a, b], [b, b, a], [b, b, b]]), np.array([0.25, 0.25, 0.25, 0.25]))
    if n == 5:
        a, b, c = 0.25, 0.5, 1 / 6
        return (np.array([[a, a, a], [b, c, c], [c, b, c], [c, c, b], [c, c, c]]),
                np.array([-0.8, 0.45, 0.45, 0.45, 0.45]))
    raise ValueError("n must be 1, 4 or 5 (the rules the reference's solvers use)")


def basis_ksi_eta_zeta(ksi, eta, zeta):
    return np.array([[-1.0, 1.0, 0.0, 0.0], [-1.0, 0.0, 1.0, 0.0], [-1.0, 0.0, 0.0, 1.0]])


def interpolation_3d(ksi, eta, zeta):
    return np.array([1.0 - ksi - eta - zeta, ksi, eta, zeta])
