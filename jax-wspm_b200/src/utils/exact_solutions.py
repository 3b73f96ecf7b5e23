"""Tracy-type analytical solutions for Test1/2/3 (drop-in for src/utils/exact_solutions.py:4-78).

Host NumPy, evaluated once per run at the last recorded time.
"""
import numpy as np


def _series(y, t, nt, beta, d, L):
    k = np.arange(1, nt + 1, dtype=np.float64)
    lind = np.pi * k / L
    mu = (beta ** 2 + lind ** 2) / d
    terms = ((-1.0) ** k)[:, None] * (lind / mu)[:, None] * np.sin(np.outer(lind, y)) * np.exp(-mu * t)[:, None]
    # sum in k order, as the reference's accumulation loop does
    s = np.zeros_like(np.asarray(y, dtype=np.float64))
    for row in terms:
        s = s + row
    return s


def exact_solution(x, y, t, test_number, L, alpha0, eps0, d, nt=200):
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    if test_number == 1:
        b1 = np.sqrt(0.25 * alpha0 ** 2 + (np.pi / L) ** 2)
        b3 = np.sqrt(0.25 * alpha0 ** 2 + (3 * np.pi / L) ** 2)
        s1, s2 = _series(y, t, nt, b1, d, L), _series(y, t, nt, b3, d, L)
        psi = (0.75 * np.sin(np.pi * x / L) * (np.sinh(b1 * y) / np.sinh(b1 * L) + (2 / (L * d)) * s1)
               - 0.25 * np.sin(3 * np.pi * x / L) * (np.sinh(b3 * y) / np.sinh(b3 * L) + (2 / (L * d)) * s2))
    elif test_number == 2:
        b1 = np.sqrt(0.25 * alpha0 ** 2 + (np.pi / L) ** 2)
        psi = (np.sinh(b1 * y) / np.sinh(b1 * L) + (2 / (L * d)) * _series(y, t, nt, b1, d, L)) * np.sin(np.pi * x / L)
    elif test_number == 3:
        b1 = np.sqrt(0.25 * alpha0 ** 2 + (2 * np.pi / L) ** 2)
        s1 = np.zeros_like(y)
        for k1 in range(nt + 1):
            lind = np.pi * k1 / L
            mu1 = (0.25 * alpha0 ** 2 + lind ** 2) / d
            mu2 = (0.25 * alpha0 ** 2 + lind ** 2 + (2 * np.pi / L) ** 2) / d
            s1 = s1 + ((-1) ** k1) * lind * (1 / mu1 * np.exp(-mu1 * t)
                                            - 1 / mu2 * np.cos(2 * np.pi * x / L) * np.exp(-mu2 * t)) * np.sin(lind * y)
        psi = (np.sinh(0.5 * alpha0 * y) / np.sinh(0.5 * alpha0 * L)
               - np.cos(2 * np.pi * x / L) * (np.sinh(b1 * y) / np.sinh(b1 * L)) + (2 / (L * d)) * s1)
    else:
        raise ValueError("Invalid test number. Please choose 1, 2, or 3.")
    scale = 1.0 if test_number in (1, 2) else 0.5
    hb = scale * (1 - eps0) * np.exp(0.5 * alpha0 * (L - y)) * psi
    hex_ = np.log(np.maximum(eps0 + hb, 1e-10)) / alpha0
    return hex_, np.exp(alpha0 * hex_)
