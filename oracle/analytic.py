"""Analytical solutions and final-step error metrics (oracle restatement).

src/utils/exact_solutions.py:4-78 (Tracy-type series, 200 terms) and
src/utils/error_calculation.py:9-56 (RMS "l2", L-infinity and relative L2 of
pressure head and effective saturation at the last recorded time).
"""
import numpy as np


def exact_solution(x, y, t, test_number, L, alpha0, eps0, d, nt=200):
    def series(beta, lind_of, mu_of):
        s = 0.0
        for k in range(1, nt + 1):
            lind = lind_of(k)
            mu = mu_of(lind, beta)
            s = s + ((-1) ** k) * lind / mu * np.sin(lind * y) * np.exp(-mu * t)
        return s

    if test_number == 1:
        beta1 = np.sqrt(0.25 * alpha0 ** 2 + (np.pi / L) ** 2)
        beta3 = np.sqrt(0.25 * alpha0 ** 2 + (3 * np.pi / L) ** 2)
        lind_of = lambda k: np.pi * k / L
        mu_of = lambda lind, beta: (beta ** 2 + lind ** 2) / d
        s1 = series(beta1, lind_of, mu_of)
        s2 = series(beta3, lind_of, mu_of)
        psi1 = 0.75 * np.sin(np.pi * x / L) * (np.sinh(beta1 * y) / np.sinh(beta1 * L) + (2 / (L * d)) * s1)
        psi2 = 0.25 * np.sin(3 * np.pi * x / L) * (np.sinh(beta3 * y) / np.sinh(beta3 * L) + (2 / (L * d)) * s2)
        psi = psi1 - psi2
    elif test_number == 2:
        beta1 = np.sqrt(0.25 * alpha0 ** 2 + (np.pi / L) ** 2)
        lind_of = lambda k: np.pi * k / L
        mu_of = lambda lind, beta: (beta ** 2 + lind ** 2) / d
        s1 = series(beta1, lind_of, mu_of)
        psi = (np.sinh(beta1 * y) / np.sinh(beta1 * L) + (2 / (L * d)) * s1)
        psi = psi * np.sin(np.pi * x / L)
    elif test_number == 3:
        beta1 = np.sqrt(0.25 * alpha0 ** 2 + (2 * np.pi / L) ** 2)
        s1 = 0.0
        for k1 in range(nt + 1):
            lind = np.pi * k1 / L
            mu1 = (0.25 * alpha0 ** 2 + lind ** 2) / d
            mu2 = (0.25 * alpha0 ** 2 + lind ** 2 + (2 * np.pi / L) ** 2) / d
            s1 = s1 + ((-1) ** k1) * lind * (1 / mu1 * np.exp(-mu1 * t)
                                            - 1 / mu2 * np.cos(2 * np.pi * x / L) * np.exp(-mu2 * t)) * np.sin(lind * y)
        psi = (np.sinh(0.5 * alpha0 * y) / np.sinh(0.5 * alpha0 * L)
               - np.cos(2 * np.pi * x / L) * (np.sinh(beta1 * y) / np.sinh(beta1 * L)) + (2 / (L * d)) * s1)
    else:
        raise ValueError("Invalid test number. Please choose 1, 2, or 3.")
    if test_number in (1, 2):
        hb = (1 - eps0) * np.exp(0.5 * alpha0 * (L - y)) * psi
    else:
        hb = 0.5 * (1 - eps0) * np.exp(0.5 * alpha0 * (L - y)) * psi
    hex_ = np.log(np.maximum(eps0 + hb, 1e-10)) / alpha0
    return hex_, np.exp(alpha0 * hex_)


def final_errors(points, pressure_head, theta, final_time, test_number,
                 alpha0=0.164, thetas=0.45, thetar=0.15, Ks=0.1):
    """The six metrics of calculate_final_errors (error_calculation.py:9-56)."""
    L = 15.24
    hd = -15.24
    eps0 = np.exp(alpha0 * hd)
    d = alpha0 * (thetas - thetar) / Ks
    h_ex, se_ex = exact_solution(points[:, 0], points[:, 1], final_time, test_number,
                                 L=L, alpha0=alpha0, eps0=eps0, d=d)
    se = (theta - thetar) / (thetas - thetar)
    return {
        "l2_pressure": float(np.sqrt(np.mean((pressure_head - h_ex) ** 2))),
        "linf_pressure": float(np.max(np.abs(pressure_head - h_ex))),
        "l2_saturation": float(np.sqrt(np.mean((se - se_ex) ** 2))),
        "linf_saturation": float(np.max(np.abs(se - se_ex))),
        "l2_relative_pressure": float(np.sqrt(np.sum((pressure_head - h_ex) ** 2)) / np.sqrt(np.sum(h_ex ** 2))),
        "l2_relative_saturation": float(np.sqrt(np.sum((se - se_ex) ** 2)) / np.sqrt(np.sum(se_ex ** 2))),
    }
