"""Final-step error metrics (drop-in for src/utils/error_calculation.py:9-56)."""
import numpy as np

from wspm_b200 import context

from .exact_solutions import exact_solution


def calculate_final_errors(numerical_results, config):
    points = context.as_host(numerical_results["points"], np.float64)
    h = context.as_host(numerical_results["pressure_head"], np.float64)[-1]
    theta = context.as_host(numerical_results["theta"], np.float64)[-1]
    t = float(context.as_host(numerical_results["times"], np.float64)[-1])
    L, hd = 15.24, -15.24
    a0, ths, thr, ks = (config.exponential.alpha0, config.exponential.thetas, config.exponential.thetar,
                        config.exponential.Ks)
    eps0 = np.exp(a0 * hd)
    d = a0 * (ths - thr) / ks
    n = {"Test1": 1, "Test2": 2, "Test3": 3}[config.test_case]
    h_ex, se_ex = exact_solution(points[:, 0], points[:, 1], t, n, L=L, alpha0=a0, eps0=eps0, d=d)
    se = (theta - thr) / (ths - thr)
    return {"l2_pressure": float(np.sqrt(np.mean((h - h_ex) ** 2))),
            "linf_pressure": float(np.max(np.abs(h - h_ex))),
            "l2_saturation": float(np.sqrt(np.mean((se - se_ex) ** 2))),
            "linf_saturation": float(np.max(np.abs(se - se_ex))),
            "l2_relative_pressure": float(np.sqrt(np.sum((h - h_ex) ** 2)) / np.sqrt(np.sum(h_ex ** 2))),
            "l2_relative_saturation": float(np.sqrt(np.sum((se - se_ex) ** 2)) / np.sqrt(np.sum(se_ex ** 2)))}
