"""van Genuchten-Mualem model (drop-in for src/models/van_genuchten.py:9-79).

``van_genuchten_model(h, phi)`` evaluates C, K and theta for every entry of
``h`` at once on the GPU (the reference vmaps a scalar function).
"""
from wspm_b200 import context
from wspm_b200.device import soil


def van_genuchten_model(h, phi):
    """(C, K, theta) as CUDA float64 tensors; phi = [alpha, theta_S, theta_R, n, m, Ksat]."""
    return soil("vg", context.as_cuda_f64(h), [float(v) for v in context.as_host(phi, float)])


def validate_parameters(phi) -> bool:
    alpha, theta_S, theta_R, n, m, Ksat = [float(v) for v in context.as_host(phi, float)]
    if theta_S <= theta_R:
        raise ValueError("Saturated water content must be greater than residual water content")
    if alpha <= 0:
        raise ValueError("Alpha parameter must be positive")
    if n <= 1:
        raise ValueError("n parameter must be greater than 1")
    if m <= 0 or m >= 1:
        raise ValueError("m parameter must be between 0 and 1")
    if Ksat <= 0:
        raise ValueError("Saturated hydraulic conductivity must be positive")
    if theta_R < 0 or theta_S > 1:
        raise ValueError("Water content values must be between 0 and 1")
    return True
