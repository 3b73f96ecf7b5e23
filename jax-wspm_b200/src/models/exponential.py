"""Gardner exponential model (drop-in for src/models/exponential.py:10-84)."""
from wspm_b200 import context
from wspm_b200.device import soil


def exponential_model(h, phi):
    """(C, K, theta) as CUDA float64 tensors; phi = [alpha0, tetas, tetar, ks]."""
    return soil("exp", context.as_cuda_f64(h), [float(v) for v in context.as_host(phi, float)])


def compute_soil_properties(pressure_head, soil_params):
    return exponential_model(pressure_head, soil_params)


def validate_parameters(soil_params) -> bool:
    alpha0, tetas, tetar, ks = [float(v) for v in context.as_host(soil_params, float)]
    if tetas <= tetar:
        raise ValueError("Saturated water content must be greater than residual water content")
    if alpha0 <= 0:
        raise ValueError("Alpha parameter must be positive")
    if ks <= 0:
        raise ValueError("Saturated hydraulic conductivity must be positive")
    if tetar < 0 or tetas > 1:
        raise ValueError("Water content values must be between 0 and 1")
    return True
