"""Transport utilities (drop-in for src/models/transport_utilities.py:118-242) on the device.

``calculate_fluxes_and_dispersion_FE`` runs ``wspm_flux_dispersion_2d`` (the
per-node mean of incident P1 gradients by row gather instead of the
reference's O(N*E) scan); ``calculate_peclet_courant`` runs
``wspm_peclet_courant``.  Arrays in, CUDA float64 tensors out.
"""
import numpy as np

from wspm_b200 import context
from wspm_b200.device import flux_dispersion, peclet_courant


def calculate_fluxes_and_dispersion_FE(points, triangles, pressure_head, phi, DL, DT, Dm):
    """(qx, qz, |q|, Dxx, Dxz, Dzz, theta) per node (transport_utilities.py:118-192)."""
    dm = context.mesh_for(points, triangles)
    return flux_dispersion(dm, context.as_cuda_f64(pressure_head), tuple(np.asarray(phi, dtype=np.float64)), DL,
                           DT, Dm)


def calculate_element_size(points, triangles):
    """Shortest edge per triangle (transport_utilities.py:196-203)."""
    v = np.asarray(points)[np.asarray(triangles)]
    e = v - np.roll(v, 1, axis=1)
    return np.min(np.sqrt(np.sum(e ** 2, axis=2)), axis=1)


def calculate_peclet_courant(points, triangles, water_flux_x, water_flux_z, theta, Dispersion_xx, Dispersion_zz,
                             dt):
    """(max Peclet, max Courant) over the mesh (transport_utilities.py:205-242)."""
    dm = context.mesh_for(points, triangles)
    f = context.as_cuda_f64
    out = peclet_courant(dm, f(water_flux_x), f(water_flux_z), f(theta), f(Dispersion_xx), f(Dispersion_zz), dt)
    pe, cr = out.cpu().numpy()
    return float(pe), float(cr)
