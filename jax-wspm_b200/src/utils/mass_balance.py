"""Mass balance of a Richards run (the reference's richards_mass_balance driver, an editor checkpoint:
src/solvers/.ipynb_checkpoints/richards_mass_balance-checkpoint.py:25-69, 247-332).

``integrate_2d_domain`` runs ``wspm_integrate_2d`` (same 3-point rule and
|det J| weighting as the reference, hence twice the integral); the balance
error of a run is |1 - (M_num(t) - M_0) / (M_exact(t) - M_0)| * 100 as there.
"""
import numpy as np

from wspm_b200 import context
from wspm_b200.device import integrate_2d


def integrate_2d_domain(f, points, triangles):
    return float(integrate_2d(context.mesh_for(points, triangles), context.as_cuda_f64(f)))


def mass_balance_error(mass_numerical, mass_exact, initial_mass):
    """Percent error of the numerical against the exact mass change (checkpoint :336-339)."""
    num = np.asarray(mass_numerical) - initial_mass
    ex = np.asarray(mass_exact) - initial_mass
    return np.abs(1.0 - num / ex) * 100.0
