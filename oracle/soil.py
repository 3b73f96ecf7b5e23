"""Soil constitutive models (oracle restatement, vectorised over nodes).

Follows src/models/van_genuchten.py:9-47 and src/models/exponential.py:10-41.
"""
import numpy as np


def van_genuchten_model(h, phi):
    """(C, K, theta) for van Genuchten-Mualem; phi = [alpha, thS, thR, n, m, Ks].

    Literal restatement of src/models/van_genuchten.py:24-47 (jnp.where on
    ``h < 0``; the unselected branch is evaluated but discarded).
    """
    alpha, theta_S, theta_R, n, m, Ksat = [float(v) for v in phi]
    h = np.asarray(h, dtype=np.float64)
    neg = h < 0
    with np.errstate(all="ignore"):
        ah = alpha * np.abs(h)
        theta = np.where(neg, (theta_S - theta_R) * ((1 + ah ** n) ** (-m)) + theta_R, theta_S)
        Se = np.where(neg, (theta - theta_R) / (theta_S - theta_R), 1.0)
        K = np.where(neg, Ksat * ((Se ** 0.5) * (1 - (1 - Se ** (1 / m)) ** m) ** 2), Ksat)
        C = np.where(neg, (theta_S - theta_R) * alpha * m * n * ah ** (n - 1)
                     * (1 + ah ** n) ** (-m - 1), 0.0)
    return C, K, theta


def exponential_model(h, phi):
    """(C, K, theta) for the Gardner exponential model; phi = [alpha0, thS, thR, Ks].

    Literal restatement of src/models/exponential.py:24-41 (``h <= 0``).
    """
    alpha0, tetas, tetar, ks = [float(v) for v in phi]
    h = np.asarray(h, dtype=np.float64)
    nonpos = h <= 0
    with np.errstate(all="ignore"):
        e = np.exp(alpha0 * h)
        theta = np.where(nonpos, (tetas - tetar) * e + tetar, tetas)
        K = np.where(nonpos, ks * e, ks)
        C = np.where(nonpos, alpha0 * (tetas - tetar) * e, 0.0)
    return C, K, theta
