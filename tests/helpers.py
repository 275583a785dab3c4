import numpy as np


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def ellipsoid_pair(p, sep=3.0, c_axis=0.5):
    """Two smooth ellipsoids on the reference grid, AxisMajor [2][3][Ngrid]."""
    from oracle import sh
    x = sh.legendre_nodes(p)
    th = np.arccos(x)[:, None]
    ph = (np.pi * np.arange(2 * p) / p)[None, :]
    X = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), c_axis * np.cos(th) + 0 * ph]).reshape(3, -1)
    return np.concatenate([X, X + np.array([sep, 0.3, -0.2])[:, None]]).reshape(-1)


def unit_sphere(p):
    from oracle import sh
    x = sh.legendre_nodes(p)
    th = np.arccos(x)[:, None]
    ph = (np.pi * np.arange(2 * p) / p)[None, :]
    return np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th) + 0 * ph]).reshape(-1)


def small_suspension(nves_side, p, seed, spacing=3.0):
    from ves3d_b200 import workloads
    return workloads.suspension(nves_side, p, spacing, semi_axes=(1.0, 1.0, 0.6), deg=4, amp=0.05, seed=seed)
