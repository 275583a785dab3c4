"""The oracle's restatement of the near-singular correction (oracle/near.py) on the CPU:
its spherical-harmonic point evaluation against the grid transforms and finite
differences, its projection, and the sphere identities it recovers near the surface."""
import numpy as np

from oracle import near, sh, stokes
from tests.helpers import small_suspension, unit_sphere


def test_point_basis_matches_grid_and_finite_differences():
    p = 10
    X, _ = small_suspension(1, p, 3)
    S3 = sh.grid2shc(X, p, p).reshape(3, -1)
    th, ph = near.grid_angles(p)
    for k in (0, 37, 150):
        assert np.abs(S3 @ near.basis(p, th[k], ph[k])[0] - X.reshape(3, -1)[:, k]).max() < 1e-13
    t0, p0, h = 0.7, 1.3, 1e-6
    _, bt, bp = near.basis(p, t0, p0)
    fd_t = (near.basis(p, t0 + h, p0)[0] - near.basis(p, t0 - h, p0)[0]) / (2 * h)
    fd_p = (near.basis(p, t0, p0 + h)[0] - near.basis(p, t0, p0 - h)[0]) / (2 * h)
    assert np.abs(bt - fd_t).max() < 1e-8 and np.abs(bp - fd_p).max() < 1e-8


def test_projection_on_a_sphere_is_radial_with_outward_normal():
    p = 8
    a = 2.0
    S3 = sh.grid2shc(a * unit_sphere(p), p, p).reshape(3, -1)
    th, ph = near.grid_angles(p)
    T = np.array([0.3, 2.5, 0.4])
    _, _, P, nu = near.project(S3, p, T, th[50], ph[50])
    assert abs(np.linalg.norm(P) - a) < 1e-13
    assert np.abs(P / a - T / np.linalg.norm(T)).max() < 1e-12
    assert abs(nu @ (P / a) - 1.0) < 1e-12


def test_near_correction_recovers_sphere_identities():
    p = 8
    a = 2.0
    X = a * unit_sphere(p)
    ng = sh.ngrid(p)
    c = np.array([0.3, -1.0, 0.5])
    g = np.repeat(c[:, None], ng, axis=1).reshape(-1)
    dirs = np.random.default_rng(0).normal(size=(4, 3))
    dirs /= np.linalg.norm(dirs, axis=1)[:, None]
    T = np.concatenate([dirs * (a + 0.02), dirs * (a - 0.02)])
    r = np.linalg.norm(T, axis=1)
    ref = np.where((r > a)[:, None], 0.0, -c[None])
    u = near.target_velocity_near(X, np.zeros_like(g), p, T, g=g)
    u0 = stokes.target_velocity(X, np.zeros_like(g), p, T, g).reshape(-1, 3)
    assert np.abs(u0 - ref).max() > 0.1      # smooth quadrature alone
    assert np.abs(u - ref).max() < 1e-3      # corrected
