"""The oracle's polydisperse double layer and viscosity contrast (CPU): with one order they
are the uniform oracle's (stokes_velocity_sl + stokes_velocity_dl, ImplicitStep with the
contrast), and with mixed orders the double layer of a constant density meets Gauss's
identity at every surface point (-c/2 on its own vesicle, 0 from the others)."""
import numpy as np

from oracle import sh, stokes
from oracle import surface as su
from tests.helpers import rel_err, small_suspension
from ves3d_b200 import workloads


def test_poly_dl_single_order_is_uniform():
    p = 6
    X, f = small_suspension(2, p, 61, spacing=2.7)
    nv = X.size // (3 * sh.ngrid(p))
    g = np.random.default_rng(62).standard_normal(X.size)
    u = stokes.stokes_velocity_poly(X, f, np.full(nv, p), g=g)
    ref = stokes.stokes_velocity_sl(X, f, p) + stokes.stokes_velocity_dl(X, g, p)
    assert rel_err(u, ref) < 1e-13


def test_poly_dl_gauss_identity_mixed_orders():
    X, _, orders = workloads.polydisperse(4, orders=(6, 8), radius=(0.8, 1.2), volume_fraction=0.05, seed=63)
    assert len(set(orders.tolist())) == 2
    c = np.array([0.4, -1.0, 0.7])
    g = np.concatenate([np.repeat(c[:, None], sh.ngrid(int(p)), axis=1).reshape(-1) for p in orders])
    u = stokes.stokes_velocity_poly(X, np.zeros_like(X), orders, g=g)
    k = 0
    for p in orders:
        ng = sh.ngrid(int(p))
        blk = u[k:k + 3 * ng].reshape(3, ng)
        assert np.abs(blk + 0.5 * c[:, None]).max() < 2e-3, p  # jump value on the surface
        k += 3 * ng


def test_poly_contrast_single_order_is_uniform():
    p = 6
    X, _ = small_suspension(2, p, 64, spacing=2.7)
    nv = X.size // (3 * sh.ngrid(p))
    lam = np.linspace(0.2, 4.0, nv)
    a = su.ImplicitStep(X, p, 0.05, 0.01, 1.0, viscosity_contrast=lam)
    b = su.PolyImplicitStep(X, np.full(nv, p), 0.05, 0.01, 1.0, viscosity_contrast=lam)
    z = np.random.default_rng(65).standard_normal(4 * X.size // 3)
    assert rel_err(b.matvec(z), a.matvec(z)) < 1e-13
