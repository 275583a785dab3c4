"""Near-singular correction of the off-surface targets (NearSingular, src/NearSingular.cc
of the reference, as StokesVelocity composes it for SetTrgCoord targets) on the GPU:
against the oracle's restatement (oracle/near.py) at 1e-10, and against the sphere
identities at targets down to 0.5% of the radius from the surface, where the smooth
quadrature alone is off by O(1)."""
import numpy as np
import pytest

from oracle import near, sh, stokes
from tests.helpers import rel_err, small_suspension, unit_sphere
from ves3d_b200.stokes_velocity import StokesVelocity

pytestmark = pytest.mark.gpu


def _targets_near(X, p, rng, n, dists):
    """Targets at the given distances off random surface points, outside and inside."""
    ng = sh.ngrid(p)
    Xv = X.reshape(-1, 3, ng)
    nrm = stokes.unit_normal(X, p).reshape(-1, 3, ng)
    out = []
    for i in range(n):
        v, k = rng.integers(Xv.shape[0]), rng.integers(ng)
        d = dists[i % len(dists)] * (1 if i % 2 == 0 else -1)
        out.append(Xv[v, :, k] + d * nrm[v, :, k])
    return np.array(out)


@pytest.mark.parametrize("with_dl", [False, True])
def test_near_correction_matches_oracle(with_dl):
    p = 8
    X, f = small_suspension(2, p, 31, spacing=2.6)
    rng = np.random.default_rng(32)
    g = rng.standard_normal(X.size) if with_dl else None
    T = np.concatenate([_targets_near(X, p, rng, 12, [0.02, 0.1, 0.3]), rng.uniform(-2.0, 5.0, (6, 3))])
    ref, info = near.target_velocity_near(X, f, p, T, g=g, return_info=True)
    assert len(info["pairs"]) >= 8
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        if with_dl:
            sv.SetDensityDL(g)
        sv.SetTrgCoord(T)
        sv.set_near_singular(True)
        u = sv.eval_targets().reshape(-1, 3)
        r_near, n_near = sv.near_info()
        sv.set_near_singular(False)
        u0 = sv.eval_targets().reshape(-1, 3)
    assert abs(r_near - info["r_near"]) < 1e-13 * r_near
    assert n_near == len(info["pairs"])
    assert rel_err(u, ref) < 1e-10
    # off again: the plain smooth quadrature of the order-p points, as before
    assert rel_err(u0, stokes.target_velocity(X, f, p, T, g).reshape(-1, 3)) < 1e-12


def test_near_correction_sphere_identities():
    """Unit-density single layer on a sphere of radius 2 (inside 2a/3 f, outside the
    translating sphere's flow) and the double layer of a constant (Gauss: -c inside, 0
    outside) at targets 0.01 to 0.3 off the surface."""
    p = 12
    a = 2.0
    X = a * unit_sphere(p)
    ng = sh.ngrid(p)
    f = np.zeros((3, ng))
    f[0] = 1.0
    c = np.array([0.3, -1.0, 0.5])
    g = np.repeat(c[:, None], ng, axis=1).reshape(-1)
    dirs = np.random.default_rng(5).normal(size=(8, 3))
    dirs /= np.linalg.norm(dirs, axis=1)[:, None]
    T = np.concatenate([dirs * (a + d) for d in (0.01, 0.1, 0.3)] + [dirs * (a - d) for d in (0.01, 0.1, 0.3)])
    r = np.linalg.norm(T, axis=1)
    xh = T / r[:, None]
    e0 = np.array([1.0, 0.0, 0.0])
    ext = (0.5 * a * a / r)[:, None] * (e0[None] + xh[:, :1] * xh) + (a ** 4 / 6 / r ** 3)[:, None] * (
        e0[None] - 3 * xh[:, :1] * xh)
    ref_sl = np.where((r > a)[:, None], ext, (2 * a / 3) * e0[None])
    ref_dl = np.where((r > a)[:, None], 0.0, -c[None])
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f.reshape(-1))
        sv.SetTrgCoord(T)
        u0 = sv.eval_targets().reshape(-1, 3)
        sv.set_near_singular(True)
        u = sv.eval_targets().reshape(-1, 3)
        sv.SetDensitySL(np.zeros(X.size))
        sv.SetDensityDL(g)
        w = sv.eval_targets().reshape(-1, 3)
    assert np.abs(u0 - ref_sl).max() > 1e-2  # the smooth quadrature alone fails near the surface
    assert np.abs(u - ref_sl).max() < 1e-3
    assert np.abs(w - ref_dl).max() < 1e-4
