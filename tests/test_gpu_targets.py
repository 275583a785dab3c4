"""GPU velocity at off-surface targets (SetTrgCoord / ves3d_sv_eval_trg) against the oracle's
smooth quadrature (oracle/stokes.py target_velocity, built on the reference's direct kernels)
at 1e-12, and the sphere identities: the single layer of a uniform density is (2/3) a f
inside, the translating sphere's flow outside; the double layer of a constant c is -c
inside and 0 outside."""
import numpy as np
import pytest

from oracle import sh, stokes
from tests.helpers import rel_err, small_suspension, unit_sphere
from ves3d_b200._lib import Ves3dError
from ves3d_b200.stokes_velocity import StokesVelocity

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("with_dl", [False, True])
def test_targets_match_oracle(with_dl):
    p = 8
    X, f = small_suspension(2, p, 21)
    rng = np.random.default_rng(22)
    g = rng.standard_normal(X.size) if with_dl else None
    T = rng.uniform(-3.0, 6.0, (50, 3))
    ng = sh.ngrid(p)
    T[0] = X.reshape(-1, 3, ng)[1, :, 7]  # a target on a surface point: that pair counts nothing
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        if with_dl:
            sv.SetDensityDL(g)
        sv.SetTrgCoord(T)
        u = sv.eval_targets()
        v = sv()  # the surface evaluation is unaffected by the targets
        sv.SetTrgCoord(None)
        with pytest.raises(Ves3dError):
            sv.eval_targets(np.empty(3))
    assert rel_err(u, stokes.target_velocity(X, f, p, T, g)) < TOL
    ref_v = stokes.stokes_velocity_sl(X, f, p) + (stokes.stokes_velocity_dl(X, g, p) if with_dl else 0.0)
    assert rel_err(v, ref_v) < TOL


def test_target_identities_on_a_sphere():
    p = 12
    a = 2.0
    X = a * unit_sphere(p)
    f = np.zeros((3, sh.ngrid(p)))
    f[0] = 1.0
    c = np.array([0.3, -1.0, 0.5])
    g = np.repeat(c[:, None], sh.ngrid(p), axis=1).reshape(-1)
    T = np.array([[0.0, 0.0, 0.0], [0.3, -0.2, 0.1], [5.0, 0.0, 0.0]])
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f.reshape(-1))
        sv.SetTrgCoord(T)
        u = sv.eval_targets().reshape(-1, 3)
        sv.SetDensitySL(np.zeros(X.size))
        sv.SetDensityDL(g)
        w = sv.eval_targets().reshape(-1, 3)
    assert np.abs(u[:2, 0] - 2.0 * a / 3.0).max() < 1e-12 and np.abs(u[:2, 1:]).max() < 1e-12
    assert abs(u[2, 0] - (a * a / 5.0 - a ** 4 / (3 * 125.0))) < 1e-9
    assert np.abs(w[:2] + c).max() < 1e-12 and np.abs(w[2]).max() < 1e-8
