"""Order p = 24 (a quarter of the polydisperse 4,096-vesicle suspension) and the full
512-vesicle p = 16 suspension against the oracle. At p = 24 the self-matrix build runs the
fused ring with one CTA per SM (its tables fill the shared memory) and the CUDA-core form
of the rotate-transpose, which the smaller orders do not reach; the stage-by-stage build
(VES3D_FUSED_BUILD=0) is checked at p = 24 too.
Tolerances: 1e-12 relative max-norm for FP64 against the oracle, 1e-6 for the mixed
form, 5e-9 against the reference's own output (its self-part noise floor)."""
import os

import numpy as np
import pytest

from oracle import sh, stokes
from tests.helpers import ellipsoid_pair, rel_err
from ves3d_b200 import workloads
from ves3d_b200.stokes_velocity import PolydisperseStokesVelocity, StokesVelocity

pytestmark = pytest.mark.gpu
TOL = 1e-12
MIXED_TOL = 1e-6
REF_SELF_NOISE = 5e-9
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_noise_floor_p12_p24.npz")


def test_p24_self_matrix_matches_oracle():
    p = 24
    X = ellipsoid_pair(p)
    with StokesVelocity(p, 2 * p) as sv:
        sv.SetSrcCoord(X)
        SL = sv.self_matrix()
    assert rel_err(SL, sh.stokes_singular_matrix(X, p, 2 * p)) < TOL


def test_p24_stage_by_stage_build_matches_oracle(monkeypatch):
    monkeypatch.setenv("VES3D_FUSED_BUILD", "0")
    p = 24
    X = ellipsoid_pair(p)[: 3 * sh.ngrid(p)]
    with StokesVelocity(p, 2 * p) as sv:
        sv.SetSrcCoord(X)
        SL = sv.self_matrix()
    assert rel_err(SL, sh.stokes_singular_matrix(X, p, 2 * p)) < TOL


def test_p24_self_velocity_matches_reference_golden():
    """The reference's own p = 24 self velocity (two builds of it, tests/golden)."""
    g = dict(np.load(GOLDEN))
    X, f = g["p24_X"], g["p24_f"]
    with StokesVelocity(24, 48) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        vel = sv()
        vself, _ = sv.parts()
    assert rel_err(vself, sh.self_apply(sh.stokes_singular_matrix(X, 24, 48), f, 24)) < TOL
    assert rel_err(vself, g["p24_vel_self"]) < REF_SELF_NOISE
    assert rel_err(vself, g["p24_vel_self_naive"]) < REF_SELF_NOISE
    assert rel_err(vel, vself) == 0.0  # one vesicle: no far part


@pytest.mark.parametrize("prec,tol", [("fp64", TOL), ("mixed", MIXED_TOL)])
def test_p24_velocity_matches_oracle(prec, tol):
    p = 24
    X = ellipsoid_pair(p)
    f = np.random.default_rng(240).standard_normal(X.size)
    ref = stokes.stokes_velocity_sl(X, f, p, 2 * p)
    with StokesVelocity(p, 2 * p, precision=prec) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        vel = sv()
    assert rel_err(vel, ref) < tol


@pytest.mark.parametrize("prec,tol", [("fp64", TOL), ("mixed", MIXED_TOL)])
def test_polydisperse_with_p24_matches_oracle(prec, tol):
    """All four orders of the polydisperse configuration, p = 24 included."""
    X, f, orders = workloads.polydisperse(8, orders=(8, 12, 16, 24), radius=(0.7, 1.3), volume_fraction=0.05,
                                          seed=2402)
    assert set(orders.tolist()) == {8, 12, 16, 24}
    ref = stokes.stokes_velocity_poly(X, f, orders)
    with PolydisperseStokesVelocity(prec) as sv:
        sv.SetSrcCoord(X, orders)
        sv.SetDensitySL(f)
        vel = sv()
    assert rel_err(vel, ref) < tol


@pytest.fixture(scope="module")
def c2_fp64():
    """The full 512-vesicle p = 16 suspension, FP64 and mixed, on the GPU."""
    X, f, p = workloads.make("c2_512ves_p16")
    out = {}
    for prec in ("fp64", "mixed"):
        with StokesVelocity(p, precision=prec) as sv:
            sv.SetSrcCoord(X)
            sv.SetDensitySL(f)
            out[prec] = sv()
    return X, f, p, out


def test_c2_whole_vesicles_match_oracle(c2_fp64):
    """Every point of three whole vesicles of the full suspension against the oracle
    (self part from the oracle's self matrix, far part over all 278,528 sources): FP64 at
    1e-12, the mixed form at 1e-6; relative to the max-norm of the whole velocity."""
    X, f, p, out = c2_fp64
    ng = sh.ngrid(p)
    nves = X.size // (3 * ng)
    D = stokes.far_density(X, f, p)
    off = stokes.uniform_offsets(nves, p)
    scale = {k: np.abs(v).max() for k, v in out.items()}
    for v in (0, 257, nves - 1):
        a, b = 3 * ng * v, 3 * ng * (v + 1)
        self_v = sh.self_apply(sh.stokes_singular_matrix(X[a:b], p, 2 * p), f[a:b], p)
        far_v = stokes.far(X, D, off, np.arange(v * ng, (v + 1) * ng)).T.reshape(-1)
        ref = self_v + far_v
        for prec, tol in (("fp64", TOL), ("mixed", MIXED_TOL)):
            err = np.abs(out[prec][a:b] - ref).max() / scale[prec]
            assert err < tol, (prec, v, err)
