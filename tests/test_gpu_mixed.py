"""Mixed-precision form (packed-FP32 far field with FP64 accumulation) against the FP64
oracle; tolerance 1e-6 relative, max-norm (the accuracy target of the mixed form)."""
import numpy as np
import pytest

from oracle import sh, stokes
from tests.helpers import rel_err, small_suspension
from ves3d_b200.stokes_velocity import StokesVelocity

pytestmark = pytest.mark.gpu
MIXED_TOL = 1e-6


@pytest.mark.parametrize("nside,p,seed", [(2, 6, 21), (2, 12, 22), (2, 12, 31), (3, 8, 34)])
def test_mixed_vs_oracle(nside, p, seed):
    X, f = small_suspension(nside, p, seed)
    with StokesVelocity(p, precision="mixed") as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        vel = sv()
        _, far = sv.parts()
    ref_far = stokes.far_velocity(X, f, p)
    ref = sh.self_apply(sh.stokes_singular_matrix(X, p, 2 * p), f, p) + ref_far
    assert rel_err(far, ref_far) < MIXED_TOL
    assert rel_err(vel, ref) < MIXED_TOL


def test_mixed_vs_fp64_full_c2():
    """Full 512-vesicle p=16 suspension: mixed against the FP64 GPU path (itself checked
    against the oracle to 1e-12), far part and total."""
    from ves3d_b200 import workloads
    X, f, p = workloads.make("c2_512ves_p16")
    out = {}
    for prec in ("fp64", "mixed"):
        with StokesVelocity(p, precision=prec) as sv:
            sv.SetSrcCoord(X)
            sv.SetDensitySL(f)
            v = sv()
            out[prec] = (v, sv.parts()[1])
    assert rel_err(out["mixed"][1], out["fp64"][1]) < MIXED_TOL
    assert rel_err(out["mixed"][0], out["fp64"][0]) < MIXED_TOL


def test_far_targets_in_chunks_p24():
    """p=24 vesicles (1,200 points) run as two target chunks per vesicle."""
    X, f = small_suspension(1, 24, 23)
    X2 = np.concatenate([X, X.reshape(3, -1).__add__(np.array([[2.7], [0.2], [0.1]])).reshape(-1)])
    f2 = np.concatenate([f, -0.5 * f])
    p = 24
    ref_far = stokes.far_velocity(X2, f2, p)
    for prec, tol in (("fp64", 1e-12), ("mixed", MIXED_TOL)):
        with StokesVelocity(p, precision=prec) as sv:
            sv.SetSrcCoord(X2)
            sv.SetDensitySL(f2)
            sv()
            _, far = sv.parts()
        assert rel_err(far, ref_far) < tol, prec


def test_mixed_deterministic():
    X, f = small_suspension(2, 6, 24)
    with StokesVelocity(6, precision="mixed") as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        a = sv()
        b = sv()
    assert np.array_equal(a, b)


def test_tensor_core_build_vs_fp64_and_oracle():
    """The mixed form builds its p = 16 self matrices with the DFT GEMMs on the tcgen05
    tensor cores (split-BF16, FP32 accumulation): self matrices against the FP64 build,
    velocity against the FP64 oracle, both within the mixed form's 1e-6."""
    p = 16
    X, f = small_suspension(2, p, 61)
    with StokesVelocity(p, precision="fp64") as sv:
        sv.SetSrcCoord(X)
        SL64 = sv.self_matrix()
    with StokesVelocity(p, precision="mixed") as sv:
        sv.SetSrcCoord(X)
        SLm = sv.self_matrix()
        sv.SetDensitySL(f)
        vel = sv()
        vself, _ = sv.parts()
    ref_self = sh.self_apply(sh.stokes_singular_matrix(X, p, 2 * p), f, p)
    ref = ref_self + stokes.far_velocity(X, f, p)
    assert 0 < rel_err(SLm, SL64) < MIXED_TOL  # a different build, within the bar
    assert rel_err(vself, ref_self) < MIXED_TOL
    assert rel_err(vel, ref) < MIXED_TOL


def test_tensor_core_build_is_deterministic_and_matches_fp64_ring_env(monkeypatch):
    """Two tensor-core builds give the same bits; VES3D_TC_BUILD=0 falls back to the FP64
    ring in the mixed form (the A/B switch)."""
    p = 16
    X, _ = small_suspension(1, p, 62)
    with StokesVelocity(p, precision="mixed") as sv:
        sv.SetSrcCoord(X)
        a = sv.self_matrix()
        sv.SetSrcCoord(X)
        b = sv.self_matrix()
    assert np.array_equal(a, b)
    monkeypatch.setenv("VES3D_TC_BUILD", "0")
    with StokesVelocity(p, precision="mixed") as sv:
        sv.SetSrcCoord(X)
        c = sv.self_matrix()
    with StokesVelocity(p, precision="fp64") as sv:
        sv.SetSrcCoord(X)
        d = sv.self_matrix()
    assert np.array_equal(c, d)


@pytest.mark.parametrize("p", [12, 24])
def test_fp32_build_stages_after_the_fp64_ring(p, monkeypatch):
    """At p = 12 and 24 the mixed form rotates the FP64 ring's results back and takes them to
    coefficients in FP32: self matrices within 1e-6 of the FP64 build (and not its bits);
    VES3D_TC_BUILD=0 keeps the FP64 stages (bitwise the FP64 build)."""
    X, _ = small_suspension(1, p, 63)
    with StokesVelocity(p, precision="fp64") as sv:
        sv.SetSrcCoord(X)
        d = sv.self_matrix()
    with StokesVelocity(p, precision="mixed") as sv:
        sv.SetSrcCoord(X)
        m = sv.self_matrix()
    assert 0 < rel_err(m, d) < MIXED_TOL
    monkeypatch.setenv("VES3D_TC_BUILD", "0")
    with StokesVelocity(p, precision="mixed") as sv:
        sv.SetSrcCoord(X)
        c = sv.self_matrix()
    assert np.array_equal(c, d)


@pytest.mark.parametrize("p", [12, 16])
def test_implicit_steps_take_fp64_self_matrices(p):
    """Self matrices from the mixed form's FP32 build stages (the tensor-core build at p = 16,
    the FP32 stages after the FP64 ring at p = 12) are rebuilt in FP64 once the context takes
    implicit steps: the mixed refinement's outer residuals are those of the FP64 system."""
    X, _ = small_suspension(1, p, 64)
    with StokesVelocity(p, precision="fp64") as sv:
        sv.SetSrcCoord(X)
        d = sv.self_matrix()
    with StokesVelocity(p, precision="mixed") as sv:
        sv.SetSrcCoord(X)
        m = sv.self_matrix()
        sv.set_implicit_params(0.01, 0.05, 1.0)
        after = sv.self_matrix()
    assert not np.array_equal(m, d)
    assert np.array_equal(after, d)
