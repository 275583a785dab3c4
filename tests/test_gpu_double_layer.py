"""GPU parity of the double layer (SetDensityDL) against the CPU oracle, whose DL matrices
and DL kernel are pinned to the reference's own (test_oracle_pin.py): the DL self matrices,
the direct DL sums of Device<GPU>::DirectStokesDoubleLayer, the operator's single + double
layer evaluation and its parts, the CUDA graph, and Gauss's identity at size.
Tolerance for the FP64 form: 1e-12 relative, max-norm."""
import numpy as np
import pytest

from oracle import sh, stokes
from tests.helpers import ellipsoid_pair, rel_err, small_suspension
from ves3d_b200 import _lib, workloads
from ves3d_b200.stokes_velocity import StokesVelocity

pytestmark = pytest.mark.gpu
TOL = 1e-12


def test_dl_matrix_matches_oracle():
    p = 6
    X = ellipsoid_pair(p)
    g = np.random.default_rng(6).standard_normal(X.size)
    with StokesVelocity(p, 2 * p) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensityDL(g)
        DL = sv.dl_matrix()
    assert rel_err(DL, sh.stokes_singular_matrix(X, p, 2 * p, single=False)) < TOL


@pytest.mark.parametrize("nside,p,seed", [(1, 6, 1), (2, 6, 2), (2, 12, 3)])
def test_single_and_double_layer_match_oracle(nside, p, seed):
    X, f = small_suspension(nside, p, seed)
    g = np.random.default_rng(seed + 100).standard_normal(X.size)
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        sv.SetDensityDL(g)
        vel = sv()
        vself, vfar = sv.parts()
    assert rel_err(vel, stokes.stokes_velocity_sl(X, f, p) + stokes.stokes_velocity_dl(X, g, p)) < TOL
    if nside > 1:  # one vesicle has no far part
        far = stokes.far_velocity(X, f, p) + stokes.far_dl_velocity(X, g, p)
        assert rel_err(vfar, far) < TOL
        assert rel_err(vself + vfar, vel) < 1e-14


@pytest.mark.parametrize("nside,p,seed", [(2, 8, 5), (2, 16, 3)])
def test_mixed_double_layer_matches_oracle(nside, p, seed, monkeypatch):
    """Mixed form with the far double layer in FP32 pair arithmetic (k_far_dl_f32_flat,
    opt-in: VES3D_FAR_DL_F32=1, read when the context is created). The double layer alone,
    then single + double layer, the evaluation and its far part within 1e-6 (relative,
    max-norm) of the FP64 oracle."""
    monkeypatch.setenv("VES3D_FAR_DL_F32", "1")
    X, f = small_suspension(nside, p, seed)
    g = np.random.default_rng(seed + 100).standard_normal(X.size)
    with StokesVelocity(p, precision="mixed") as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(np.zeros_like(X))
        sv.SetDensityDL(g)
        sv()
        _, vfar_dl = sv.parts()
        sv.SetDensitySL(f)
        vel = sv()
        _, vfar = sv.parts()
    assert rel_err(vfar_dl, stokes.far_dl_velocity(X, g, p)) < 1e-6
    assert rel_err(vel, stokes.stokes_velocity_sl(X, f, p) + stokes.stokes_velocity_dl(X, g, p)) < 1e-6
    assert rel_err(vfar, stokes.far_velocity(X, f, p) + stokes.far_dl_velocity(X, g, p)) < 1e-6


def test_double_layer_on_and_off():
    """Turning the double layer off returns the single-layer evaluation; the difference
    while it is on is the double-layer velocity; new surfaces clear the density."""
    p = 6
    X, f = small_suspension(2, p, 4)
    g = np.random.default_rng(9).standard_normal(X.size)
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        v0 = sv()
        sv.SetDensityDL(g)
        v1 = sv()
        sv.SetDensityDL(None)
        v2 = sv()
        sv.SetDensityDL(g)
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        v3 = sv()
    assert rel_err(v2, v0) < 1e-14 and rel_err(v3, v0) < 1e-14
    assert rel_err(v1 - v0, stokes.stokes_velocity_dl(X, g, p)) < 1e-11


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_double_layer_in_the_captured_evaluation(precision):
    """The CUDA graph of the evaluation records the double layer: relaunched on new
    double-layer densities it gives bitwise the eager evaluation."""
    import torch
    p = 8
    X, f = small_suspension(2, p, 71, spacing=2.7)
    rng = np.random.default_rng(5)
    with StokesVelocity(p, precision=precision) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        sv.SetDensityDL(rng.standard_normal(X.size))
        sv.capture_eval()
        for _ in range(2):
            sv.SetDensityDL(torch.from_numpy(rng.standard_normal(X.size)).cuda())
            sv.launch_eval_graph()
            torch.cuda.synchronize()
            self_g, far_g = sv.parts()
            sv()
            self_e, far_e = sv.parts()
            assert np.array_equal(self_g, self_e) and np.array_equal(far_g, far_e)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_double_layer_of_constant_densities_at_size(precision):
    """Gauss's identity on 64 vesicles of p = 12: a constant double-layer density c_v on each
    vesicle gives -c_v / 2 on its surface and nothing on the others (the oracle measures
    4.2e-6 on this suspension); the far double layer is FP64 in both forms (FP32 pairs only
    on request)."""
    p = 12
    X, _ = workloads.suspension(4, p, 3.0, semi_axes=(1.0, 1.0, 0.6), deg=4, amp=0.05, seed=8)
    ng = sh.ngrid(p)
    nv = X.size // (3 * ng)
    C = np.random.default_rng(2).standard_normal((nv, 3))
    g = np.repeat(C[:, :, None], ng, axis=2).reshape(-1)
    with StokesVelocity(p, precision=precision) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(np.zeros_like(X))
        sv.SetDensityDL(g)
        u = sv().reshape(nv, 3, ng)
    assert np.abs(u + 0.5 * C[:, :, None]).max() < 2e-5


@pytest.mark.parametrize("weighted", [True, False])
def test_direct_stokes_double_layer_matches_oracle(weighted):
    """ves3d_cuda_stokes_double_layer_f64 (cuda_stokes_double_layer) against the oracle's
    DirectStokesDoubleLayerKernel, a coincident pair included."""
    import torch
    rng = np.random.default_rng(12)
    ns, nt, nv, head, tail = 100, 70, 3, 5, 60
    S = rng.standard_normal(3 * ns * nv)
    T = rng.standard_normal(3 * nt * nv)
    T[head], T[nt + head], T[2 * nt + head] = S[0], S[ns], S[2 * ns]
    N = rng.standard_normal(3 * ns * nv)
    D = rng.standard_normal(3 * ns * nv)
    Q = rng.uniform(0.5, 1.5, ns) if weighted else None
    d = {k: torch.from_numpy(v).cuda() for k, v in dict(S=S, T=T, N=N, D=D).items()}
    U = torch.zeros(3 * nt * nv, dtype=torch.float64, device="cuda")
    dq = torch.from_numpy(Q).cuda() if weighted else None
    _lib.check(_lib.lib().ves3d_cuda_stokes_double_layer_f64(
        ns, nt, nv, head, tail, d["T"].data_ptr(), d["S"].data_ptr(), d["N"].data_ptr(), d["D"].data_ptr(),
        U.data_ptr(), dq.data_ptr() if weighted else None, None), "cuda_stokes_double_layer")
    torch.cuda.synchronize()
    ref = stokes.direct_stokes_dl(ns, nt, nv, head, tail, Q, T, S, N, D)
    assert rel_err(U.cpu().numpy(), ref) < TOL


def test_double_layer_against_the_reference_fixture():
    """The GPU double layer against the reference's own outputs (tests/golden/
    ref_p6_double_layer.npz): the DL self matrix and self velocity within the reference's
    self-part noise (5e-9), the far double layer at 1e-12."""
    import os
    gdl = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_p6_double_layer.npz")))
    p = int(gdl["p"])
    n = 3 * p * (p + 2)
    with StokesVelocity(p, 2 * p) as sv:
        sv.SetSrcCoord(gdl["X"])
        sv.SetDensitySL(np.zeros_like(gdl["X"]))
        sv.SetDensityDL(gdl["g"])
        DL = sv.dl_matrix()
        vel = sv()
        vself, _ = sv.parts()
    assert rel_err(DL[0].reshape(-1), gdl["DL0"]) < 5e-9
    assert rel_err(vself, gdl["vel_self"]) < 5e-9  # the single-layer density is zero
    with StokesVelocity(p, 2 * p) as sv:
        sv.SetSrcCoord(gdl["Xs"])
        sv.SetDensitySL(np.zeros_like(gdl["Xs"]))
        sv.SetDensityDL(gdl["gs"])
        sv()
        _, vfar = sv.parts()
    assert rel_err(vfar, gdl["far_dl"]) < TOL
    assert n == DL.shape[1] and vel.size == gdl["X"].size


def test_monitor_error_lowers_the_order_on_a_sphere():
    """MonitorError on one sphere: the double layer of density 1 is -1/2 to rounding, so the
    self order drops by 2 (error below tol/2); the single-layer density set before survives,
    and the operator at the new order matches the oracle at that order."""
    from tests.helpers import unit_sphere
    p = 12
    X = unit_sphere(p)
    f = np.random.default_rng(3).standard_normal(X.size)
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        v0 = sv()
        total, err = sv.MonitorError(1e-6)
        assert err[0] < 1e-10 and err[1] == 0.0 and err[2] == 0.0 and total == err[0]
        assert sv.sh_order_up == 2 * p - 2
        v1 = sv()
    assert rel_err(v0, stokes.stokes_velocity_sl(X, f, p, 2 * p)) < TOL
    assert rel_err(v1, stokes.stokes_velocity_sl(X, f, p, 2 * p - 2)) < TOL


def test_monitor_error_raises_the_order_above_tol():
    """On eight non-spherical vesicles at p = 8 the self error exceeds a tiny tol, so the
    order rises by 2; the far part of constant densities vanishes to the quadrature error."""
    p = 8
    X, _ = small_suspension(2, p, 3)
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        total, err = sv.MonitorError(1e-14)
        assert sv.sh_order_up == 2 * p + 2
        assert err[0] > 1e-14 and err[2] < 5e-3 and abs(total - err[0] - err[2]) < 1e-15
