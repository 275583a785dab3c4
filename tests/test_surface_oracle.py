"""CPU checks of the geometry / force / BiCGStab oracle (oracle/surface.py): analytic
identities, and the reference's own BiCGStab class (oracle/_ref)."""
import ctypes

import numpy as np
import pytest

from oracle import sh, surface as su
from tests.helpers import ellipsoid_pair, unit_sphere


@pytest.mark.parametrize("p", [8, 12])
def test_sphere_curvatures(p):
    g = su.geometry(2.0 * unit_sphere(p), p)
    # the reference's conventions: outward normal, H = -1/R on a sphere
    assert np.abs(g["H"] + 0.5).max() < 1e-12
    assert np.abs(g["K"] - 0.25).max() < 1e-12
    X = (2.0 * unit_sphere(p)).reshape(1, 3, -1)
    assert np.abs((g["n"] * X).sum(1) - 2.0).max() < 1e-12


def test_surface_divergence_of_position_is_two():
    p = 12
    g = su.geometry(ellipsoid_pair(p), p)
    assert np.abs(su.div(g["X"], g) - 2.0).max() < 1e-11


def test_laplace_beltrami_eigenvalue_on_sphere():
    p = 12
    g = su.geometry(unit_sphere(p), p)
    P = g["X"][0]
    f = (P[0] * P[1] * P[2])[None]  # degree 3: eigenvalue -12
    lap = su.div(su.grad(f, g), g)
    assert np.abs(lap + 12.0 * f).max() < 1e-11
    assert np.abs((su.grad(f, g) * g["n"]).sum(1)).max() < 1e-14


def test_gauss_bonnet():
    p = 16
    g = su.geometry(ellipsoid_pair(p), p)
    x = sh.legendre_nodes(p)
    w = sh.gauss_legendre(p + 1)[1]
    qw = np.repeat(w * np.pi / p / np.sqrt(1 - x * x), 2 * p)
    gb = (g["K"] * g["W"] * qw).sum(axis=1) / (4 * np.pi)
    assert np.abs(gb - 1.0).max() < 1e-5


def test_sphere_has_no_bending_force():
    p = 12
    g = su.geometry(unit_sphere(p), p)
    assert np.abs(su.bending_force(g, 0.1)).max() < 1e-10


def test_bicgstab_matches_reference_class(ref):
    L = ref.lib()
    L.ref_bicgstab_dense.restype = ctypes.c_int
    dp = ctypes.POINTER(ctypes.c_double)
    rng = np.random.default_rng(0)
    for n, tol in ((60, 1e-10), (120, 1e-8)):
        A = np.eye(n) * 3 + rng.standard_normal((n, n)) * (2.0 / np.sqrt(n))
        b = rng.standard_normal(n)
        x = np.zeros(n)
        t = ctypes.c_double(tol)
        it = ctypes.c_int(300)
        code = L.ref_bicgstab_dense(A.ctypes.data_as(dp), b.ctypes.data_as(dp), x.ctypes.data_as(dp),
                                    ctypes.c_long(n), ctypes.byref(t), ctypes.byref(it))
        xo, c2, i2, r2 = su.bicgstab(lambda v: A @ v, b, np.zeros(n), tol, 300)
        assert code == c2 == 100 and it.value == i2
        assert abs(r2 - t.value) <= 1e-3 * t.value  # residual of an iterate that rounds differently
        assert np.abs(x - xo).max() < 1e-12


def test_integrals_dumbbell_known_answers():
    """SurfaceTest's dumbbell (test/SurfaceTest.cc:72, :79): area 16.2179377312307 and
    volume 5.24886489292959 to 5e-8 relative; the reference compares magnitudes."""
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_dumbbell_p6.npz"))
    area, vol, cen = su.integrals(d["X"], int(d["p"]))
    assert abs(area[0] / float(d["area"]) - 1) < float(d["rtol"])
    assert abs(vol[0] / float(d["volume"]) - 1) < float(d["rtol"])
    assert np.abs(cen).max() < 1e-8


def test_dumbbell_curvature_and_operators_known_answers():
    """SurfaceTest's dumbbell (test/SurfaceTest.cc:86-151), reproduced with the reference's
    low-pass filter at 2p/3: max |H| (8e-8); max |grad x_i| and max |Lap x_i| for the three
    coordinate fields (1e-7); max |Lap X . n| (1e-7); max |H - Lap X . n / 2| and
    max |H + div n / 2| (1e-6; both fix the sign of H against the normal); the linearised
    curvature of the position is H (1e-14)."""
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_dumbbell_p6.npz"))
    p = int(d["p"])
    X = d["X"].reshape(1, 3, -1)
    geo = su.geometry(X, p, filter_freq=2 * p // 3)
    rel = lambda a, ref: abs(np.abs(a).max() / float(ref) - 1)
    assert rel(geo["H"], d["max_abs_H"]) < float(d["rtol_H"])
    lap = []
    for c in range(3):
        g = su.grad(X[:, c], geo)
        lap.append(su.div(g, geo))
        assert rel(g, d["max_abs_grad"][c]) < float(d["rtol_grad"])
        assert rel(lap[-1], d["max_abs_lap"][c]) < float(d["rtol_grad"])
    lap_dot_n = (np.stack(lap, 1) * geo["n"]).sum(1)
    assert rel(lap_dot_n, d["max_abs_lap_dot_n"]) < float(d["rtol_grad"])
    assert rel(geo["H"] - 0.5 * lap_dot_n, d["max_abs_H_minus_half_lap_dot_n"]) < float(d["rtol_mixed"])
    assert rel(geo["H"] + 0.5 * su.div(geo["n"], geo), d["max_abs_H_plus_half_div_n"]) < float(d["rtol_mixed"])
    assert np.abs(su.lin_mean_curv(X, geo) - geo["H"]).max() < 1e-14
    # without the filter (the GPU path's choice) the same operators differ only by the
    # filtered-out high degrees
    geo0 = su.geometry(X, p)
    assert rel(geo0["H"], d["max_abs_H"]) < 0.2


def test_integrals_sphere_and_translation():
    from ves3d_b200 import workloads
    p, R = 12, 1.7
    X = R * workloads.shape(p, np.zeros(3), deg=0).reshape(-1)
    area, vol, cen = su.integrals(X, p)
    assert abs(area[0] / (4 * np.pi * R * R) - 1) < 1e-12
    assert abs(vol[0] / (4 / 3 * np.pi * R ** 3) - 1) < 1e-12
    shift = np.array([0.5, -2.0, 1.25])
    Xs = (X.reshape(3, -1) + shift[:, None]).reshape(-1)
    a2, v2, c2 = su.integrals(Xs, p)
    assert abs(a2[0] - area[0]) < 1e-12 * area[0] and abs(v2[0] - vol[0]) < 1e-12 * abs(vol[0])
    assert np.abs(c2[0] - cen[0] - shift).max() < 1e-12


def test_poly_implicit_step_single_order_is_uniform():
    """The oracle's polydisperse implicit step with one order is ImplicitStep exactly, and
    with two orders its operator is linear and its coefficient maps invert each other."""
    from tests.helpers import small_suspension
    from ves3d_b200 import workloads
    X, _ = small_suspension(2, 6, 61, spacing=2.7)
    nv = X.size // (3 * 2 * 6 * 7)
    P = su.PolyImplicitStep(X, [6] * nv, 0.05, 0.01, 1.0, excess_density=1.0)
    S = su.ImplicitStep(X, 6, 0.05, 0.01, 1.0, excess_density=1.0)
    z = np.random.default_rng(1).standard_normal(4 * X.size // 3)
    assert np.abs(P.matvec(z) - S.matvec(z)).max() == 0.0
    assert np.abs(P.rhs() - S.rhs()).max() == 0.0
    X2, _, orders = workloads.polydisperse(3, orders=(4, 6), radius=(0.8, 1.2), volume_fraction=0.05, seed=5)
    Q = su.PolyImplicitStep(X2, orders, 0.05, 0.01, 0.0, excess_density=1.0)
    rng = np.random.default_rng(2)
    a, b = rng.standard_normal((2, 4 * X2.size // 3))
    assert np.abs(Q.matvec(2 * a - b) - (2 * Q.matvec(a) - Q.matvec(b))).max() < 1e-12 * np.abs(Q.matvec(a)).max()
    c = Q.to_coef(a)
    assert np.abs(Q.to_coef(Q.to_grid(c)) - c).max() < 1e-12


def test_relaxing_vesicle_loses_bending_energy():
    """The bending traction is restoring (the reference's bending_coeff = -bending_modulus,
    src/VesicleProps.cc:39-41): implicit steps of a free, perturbed ellipsoid lower its
    bending energy every step and keep its area and volume (local inextensibility)."""
    from ves3d_b200 import workloads
    p, dt = 8, 0.01
    X = workloads.shape(p, np.zeros(3), semi_axes=(1.0, 1.0, 0.6), deg=4, amp=0.05,
                        rng=np.random.default_rng(1)).reshape(-1)
    qw = sh.smooth_weights_grid(p)
    E, A, V = [], [], []
    for _ in range(3):
        st = su.ImplicitStep(X, p, 0.05, dt, 0.0)
        x, code, it, rr = st.solve(tol=1e-10, max_iter=500)
        assert code == 100
        g = st.geo
        E.append((g["H"] ** 2 * g["W"] * qw).sum())
        a, v, _ = su.integrals(X, p)
        A.append(a[0])
        V.append(v[0])
        X = X + dt * x[:X.size]
    assert E[0] > E[1] > E[2]
    assert abs(A[-1] / A[0] - 1) < 1e-5 and abs(V[-1] / V[0] - 1) < 1e-5


def test_low_pass_filters():
    """SHTrans's filters (oracle restatement): the hard cut keeps exactly the degrees up to
    the cut and is idempotent; the polynomial filter weights degree n by 1 - (n/f)^e and
    removes degrees >= f; both act per coefficient (ScaleFreq)."""
    p = 12
    rng = np.random.default_rng(4)
    X = rng.standard_normal(3 * 2 * p * (p + 1))
    hard = sh.low_pass(X, p)
    assert np.abs(sh.low_pass(hard, p) - hard).max() < 1e-13
    S = sh.grid2shc(hard, p, p).reshape(3, -1)
    off = sh.block_offsets(p)
    deg = np.concatenate([(jf + 1) // 2 + np.arange(off[jf + 1] - off[jf]) for jf in range(2 * p)])
    assert np.abs(S[:, deg > 2 * p // 3]).max() < 1e-13
    S0 = sh.grid2shc(X, p, p).reshape(3, -1)
    assert np.abs(S[:, deg <= 2 * p // 3] - S0[:, deg <= 2 * p // 3]).max() < 1e-13
    c = sh.filter_coeffs(p, 6, 4.0)
    assert np.allclose(c[deg < 6], 1 - (deg[deg < 6] / 6.0) ** 4) and np.all(c[deg >= 6] == 0)
    Sp = sh.grid2shc(sh.low_pass(X, p, 6, 4.0), p, p).reshape(3, -1)
    assert np.abs(Sp - S0 * c[None, :]).max() < 1e-12


def test_poly_sedimentation_solve_sinks():
    """The oracle's polydisperse implicit step under gravity (-z, excess density 1): BiCGStab
    meets the tolerance and the suspension sinks; without gravity and flow nothing moves
    but the relaxation of the shapes."""
    from ves3d_b200 import workloads
    X, _, orders = workloads.polydisperse(3, orders=(4, 6), radius=(0.8, 1.2), volume_fraction=0.05, seed=8)
    step = su.PolyImplicitStep(X, orders, 0.05, 0.01, 0.0, excess_density=1.0)
    x, code, it, rr = step.solve(tol=1e-9, max_iter=600)
    assert code == 100 and rr < 1e-9
    us, _ = step.split(x)
    uz = np.concatenate([u[:, 2].reshape(-1) for u in us])
    assert uz.mean() < 0
    rest = su.PolyImplicitStep(X, orders, 0.05, 0.01, 0.0)
    x0, code0, _, _ = rest.solve(tol=1e-9, max_iter=600)
    u0, _ = rest.split(x0)
    assert code0 == 100
    assert np.abs(np.concatenate([u[:, 2].reshape(-1) for u in u0]).mean()) < 0.1 * abs(uz.mean())


def test_viscosity_contrast_of_one_is_no_contrast():
    from tests.helpers import small_suspension
    p = 8
    X, _ = small_suspension(2, p, 3)
    A = su.ImplicitStep(X, p, 0.05, 0.01, 1.0)
    B = su.ImplicitStep(X, p, 0.05, 0.01, 1.0, SL=A.SL, viscosity_contrast=1.0)
    z = np.random.default_rng(1).standard_normal(4 * A.nv * A.ng)
    assert not B.contrast and np.array_equal(A.matvec(z), B.matvec(z))


def test_viscosity_contrast_keeps_rigid_translations():
    """(1 + l)/2 c - S[f(dt c, 0)] - D[(1 - l) c] = c and -div(...) = 0 for a constant
    velocity c per vesicle, whatever the contrast l: the linearised bending of a rigid
    displacement vanishes and D[c] = -c/2 on a closed surface. Exact up to the double layer's
    quadrature error (3.5e-5 at p = 12 with l from 0.1 to 5)."""
    from tests.helpers import small_suspension
    p = 12
    X, _ = small_suspension(2, p, 3)
    lam = np.array([3.0, 0.2, 1.0, 5.0, 0.5, 2.0, 1.0, 0.1])
    step = su.ImplicitStep(X, p, 0.05, 0.01, 1.0, viscosity_contrast=lam)
    C = np.random.default_rng(1).standard_normal((step.nv, 3))
    z = np.concatenate([np.repeat(C[:, :, None], step.ng, axis=2).reshape(-1), np.zeros(step.nv * step.ng)])
    assert step.contrast
    assert np.abs(step.matvec(z) - z).max() < 1e-4 * np.abs(C).max()


def test_viscosity_contrast_solve_converges():
    """The contrast step solves by the same BiCGStab; a more viscous interior (l = 4) deforms
    the vesicle less in shear than l = 1 (velocity minus its mean: 4.80 against 5.95 here,
    7.02 at l = 0.25, 4.49 at l = 10)."""
    from tests.helpers import small_suspension
    p = 8
    X, _ = small_suspension(1, p, 5)
    A = su.ImplicitStep(X, p, 0.05, 0.01, 1.0)
    B = su.ImplicitStep(X, p, 0.05, 0.01, 1.0, SL=A.SL, viscosity_contrast=4.0)
    xa, code_a, _, rr_a = A.solve(tol=1e-10, max_iter=400)
    xb, code_b, _, rr_b = B.solve(tol=1e-10, max_iter=400)
    assert code_a == code_b == 100 and rr_a < 1e-9 and rr_b < 1e-9  # 100: converged (BiCGStab.cc)
    nu = A.nv * 3 * A.ng
    ua, ub = xa[:nu].reshape(A.nv, 3, A.ng), xb[:nu].reshape(A.nv, 3, A.ng)
    # the deformation part (velocity minus its mean) is damped by the interior viscosity
    da = ua - ua.mean(axis=2, keepdims=True)
    db = ub - ub.mean(axis=2, keepdims=True)
    assert np.linalg.norm(db) < np.linalg.norm(da)
