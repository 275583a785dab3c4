"""Pin the CPU oracle (oracle/sh.py, oracle/direct.c) against the reference's own code
compiled in place (oracle/_ref) and against analytic identities. CPU only."""
import numpy as np
import pytest

from oracle import sh, stokes
from tests.helpers import ellipsoid_pair, rel_err, unit_sphere

# The reference's self part is reproducible only to ~1e-9 relative even against itself
# (OpenBLAS vs plain-loop GEMM builds of the same source, test below): its MatRotate
# forms sin(theta) = sqrt(1 - x^2) at rotated grid points that lie on a pole.
REF_SELF_NOISE = 5e-9
FAR_TOL = 1e-13
PRIM_TOL = 1e-13


@pytest.mark.parametrize("p", [6, 12, 16])
def test_quadrature_rules(ref, p):
    assert rel_err(sh.legendre_nodes(p), ref.legendre_nodes(p)) < PRIM_TOL
    assert rel_err(sh.legendre_weights(p), ref.legendre_weights(p)) < PRIM_TOL
    assert rel_err(sh.singular_weights(2 * p), ref.singular_weights(2 * p)) < PRIM_TOL


@pytest.mark.parametrize("p,p1", [(6, 6), (6, 12), (12, 12), (12, 24), (16, 32), (12, 9)])
def test_transforms(ref, p, p1):
    rng = np.random.default_rng(p * 100 + p1)
    X = rng.standard_normal(5 * sh.ngrid(p))
    assert rel_err(sh.grid2shc(X, p, p1), ref.grid2shc(X, p, p1)) < PRIM_TOL
    S = rng.standard_normal(5 * sh.ncoef(p))
    if p1 >= p:
        A = sh.shc2grid(S, p, p1, grads=True)
        B = ref.shc2grid(S, p, p1, grads=True)
        for a, b in zip(A, B):
            assert rel_err(a, b) < PRIM_TOL
    assert rel_err(sh.shc2pole(S, p), ref.shc2pole(S, p)) < PRIM_TOL


def _poly(Q):
    a, b, c = Q
    return a * b * c + 0.3 * a ** 4 - b ** 3 * c + 0.7 * c ** 2 - a + 0.2 * b * c * c * a


@pytest.mark.parametrize("p", [6, 12])
def test_rotation_exact_on_polynomials(ref, p):
    """Rotating a degree-4 polynomial restricted to the sphere must equal sampling it at
    rotated points. The oracle's rotation (stable sin(theta)) is exact to rounding; the
    reference's carries the pole noise."""
    x = sh.legendre_nodes(p)
    i = np.repeat(np.arange(p + 1), 2 * p)
    j = np.tile(np.arange(2 * p), p + 1)
    s = np.sqrt(1 - x[i] ** 2)
    P = np.stack([x[i], s * np.sin(np.pi * j / p), s * np.cos(np.pi * j / p)])
    S = sh.grid2shc(_poly(P), p, p)
    ours = sh.rotate_all(S, p, 1).reshape(p + 1, p, -1)
    theirs = ref.rotate_all(S, p, 1).reshape(p + 1, p, -1)
    e_ours = e_ref = 0.0
    for t in range(p + 1):
        c_, s_ = -x[t], -np.sqrt(1 - x[t] ** 2)
        Rm = np.array([[c_, 0, -s_], [0, 1, 0], [s_, 0, c_]])
        for jj in range(p):
            ph = np.pi * jj / p
            Rz = np.array([[1, 0, 0], [0, np.cos(ph), np.sin(ph)], [0, -np.sin(ph), np.cos(ph)]])
            truth = _poly(Rz @ Rm @ P)
            e_ours = max(e_ours, np.abs(sh.shc2grid(ours[t, jj], p, p) - truth).max())
            e_ref = max(e_ref, np.abs(sh.shc2grid(theirs[t, jj], p, p) - truth).max())
    assert e_ours < 1e-13
    assert e_ref < 1e-9  # reference: exact up to its pole noise


@pytest.mark.parametrize("p", [6, 12])
def test_reference_self_noise_floor(ref, p):
    """Two builds of the reference that differ only in GEMM loop order disagree on the
    self velocity by ~1e-10..1e-9; the oracle agrees with both within that floor."""
    X = ellipsoid_pair(p)
    f = np.random.default_rng(p).standard_normal(X.size)
    A, _ = ref.singular_matrices(X, p, 2 * p)
    B = ref.naive_singular_matrices(X, p, 2 * p)
    va = ref.self_apply(A, f, p)
    vb = ref.self_apply(B, f, p)
    ours = sh.self_apply(sh.stokes_singular_matrix(X, p, 2 * p), f, p)
    floor = rel_err(va, vb)
    assert 1e-13 < floor < REF_SELF_NOISE
    assert rel_err(ours, va) < REF_SELF_NOISE
    assert rel_err(ours, vb) < REF_SELF_NOISE
    # with the reference's own sin(theta) formula the oracle sits at the same floor
    ours_u = sh.self_apply(sh.stokes_singular_matrix(X, p, 2 * p, stable=False), f, p)
    assert rel_err(ours_u, va) < REF_SELF_NOISE


@pytest.mark.parametrize("p", [6, 12])
def test_sphere_identity(ref, p):
    """Single layer on the unit sphere of f = (1,0,0) is (2/3) f (MonitorError-style
    identity used by test/StokesDoubleLayerTest.cc:120-128)."""
    X = unit_sphere(p)
    f = np.zeros((3, sh.ngrid(p)))
    f[0] = 1.0
    v = sh.self_apply(sh.stokes_singular_matrix(X, p, 2 * p), f.reshape(-1), p).reshape(3, -1)
    assert np.abs(v[0] - 2.0 / 3.0).max() < 1e-10
    assert np.abs(v[1:]).max() < 1e-10
    SL, _ = ref.singular_matrices(X, p, 2 * p)
    vr = ref.self_apply(SL, f.reshape(-1), p).reshape(3, -1)
    assert np.abs(vr[0] - 2.0 / 3.0).max() < 1e-10


def test_far_field_vs_reference(ref):
    from tests.helpers import small_suspension
    X, f = small_suspension(2, 6, seed=5)
    p = 6
    ours = stokes.far_velocity(X, f, p)
    theirs, _ = ref.far_sl(X, f, p)
    assert rel_err(ours, theirs) < FAR_TOL
    a1, qw1 = ref.area_weights(X, p)
    assert rel_err(sh.area_element(X, p).reshape(-1), a1) < PRIM_TOL
    assert rel_err(sh.smooth_weights_grid(p), qw1) < PRIM_TOL


def test_direct_kernels_vs_reference(ref):
    rng = np.random.default_rng(7)
    np_ = 300
    src = rng.standard_normal(3 * np_)
    den = rng.standard_normal(3 * np_)
    assert rel_err(stokes.alltoall(src, den), ref.alltoall(src, den)) < FAR_TOL
    src[3:6] = src[0:3]  # a coincident pair contributes nothing in both
    assert rel_err(stokes.alltoall(src, den), ref.alltoall(src, den)) < FAR_TOL
    ns, stride = 3, 40
    S = rng.standard_normal(3 * ns * stride)
    T = rng.standard_normal(3 * ns * stride)
    D = rng.standard_normal(3 * ns * stride)
    Q = rng.uniform(0.5, 1.5, stride)
    a = stokes.direct_stokes(stride, stride, ns, 5, 33, Q, T, S, D)
    b = ref.direct_stokes(stride, stride, ns, 5, 33, Q, T, S, D)
    assert rel_err(a, b) < FAR_TOL


@pytest.mark.slow
def test_full_composition_c1(ref):
    """The FP64 StokesVelocity composition on the 8-vesicle p=12 suspension."""
    from ves3d_b200 import workloads
    X, f, p = workloads.make("c1_8ves_p12")
    ours = stokes.stokes_velocity_sl(X, f, p)
    theirs, _ = ref.stokes_velocity_sl(X, f, p, 2 * p)
    assert rel_err(ours, theirs) < REF_SELF_NOISE


# ---- double layer -------------------------------------------------------------------

@pytest.mark.parametrize("p", [6, 12])
def test_double_layer_self_vs_reference(ref, p):
    """The oracle's DL self matrix (StokesSingularInteg with DLMatrix) against the
    reference's, through the self velocity, within the reference's self-part noise."""
    X = ellipsoid_pair(p)
    g = np.random.default_rng(p).standard_normal(X.size)
    _, DL = ref.singular_matrices(X, p, 2 * p, sl=False, dl=True)
    theirs = ref.self_apply(DL, g, p)
    assert rel_err(sh.self_apply(sh.stokes_singular_matrix(X, p, 2 * p, single=False), g, p), theirs) < REF_SELF_NOISE
    ours_u = sh.self_apply(sh.stokes_singular_matrix(X, p, 2 * p, single=False, stable=False), g, p)
    assert rel_err(ours_u, theirs) < REF_SELF_NOISE


def test_double_layer_direct_vs_reference(ref):
    """oracle_direct_stokes_dl against DirectStokesDoubleLayerKernel, with and without
    weights, a coincident pair included."""
    rng = np.random.default_rng(11)
    ns, nt, nv = 40, 30, 3
    S = rng.standard_normal(3 * ns * nv)
    T = rng.standard_normal(3 * nt * nv)
    T[0], T[nt], T[2 * nt] = S[0], S[ns], S[2 * ns]  # target 0 of surface 0 on source 0
    N = rng.standard_normal(3 * ns * nv)
    D = rng.standard_normal(3 * ns * nv)
    Q = rng.uniform(0.5, 1.5, ns)
    for q in (Q, None):
        a = stokes.direct_stokes_dl(ns, nt, nv, 0, 25, q, T, S, N, D)
        b = ref.direct_stokes_dl(ns, nt, nv, 0, 25, q, T, S, N, D)
        assert rel_err(a, b) < FAR_TOL


@pytest.mark.parametrize("p", [6, 8])
def test_far_double_layer_vs_reference(ref, p):
    """The far double layer (other vesicles only) = the reference's DL kernel over all
    points as one surface minus its per-vesicle sums."""
    from tests.helpers import small_suspension
    X, g = small_suspension(2, p, seed=5)
    ng = sh.ngrid(p)
    nv = X.size // (3 * ng)
    N = stokes.unit_normal(X, p)
    D = stokes.far_density(X, g, p)

    def whole(A):
        return A.reshape(nv, 3, ng).transpose(1, 0, 2).reshape(-1)

    allp = ref.direct_stokes_dl(nv * ng, nv * ng, 1, 0, nv * ng, None, whole(X), whole(X), whole(N), whole(D))
    allp = allp.reshape(3, nv, ng).transpose(1, 0, 2).reshape(-1)
    own = ref.direct_stokes_dl(ng, ng, nv, 0, ng, None, X, X, N, D)
    assert rel_err(stokes.far_dl_velocity(X, g, p), allp - own) < 1e-12
    assert rel_err(N.reshape(nv, 3, ng) * sh.area_element(X, p)[:, None, :],
                   np.cross(*[a.reshape(nv, 3, ng) for a in sh.shc2grid(sh.grid2shc(X, p, p), p, p, grads=True)[1:]],
                            axis=1)) < PRIM_TOL


@pytest.mark.parametrize("p,tol", [(8, 5e-4), (12, 1e-5), (16, 1e-7)])
def test_double_layer_of_constant_densities(p, tol):
    """Gauss's identity for the Stokes double layer: a constant density c on a closed
    surface gives -c/2 on the surface (outward normal) and nothing outside it, so with a
    constant per vesicle the total (self + far) is -c_v/2 on every vesicle; the error
    falls spectrally with p (measured 1.7e-4, 2.1e-6, 2.1e-8)."""
    from tests.helpers import small_suspension
    X, _ = small_suspension(2, p, seed=3)
    ng = sh.ngrid(p)
    nv = X.size // (3 * ng)
    C = np.random.default_rng(1).standard_normal((nv, 3))
    g = np.repeat(C[:, :, None], ng, axis=2).reshape(-1)
    u = stokes.stokes_velocity_dl(X, g, p).reshape(nv, 3, ng)
    assert np.abs(u + 0.5 * C[:, :, None]).max() < tol


def test_double_layer_sphere_identity():
    p = 8
    X = unit_sphere(p)
    c = np.array([0.3, -1.0, 0.5])
    g = np.repeat(c[:, None], sh.ngrid(p), axis=1).reshape(-1)
    u = sh.self_apply(sh.stokes_singular_matrix(X, p, 2 * p, single=False), g, p).reshape(3, -1)
    assert np.abs(u + 0.5 * c[:, None]).max() < 1e-13


def test_reference_double_layer_test_setup():
    """The setup of the reference's test/StokesDoubleLayerTest.cc:59-170 (p = 6, a unit sphere
    sampled at equispaced latitudes (i+1) pi/8 about the x axis, density 1 in every
    component), whose known answer is |velocity| = 1/2 within 0.03. With the outward normal
    X_theta x X_phi of StokesVelocity the double layer is -1/2 (1.8e-5 here); the test
    asserts +1/2 through Surface::getNormal() and DirectStokesDoubleLayer, i.e. with the
    normal of the opposite orientation."""
    p = 6
    i = np.arange(p + 1)[:, None]
    j = np.arange(2 * p)[None, :]
    th = (i + 1) * np.pi / (p + 2)
    X = np.stack([np.cos(th) + 0 * j, np.sin(th) * np.sin(j * np.pi / p), np.sin(th) * np.cos(j * np.pi / p)])
    X = X.reshape(-1)
    n = stokes.unit_normal(X, p).reshape(3, -1)
    assert (n * X.reshape(3, -1)).sum(axis=0).min() > 0.99  # outward
    u = sh.self_apply(sh.stokes_singular_matrix(X, p, 2 * p, single=False), np.ones(X.size), p)
    assert np.abs(u + 0.5).max() < 0.03 and np.abs(u + 0.5).max() < 1e-4


def test_reference_double_layer_kernel_sign(ref):
    """The reference's DirectStokesDoubleLayerKernel with outward unit normals and density 1
    (times area and weights) gives -1 at a sphere's centre: D[c] = -c inside, -c/2 on the
    surface, the convention of the DL matrices and of this build."""
    p = 16
    X = unit_sphere(p)
    ng = sh.ngrid(p)
    n = stokes.unit_normal(X, p)
    w = sh.area_element(X, p).reshape(-1) * sh.smooth_weights_grid(p)
    den = np.tile(w, 3)
    T = X.copy()
    T[0] = T[ng] = T[2 * ng] = 0.0  # target 0 at the centre
    u = ref.direct_stokes_dl(ng, ng, 1, 0, 1, None, T, X, n, den)
    assert abs(u[0] + 1) < 1e-12 and abs(u[ng] + 1) < 1e-12 and abs(u[2 * ng] + 1) < 1e-12
    assert rel_err(stokes.direct_stokes_dl(ng, ng, 1, 0, 1, None, T, X, n, den), u) < FAR_TOL


def test_target_velocity_identities():
    """Off-surface targets (SetTrgCoord) on a sphere of radius a = 2 with uniform density:
    the single layer is (2/3) a f inside and, on the axis of f at distance r outside,
    (a^2/r - a^4/(3 r^3)) f (the flow of the translating sphere it equals); the double layer
    of a constant c is -c inside and 0 outside."""
    p = 12
    a = 2.0
    X = a * unit_sphere(p)
    f = np.zeros((3, sh.ngrid(p)))
    f[0] = 1.0
    T = np.array([[0.0, 0.0, 0.0], [0.3, -0.2, 0.1], [5.0, 0.0, 0.0]])
    u = stokes.target_velocity(X, f.reshape(-1), p, T).reshape(-1, 3)
    assert np.abs(u[:2, 0] - 2.0 * a / 3.0).max() < 1e-12 and np.abs(u[:2, 1:]).max() < 1e-12
    assert abs(u[2, 0] - (a * a / 5.0 - a ** 4 / (3 * 125.0))) < 1e-9  # quadrature: 7.6e-11 here
    c = np.array([0.3, -1.0, 0.5])
    g = np.repeat(c[:, None], sh.ngrid(p), axis=1).reshape(-1)
    v = stokes.target_velocity(X, np.zeros(X.size), p, T, g).reshape(-1, 3)
    assert np.abs(v[:2] + c).max() < 1e-12 and np.abs(v[2]).max() < 1e-8
