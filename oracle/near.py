"""Test infrastructure only: a numpy restatement of the near-singular correction of the
velocity at off-surface targets (NearSingular<Real_t>, src/NearSingular.cc of
lu1and10/ves3d, as composed by StokesVelocity<Real>::operator(), src/StokesVelocity.cc:
475-500). Only tests/ may use it, as the checker of the GPU path.

Composition (the reference's, with its octree and its quadratic patches replaced):
  * every target gets the smooth quadrature of every vesicle at the far upsampling order
    p_up (the reference's PVFMM far field over scoord_far, src/StokesVelocity.cc:476-489);
  * a target closer than r_near = r_ves 2 / sqrt(p_up) to a vesicle (r_ves: the largest
    distance of a surface point from its vesicle's centroid, src/NearSingular.cc:119-160)
    has that vesicle's smooth contribution replaced (SubtractDirect, :1144-1212) by an
    interpolation along the line from its projection P on the surface through the target
    (operator(), :1392-1555): the smooth quadrature at the 7 points P + r_near x_l d,
    x_l = 1 + (l - 1)/6, d the unit direction to the target, and the on-surface value at
    P (x = 0): the vesicle's own singular-quadrature velocity there, plus, with a double
    layer, +g/2 outside and -g/2 inside (the jump of the double layer, :1474-1481);
    Lagrange polynomials on those 8 nodes (InterPoints / InterPoly, :1356-1374) evaluated
    at x = |T - P| / r_near.
Deviations (the reference's octree and patches are pvfmm-based and not available here):
near pairs are found by the distance to the vesicle's upsampled points; the projection
is Gauss-Newton on the spherical-harmonic surface itself (spectrally exact) from the
nearest upsampled grid point, instead of Newton on a quadratic patch through 3 x 3 grid
points (QuadraticPatch::project, :1589-1732); the on-surface velocity and double-layer
density at P are evaluated from their spherical-harmonic coefficients instead of a
quadratic patch of the upsampled values.
"""
import numpy as np

from . import sh, stokes

INTERP_DEG = 8


def inter_points(i, deg=INTERP_DEG):
    """Interpolation nodes: 0, then 1 + (i - 1)/(deg - 2) (src/NearSingular.cc:1357-1361)."""
    return 0.0 if i == 0 else 1.0 + (i - 1.0) / (deg - 2)


def inter_poly(x, j, deg=INTERP_DEG):
    """Lagrange polynomial of node j at x (src/NearSingular.cc:1363-1374)."""
    y = 1.0
    x0 = inter_points(j, deg)
    for k in range(deg):
        if k != j:
            xk = inter_points(k, deg)
            y *= (x - xk) / (x0 - xk)
    return y


def _trig(p, phi):
    """Fourier factors of the 2p coefficient blocks and their phi-derivatives."""
    t = np.zeros(2 * p)
    dt = np.zeros(2 * p)
    t[0] = 1.0
    for k in range(1, p):
        t[2 * k - 1], dt[2 * k - 1] = np.cos(k * phi), -k * np.sin(k * phi)
        t[2 * k], dt[2 * k] = np.sin(k * phi), k * np.cos(k * phi)
    t[2 * p - 1], dt[2 * p - 1] = np.cos(p * phi), -p * np.sin(p * phi)
    return t, dt


def basis(p, theta, phi):
    """The synthesis basis of order p at (theta, phi): value, d/dtheta and d/dphi of every
    coefficient [Ncoef] (the SHC2Grid basis SQRT2PI P_n^m(cos theta) trig_m(phi) of
    sh.mat_legendre / sh.mat_fourier, at a point off the grid). theta is measured so that
    cos(theta) is the Legendre variable of the grid."""
    x = np.cos(theta)
    P = sh.legpoly([x], p)[:, 0]
    dP = -sh.legpoly_deriv([x], p)[:, 0]  # legpoly_deriv is -dP/dtheta for x = cos(theta)
    t, dt = _trig(p, phi)
    v = np.zeros(sh.ncoef(p))
    vt = np.zeros_like(v)
    vp = np.zeros_like(v)
    off = sh.block_offsets(p)
    o0 = np.concatenate([[0], np.cumsum([p + 1 - m for m in range(p + 1)])])
    for jf in range(2 * p):
        m = (jf + 1) // 2
        a, b = off[jf], off[jf + 1]
        n = np.arange(m, m + (b - a))
        v[a:b] = sh.SQRT2PI * P[o0[m] + n - m] * t[jf]
        vt[a:b] = sh.SQRT2PI * dP[o0[m] + n - m] * t[jf]
        vp[a:b] = sh.SQRT2PI * P[o0[m] + n - m] * dt[jf]
    return v, vt, vp


def grid_angles(p):
    """(theta, phi) of the order-p grid, latitude-major."""
    th = np.arccos(sh.legendre_nodes(p))
    ph = np.pi * np.arange(2 * p) / p
    return np.repeat(th, 2 * p), np.tile(ph, p + 1)


def project(S3, p, T, theta0, phi0, iters=40):
    """Closest point of the surface with coefficients S3 [3][Ncoef] to T by Gauss-Newton in
    (theta, phi) from (theta0, phi0). Returns theta, phi, P, and the unit outward normal
    there (X_theta x X_phi, the orientation of stokes.unit_normal)."""
    th, ph = theta0, phi0
    for _ in range(iters):
        b, bt, bp = basis(p, th, ph)
        X, Xt, Xp = S3 @ b, S3 @ bt, S3 @ bp
        r = X - T
        J = np.stack([Xt, Xp], axis=1)
        A = J.T @ J
        A += 1e-14 * np.trace(A) * np.eye(2)
        step = -np.linalg.solve(A, J.T @ r)
        th, ph = th + step[0], ph + step[1]
        if np.abs(step).max() < 1e-15:
            break
    b, bt, bp = basis(p, th, ph)
    P = S3 @ b
    nrm = np.cross(S3 @ bt, S3 @ bp)
    return th, ph, P, nrm / np.linalg.norm(nrm)


def _upsampled(X, f, p, p_up, g=None):
    """Upsampled quadrature of every vesicle: points [nv][3][M1], weighted single-layer
    density f area qw, unit normals and weighted double-layer density (or None)."""
    ng1 = sh.ngrid(p_up)
    S = sh.grid2shc(X, p, p)
    Xu, Xt, Xp = (a.reshape(-1, 3, ng1) for a in sh.shc2grid(S, p, p_up, grads=True))
    n = np.cross(Xt, Xp, axis=1)
    area = np.sqrt((n * n).sum(1))
    qw = sh.smooth_weights_grid(p_up)[None, :]
    fu = sh.shc2grid(sh.grid2shc(f, p, p), p, p_up).reshape(-1, 3, ng1)
    den = fu * (area * qw)[:, None, :]
    out = [Xu, den, None, None]
    if g is not None:
        gu = sh.shc2grid(sh.grid2shc(g, p, p), p, p_up).reshape(-1, 3, ng1)
        out[2] = n / area[:, None, :]  # X_theta x X_phi normalised: outward (stokes.unit_normal)
        out[3] = gu * (area * qw)[:, None, :]
    return out


def _sl(Y, src, den):
    """Single layer at points Y [K][3] of sources src [3][M] with weighted density den."""
    r = src.T[None, :, :] - Y[:, None, :]
    r2 = (r * r).sum(2)
    rinv = np.where(r2 > 0, 1.0 / np.sqrt(np.where(r2 > 0, r2, 1.0)), 0.0)
    d = den.T[None, :, :]
    rd = (r * d).sum(2)
    return ((d * rinv[:, :, None] + r * (rd * rinv ** 3)[:, :, None]).sum(1)) / (8 * np.pi)


def _dl(Y, src, nrm, den):
    """Double layer at Y: 3/(4 pi) sum (r.n)(r.d) r / |r|^5, r = Y - source."""
    r = Y[:, None, :] - src.T[None, :, :]
    r2 = (r * r).sum(2)
    rinv = np.where(r2 > 0, 1.0 / np.sqrt(np.where(r2 > 0, r2, 1.0)), 0.0)
    rn = (r * nrm.T[None]).sum(2)
    rd = (r * den.T[None]).sum(2)
    return 3.0 / (4 * np.pi) * (r * (rn * rd * rinv ** 5)[:, :, None]).sum(1)


def target_velocity_near(X, f, p, T, g=None, p_up=None, SL=None, DL=None, return_info=False):
    """Velocity at targets T [M][3] with the near-singular correction (module docstring).
    Returns [M][3] point-major (and, with return_info, the near pairs and r_near)."""
    p_up = 2 * p if p_up is None else p_up
    ng = sh.ngrid(p)
    X = np.asarray(X, np.float64)
    f = np.asarray(f, np.float64)
    nv = X.size // (3 * ng)
    T = np.asarray(T, np.float64).reshape(-1, 3)
    Xu, den, nrm, dden = _upsampled(X, f, p, p_up, g)
    # r_ves: largest distance of a (order-p) surface point from its vesicle's centroid
    Xv = X.reshape(nv, 3, ng)
    cen = Xv.mean(2)
    r_ves = np.sqrt(((Xv - cen[:, :, None]) ** 2).sum(1)).max()
    r_near = r_ves * 2.0 / np.sqrt(p_up)
    # far field at the upsampled order from every vesicle
    u = np.zeros_like(T)
    for v in range(nv):
        u += _sl(T, Xu[v], den[v])
        if g is not None:
            u += _dl(T, Xu[v], nrm[v], dden[v])
    # self velocity coefficients of every vesicle (singular quadrature)
    if SL is None:
        SL = sh.stokes_singular_matrix(X, p, p_up)
    F = sh.grid2shc(f, p, p).reshape(nv, -1)
    Vc = np.einsum("vi,vij->vj", F, SL)
    if g is not None:
        if DL is None:
            DL = sh.stokes_singular_matrix(X, p, p_up, single=False)
        G = sh.grid2shc(g, p, p).reshape(nv, -1)
        Vc = Vc + np.einsum("vi,vij->vj", G, DL)
        Gc = G.reshape(nv, 3, -1)
    Vc = Vc.reshape(nv, 3, -1)
    Sx = sh.grid2shc(X, p, p).reshape(nv, 3, -1)
    thu, phu = grid_angles(p_up)
    pairs = []
    for t in range(T.shape[0]):
        for v in range(nv):
            d2 = ((Xu[v] - T[t][:, None]) ** 2).sum(0)
            k = int(np.argmin(d2))
            if d2[k] >= r_near * r_near:
                continue
            th, ph, P, nu = project(Sx[v], p, T[t], thu[k], phu[k])
            dR = T[t] - P
            dist = np.linalg.norm(dR)
            exterior = np.dot(dR, nu) >= 0  # nu is outward (X_theta x X_phi, as unit_normal)
            dirn = dR / dist if dist > 0 else nu
            line = P[None, :] + r_near * np.array([inter_points(l) for l in range(1, INTERP_DEG)])[:, None] * dirn
            y = np.zeros((INTERP_DEG, 3))
            y[1:] = _sl(line, Xu[v], den[v])
            if g is not None:
                y[1:] += _dl(line, Xu[v], nrm[v], dden[v])
            b, _, _ = basis(p, th, ph)
            y[0] = Vc[v] @ b
            if g is not None:
                y[0] += (0.5 if exterior else -0.5) * (Gc[v] @ b)
            x = dist / r_near
            interp = sum(y[l] * inter_poly(x, l) for l in range(INTERP_DEG))
            direct = _sl(T[t][None], Xu[v], den[v])[0]
            if g is not None:
                direct += _dl(T[t][None], Xu[v], nrm[v], dden[v])[0]
            u[t] += interp - direct
            pairs.append((t, v, x, bool(exterior)))
    if return_info:
        return u, dict(pairs=pairs, r_near=r_near, r_ves=r_ves)
    return u
