"""CPU oracle (test infrastructure only): a numpy restatement of the reference's
spherical-harmonic machinery and singular self-interaction for the StokesVelocity
path. Only tests/, bench.py's cpu_baseline leg and __graft_entry__.smoke() may use
it, and only as the checker; the product never imports it.

Every function follows the reference's `SphericalHarmonics<Real>` (file
src/SphericalHarmonics.cc of lu1and10/ves3d); line numbers are cited per function.
Parity of this restatement is pinned against the reference's own compiled code
(oracle/_ref, see oracle/ref/Makefile) by tests/test_oracle_pin.py and against the
analytic sphere identities (single layer of f=(1,0,0) on the unit sphere is 2/3 f).

Layouts (reference conventions):
  grid       [fun][i][j]  i = Gauss-Legendre latitude (ascending cos theta), j = longitude j*pi/p
  coefficients [fun][Ncoef] in blocks by Fourier index jf = 0..2p-1 (m = (jf+1)//2),
             each block holding degrees n = m..p  (src/SphericalHarmonics.cc:32-38)
"""
from functools import lru_cache

import numpy as np

SQRT2PI = np.sqrt(2.0 * np.pi)


def ncoef(p):
    return p * (p + 2)


def ngrid(p):
    return 2 * p * (p + 1)


def block_len(p, jf):
    """Length of the coefficient block of Fourier index jf (src/SphericalHarmonics.cc:30-35)."""
    return p + 1 - (jf + 1) // 2


@lru_cache(maxsize=None)
def block_offsets(p):
    off = [0]
    for jf in range(2 * p):
        off.append(off[-1] + block_len(p, jf))
    assert off[-1] == ncoef(p)
    return tuple(off)


@lru_cache(maxsize=None)
def gauss_legendre(n):
    """n-point Gauss-Legendre rule on [-1,1], nodes ascending.

    The reference calls Burkardt's cgqf(n, kind=1, 0, 0, -1, 1) (src/legendre_rule.cc:269),
    i.e. the Golub-Welsch eigenvalue method on the Jacobi matrix. Restated here as
    Golub-Welsch followed by Newton polishing on P_n.
    """
    if n == 1:
        return np.array([0.0]), np.array([2.0])
    k = np.arange(1, n)
    beta = k / np.sqrt(4.0 * k * k - 1.0)
    J = np.diag(beta, 1) + np.diag(beta, -1)
    x = np.linalg.eigvalsh(J)
    for _ in range(3):
        p0 = np.ones_like(x)
        p1 = x.copy()
        for m in range(2, n + 1):
            p0, p1 = p1, ((2 * m - 1) * x * p1 - (m - 1) * p0) / m
        dp = n * (x * p1 - p0) / (x * x - 1.0)
        x = x - p1 / dp
    p0 = np.ones_like(x)
    p1 = x.copy()
    for m in range(2, n + 1):
        p0, p1 = p1, ((2 * m - 1) * x * p1 - (m - 1) * p0) / m
    dp = n * (x * p1 - p0) / (x * x - 1.0)
    w = 2.0 / ((1.0 - x * x) * dp * dp)
    return x, w


def legendre_nodes(p):
    """src/SphericalHarmonics.cc:544-555."""
    return gauss_legendre(p + 1)[0]


def legendre_weights(p):
    """Smooth quadrature weights w_i * pi / p / sin(theta_i) (src/SphericalHarmonics.cc:558-570)."""
    x, w = gauss_legendre(p + 1)
    return w * np.pi / p / np.sqrt(1.0 - x * x)


def legpoly(x, degree, u=None):
    """Normalised associated Legendre functions (src/SphericalHarmonics.cc:889-928).

    Returns array [Naleg][len(x)] ordered m-major: (m=0: n=0..d), (m=1: n=1..d), ...
    u = sin(theta); the reference always forms it as sqrt(1-x^2). Callers that know
    sin(theta) more accurately than 1-x^2 allows (points on or next to a pole) pass it.
    """
    x = np.atleast_1d(np.asarray(x, dtype=np.float64))
    N = x.size
    d = degree
    out = np.zeros(((d + 1) * (d + 2) // 2, N))
    if u is None:
        u = np.sqrt(np.maximum(1.0 - x * x, 0.0))
        u[x * x > 1.0] = 0.0
    else:
        u = np.atleast_1d(np.asarray(u, dtype=np.float64))
    # diagonal P(m,m)
    diag = [np.full(N, 1.0 / np.sqrt(4.0 * np.pi))]
    for i in range(1, d + 1):
        c = np.sqrt((2.0 * i + 1.0) / (2.0 * i))
        diag.append(-diag[-1] * u * c)
    off = 0
    for m in range(d + 1):
        out[off] = diag[m]
        pmm = np.zeros(N)
        pmmp1 = diag[m]
        for ll in range(m + 1, d + 1):
            a = np.sqrt(((2.0 * ll - 1) * (2 * ll + 1)) / ((ll - m) * (ll + m)))
            b = np.sqrt(((2.0 * ll + 1) * (ll + m - 1) * (ll - m - 1)) / ((ll - m) * (ll + m) * (2 * ll - 3))) if ll > 1 else 0.0
            pll = x * a * pmmp1 - b * pmm
            pmm, pmmp1 = pmmp1, pll
            out[off + ll - m] = pll
        off += d + 1 - m
    return out


def _aidx(d, m, n):
    return ((2 * d - m + 1) * m) // 2 + n


def legpoly_deriv(x, degree):
    """theta-derivative of legpoly (src/SphericalHarmonics.cc:931-950)."""
    x = np.atleast_1d(np.asarray(x, dtype=np.float64))
    d = degree
    P = legpoly(x, d)
    H = np.zeros_like(P)
    s = np.sqrt(1.0 - x * x)
    for m in range(d + 1):
        for n in range(m, d + 1):
            Pn = P[_aidx(d, m, n)]
            c1 = float(m)
            if m + 1 <= n:
                Pn_ = P[_aidx(d, m + 1, n)]
                c2 = np.sqrt(n + m + 1.0) * np.sqrt(float(n - m) if n > m else 1.0)
            else:
                Pn_ = P[0]
                c2 = 0.0
            H[_aidx(d, m, n)] = -(c1 * x * Pn + c2 * s * Pn_) / s
    return H


@lru_cache(maxsize=None)
def mat_fourier(p0, p1):
    """Synthesis DFT 2p0 x 2p1 (src/SphericalHarmonics.cc:607-627)."""
    j = np.arange(2 * p1)
    M = np.zeros((2 * p0, 2 * p1))
    M[0] = SQRT2PI
    for k in range(1, p0):
        M[2 * k - 1] = SQRT2PI * np.cos(j * k * np.pi / p1)
        M[2 * k] = SQRT2PI * np.sin(j * k * np.pi / p1)
    M[2 * p0 - 1] = SQRT2PI * np.cos(j * p0 * np.pi / p1)
    return M


@lru_cache(maxsize=None)
def mat_fourier_inv(p0, p1):
    """Analysis DFT 2p0 x 2p1 (src/SphericalHarmonics.cc:629-652)."""
    c = 1.0 / np.sqrt(2.0 * np.pi) / p0
    M = np.zeros((2 * p0, 2 * p1))
    q = min(p1, p0)
    j = np.arange(2 * p0)
    M[:, 0] = c * 0.5
    for k in range(1, q):
        M[:, 2 * k - 1] = c * np.cos(j * k * np.pi / p0)
        M[:, 2 * k] = c * np.sin(j * k * np.pi / p0)
    M[:, 2 * q - 1] = c * np.cos(j * q * np.pi / p0)
    if q == p0:
        M[:, 2 * q - 1] *= 0.5
    return M


@lru_cache(maxsize=None)
def mat_fourier_grad(p0, p1):
    """Longitude derivative of the synthesis DFT (src/SphericalHarmonics.cc:654-674)."""
    j = np.arange(2 * p1)
    M = np.zeros((2 * p0, 2 * p1))
    for k in range(1, p0):
        M[2 * k - 1] = -SQRT2PI * k * np.sin(j * k * np.pi / p1)
        M[2 * k] = SQRT2PI * k * np.cos(j * k * np.pi / p1)
    M[2 * p0 - 1] = -SQRT2PI * p0 * np.sin(j * p0 * np.pi / p1)
    return M


def _split_m(A, p0):
    out = []
    off = 0
    for m in range(p0 + 1):
        ln = p0 + 1 - m
        out.append(A[off:off + ln])
        off += ln
    return out


@lru_cache(maxsize=None)
def mat_legendre(p0, p1):
    """Per-m synthesis matrices (p0+1-m) x (p1+1) at the p1 nodes (:677-700)."""
    return _split_m(legpoly(legendre_nodes(p1), p0), p0)


@lru_cache(maxsize=None)
def mat_legendre_grad(p0, p1):
    """Per-m theta-derivative synthesis matrices (:733-755)."""
    return _split_m(legpoly_deriv(legendre_nodes(p1), p0), p0)


@lru_cache(maxsize=None)
def mat_legendre_inv(p0, p1):
    """Per-m analysis matrices (p0+1) x (p1+1-m): P * w * 2pi (:702-730)."""
    x, w = gauss_legendre(p0 + 1)
    blocks = _split_m(legpoly(x, p1), p1)
    return [(b * w[None, :] * 2.0 * np.pi).T.copy() for b in blocks]


def _fourier_block_ids(p):
    """For each Fourier index jf, its m; jf=0 is m=0, then (cos,sin) pairs, last is m=p cos."""
    return [(jf + 1) // 2 for jf in range(2 * p)]


def filter_coeffs(p, freq=-1, exponent=None):
    """SHTrans's frequency filters in the per-function coefficient order (src/SHTrans.cc:
    8-45): freq -1 means 2p/3 (integer division); exponent None is the hard cut of
    lowPassFilter (keep degrees n <= freq), a number the polynomial filter of
    lowPassFilterPoly (1 - (n/freq)^exponent for n < freq, else 0)."""
    freq = 2 * p // 3 if freq == -1 else freq
    off = block_offsets(p)
    c = np.empty(ncoef(p))
    for jf in range(2 * p):
        m = (jf + 1) // 2
        deg = m + np.arange(off[jf + 1] - off[jf])
        if exponent is None:
            c[off[jf]:off[jf + 1]] = np.where(deg > freq, 0.0, 1.0)
        else:
            c[off[jf]:off[jf + 1]] = np.where(deg >= freq, 0.0, 1.0 - (deg / freq) ** exponent)
    return c


def scale_freq(S, p, coeff):
    """SHTrans::ScaleFreq (src/SHTrans.cc:190-223) on function-major coefficients."""
    return (np.asarray(S, dtype=np.float64).reshape(-1, ncoef(p)) * np.asarray(coeff)[None, :]).reshape(-1)


def low_pass(X, p, freq=-1, exponent=None):
    """SHTrans::lowPassFilter / lowPassFilterPoly (src/SHTrans.cc:172-188): analysis, scaling,
    synthesis of grid functions [n_fun][(p+1) 2p]."""
    return shc2grid(scale_freq(grid2shc(X, p, p), p, filter_coeffs(p, freq, exponent)), p, p)


def grid2shc(X, p0, p1):
    """Analysis: grid at order p0 -> coefficients at order p1 (src/SphericalHarmonics.cc:152-235)."""
    X = np.asarray(X, dtype=np.float64).reshape(-1, p0 + 1, 2 * p0)
    nf = X.shape[0]
    F = X @ mat_fourier_inv(p0, p1)  # [nf][lat][jf] (2p1 columns)
    Ml = mat_legendre_inv(p0, p1)
    S = np.zeros((nf, ncoef(p1)))
    off = block_offsets(p1)
    for jf in range(2 * p1):
        m = (jf + 1) // 2
        S[:, off[jf]:off[jf + 1]] = F[:, :, jf] @ Ml[m]
    return S.reshape(-1)


def shc2grid(S, p0, p1, grads=False):
    """Synthesis: coefficients at order p0 -> grid at order p1, optionally with the
    longitude derivative ("X_theta") and latitude derivative ("X_phi") as named in the
    reference (src/SphericalHarmonics.cc:4-149)."""
    S = np.asarray(S, dtype=np.float64).reshape(-1, ncoef(p0))
    nf = S.shape[0]
    Ml = mat_legendre(p0, p1)
    off = block_offsets(p0)
    B = np.zeros((nf, p1 + 1, 2 * p0))
    for jf in range(2 * p0):
        m = (jf + 1) // 2
        B[:, :, jf] = S[:, off[jf]:off[jf + 1]] @ Ml[m]
    X = (B @ mat_fourier(p0, p1)).reshape(-1)
    if not grads:
        return X
    Xt = (B @ mat_fourier_grad(p0, p1)).reshape(-1)
    Mdl = mat_legendre_grad(p0, p1)
    Bd = np.zeros((nf, p1 + 1, 2 * p0))
    for jf in range(2 * p0):
        m = (jf + 1) // 2
        Bd[:, :, jf] = S[:, off[jf]:off[jf + 1]] @ Mdl[m]
    Xp = (Bd @ mat_fourier(p0, p1)).reshape(-1)
    return X, Xt, Xp


def shc2grid_transpose(X, p0, p1):
    """Adjoint of shc2grid(., p1, p0): grid at order p0 -> coefficients at order p1
    (src/SphericalHarmonics.cc:238-322)."""
    X = np.asarray(X, dtype=np.float64).reshape(-1, p0 + 1, 2 * p0)
    nf = X.shape[0]
    F = X @ mat_fourier(p1, p0).T  # [nf][lat][2p1]
    Ml = mat_legendre(p1, p0)
    off = block_offsets(p1)
    S = np.zeros((nf, ncoef(p1)))
    for jf in range(2 * p1):
        m = (jf + 1) // 2
        S[:, off[jf]:off[jf + 1]] = F[:, :, jf] @ Ml[m].T
    return S.reshape(-1)


def shc2pole(S, p0):
    """Values at x=-1 and x=+1 from the m=0 block (src/SphericalHarmonics.cc:325-360)."""
    S = np.asarray(S, dtype=np.float64).reshape(-1, ncoef(p0))
    QP = np.stack([legpoly(np.array([-1.0]), p0)[:p0 + 1, 0],
                   legpoly(np.array([1.0]), p0)[:p0 + 1, 0]]) * SQRT2PI
    P = S[:, :p0 + 1] @ QP.T
    return P.reshape(-1)


@lru_cache(maxsize=None)
def coeff_perm(p0):
    """Indices of degree-n coefficients, ordered by Fourier index (src/SphericalHarmonics.cc:365-376)."""
    perm = [[0] * min(2 * n + 1, 2 * p0) for n in range(p0 + 1)]
    itr = 0
    for i in range(2 * p0):
        m = (i + 1) // 2
        for n in range(m, p0 + 1):
            perm[n][i] = itr
            itr += 1
    return tuple(tuple(v) for v in perm)


@lru_cache(maxsize=None)
def mat_rotate(p0, stable=True):
    """Per (latitude angle l, degree n) rotation blocks (src/SphericalHarmonics.cc:760-860).

    The reference evaluates the rotated basis with sin(theta) = sqrt(1 - x^2). For the
    rotated grid points that land on a pole (x = -1 in exact arithmetic, e.g. grid point
    (l, p0) under rotation l) the rounding of x (~1e-16) becomes ~1e-8 in sin(theta), so
    the reference's blocks carry O(1e-8) noise whose realisation depends on how its BLAS
    rounds the 3x3 coordinate product. stable=True takes sin(theta) = hypot(y, z) of the
    rotated point instead, which is exact to rounding; stable=False reproduces the
    reference's formula.
    """
    nc = ncoef(p0)
    ng = ngrid(p0)
    x = legendre_nodes(p0)
    i = np.repeat(np.arange(p0 + 1), 2 * p0)
    j = np.tile(np.arange(2 * p0), p0 + 1)
    s = np.sqrt(1.0 - x[i] ** 2)
    C0 = np.stack([x[i], s * np.sin(np.pi * j / p0), s * np.cos(np.pi * j / p0)])
    perm = coeff_perm(p0)
    Mr = []
    for l in range(p0 + 1):
        c_ = -x[l]
        s_ = -np.sqrt(1.0 - x[l] * x[l])
        R = np.array([[c_, 0, -s_], [0, 1, 0], [s_, 0, c_]])
        C1 = R @ C0
        Mleg = legpoly(C1[0], p0, np.hypot(C1[1], C1[2]) if stable else None)
        theta = np.arctan2(C1[1], C1[2])
        M = np.zeros((nc, ng))
        o0 = 0
        o1 = 0
        for m in range(p0 + 1):
            ln = p0 + 1 - m
            M[o1:o1 + ln] = SQRT2PI * Mleg[o0:o0 + ln] * np.cos(m * theta)[None, :]
            o1 += ln
            if m != 0 and m != p0:
                M[o1:o1 + ln] = SQRT2PI * Mleg[o0:o0 + ln] * np.sin(m * theta)[None, :]
                o1 += ln
            o0 += ln
        C2C = grid2shc(M.reshape(-1), p0, p0).reshape(nc, nc)
        for n in range(p0 + 1):
            pn = np.array(perm[n])
            Mr.append(C2C[np.ix_(pn, pn)].copy())
    return Mr


def _phase(S, p0, j, sign):
    """Longitude phase exp(-i k j pi/p0) on each (cos, sin) block pair (:383-405, :494-516)."""
    out = S.copy()
    off = 0
    for k in range(p0 + 1):
        ln = p0 + 1 - k
        if k != 0 and k != p0:
            c = np.cos(k * j * np.pi / p0)
            s = sign * np.sin(k * j * np.pi / p0)
            x0 = S[..., off:off + ln]
            x1 = S[..., off + ln:off + 2 * ln]
            out[..., off:off + ln] = x0 * c - x1 * s
            out[..., off + ln:off + 2 * ln] = x0 * s + x1 * c
            off += 2 * ln
        else:
            off += ln
    return out


def _apply_blocks(B, Mr, p0, t, transpose=False):
    perm = coeff_perm(p0)
    out = np.zeros_like(B)
    for n in range(p0 + 1):
        pn = np.array(perm[n])
        M = Mr[t * (p0 + 1) + n]
        out[..., pn] = B[..., pn] @ (M.T if transpose else M)
    return out


def rotate_all(S, p0, dof, stable=True):
    """All p0(p0+1) rotations of each coefficient set (src/SphericalHarmonics.cc:363-449).

    In:  [N][dof][Ncoef].  Out: [N][t=0..p0][j=0..p0-1][dof][Ncoef].
    """
    nc = ncoef(p0)
    S = np.asarray(S, dtype=np.float64).reshape(-1, dof, nc)
    N = S.shape[0]
    Mr = mat_rotate(p0, stable)
    out = np.zeros((N, p0 + 1, p0, dof, nc))
    for j in range(p0):
        B0 = _phase(S, p0, j, -1.0)
        for t in range(p0 + 1):
            out[:, t, j] = _apply_blocks(B0, Mr, p0, t)
    return out.reshape(-1)


def move_pole(X, p0, trg_i, trg_j, stable=True):
    """MovePole(trg_i, trg_j) on grid functions X [n][(p0+1) 2p0] (src/MovePole.cc:159-195):
    the rotation of rotate_all for latitude trg_i and longitude trg_j, trg_j in [0, 2p0)
    (grid point (trg_i, trg_j) to the x = -1 pole), through the coefficients."""
    nc = ncoef(p0)
    S = grid2shc(X, p0, p0).reshape(-1, nc)
    B0 = _phase(S, p0, trg_j, -1.0)
    R = _apply_blocks(B0, mat_rotate(p0, stable), p0, trg_i)
    return shc2grid(R.reshape(-1), p0, p0)


def aggregate_rotation(mat, nlat, nlong, vec):
    """Device<CPU>::AggregateRotation for one operand (src/DeviceCPU.cc:646-680): for every
    longitude jj, CircShift the columns of the column-major np x np matrix mat within each
    latitude block by jj and apply it to the nsub grid functions vec [nsub][np]. Returns
    [nlong][nsub][np]."""
    npt = nlat * nlong
    A = np.asarray(mat, np.float64).reshape(npt, npt).T  # A[row][col]
    lat = np.arange(npt) // nlong
    lon = np.arange(npt) % nlong
    vec = np.asarray(vec, np.float64).reshape(-1, npt)
    return np.stack([vec @ A[:, lat * nlong + (lon - jj) % nlong].T for jj in range(nlong)])


def rotate_transpose(S_, p0, dof, stable=True):
    """Adjoint of rotate_all (src/SphericalHarmonics.cc:452-541); same layout in and out."""
    nc = ncoef(p0)
    S_ = np.asarray(S_, dtype=np.float64).reshape(-1, p0 + 1, p0, dof, nc)
    Mr = mat_rotate(p0, stable)
    out = np.zeros_like(S_)
    for t in range(p0 + 1):
        B0 = _apply_blocks(S_[:, t], Mr, p0, t, transpose=True)  # [N][j][dof][nc]
        for j in range(p0):
            out[:, t, j] = _phase(B0[:, j], p0, j, +1.0)
    return out.reshape(-1)


def singular_weights(p1):
    """Pole-singular quadrature weights (src/SphericalHarmonics.cc:573-604)."""
    x, w = gauss_legendre(p1 + 1)
    alp0 = legpoly(np.array([1.0]), p1)[:p1 + 1, 0]
    alp = legpoly(x, p1)[:p1 + 1]  # [j][i]
    jj = np.arange(p1 + 1)
    Yf = (4.0 * np.pi / (2 * jj + 1) * alp0) @ alp
    return (w * np.pi / p1) * Yf / np.cos(np.arccos(x) / 2.0)


SYM = np.array([[0, 1, 2], [1, 3, 4], [2, 4, 5]])  # (c_in, c_out) -> unique tensor component


def singular_kernel(X, Xt, Xp, trg, p1, single=True):
    """Pole-target kernel values (src/SphericalHarmonics.cc:971-1068).

    X, Xt, Xp: [N][3][M1] rotated/upsampled source surfaces; trg: [N][3][2] pole targets.
    Returns [N][2][6][M1] weighted tensor components (SL if single else DL).
    """
    M1 = ngrid(p1)
    X = X.reshape(-1, 3, M1)
    Xt = Xt.reshape(-1, 3, M1)
    Xp = Xp.reshape(-1, 3, M1)
    trg = trg.reshape(-1, 3, 2)
    N = X.shape[0]
    qw = singular_weights(p1)
    j0 = np.repeat(np.arange(p1 + 1), 2 * p1)
    eps = np.finfo(np.float64).eps
    nx = Xt[:, 1] * Xp[:, 2] - Xt[:, 2] * Xp[:, 1]
    ny = Xt[:, 2] * Xp[:, 0] - Xt[:, 0] * Xp[:, 2]
    nz = Xt[:, 0] * Xp[:, 1] - Xt[:, 1] * Xp[:, 0]
    out = np.zeros((N, 2, 6, M1))
    for t in range(2):
        dx = trg[:, 0, t][:, None] - X[:, 0]
        dy = trg[:, 1, t][:, None] - X[:, 1]
        dz = trg[:, 2, t][:, None] - X[:, 2]
        r2 = dx * dx + dy * dy + dz * dz
        with np.errstate(divide="ignore"):
            rinv = 1.0 / np.sqrt(r2)
        rinv[r2 <= eps] = 0.0
        rinv2 = rinv * rinv
        w = qw[j0 * t + (p1 - j0) * (1 - t)][None, :]
        if single:
            area = np.sqrt(nx * nx + ny * ny + nz * nz)
            a1 = (1.0 / (8.0 * np.pi)) * w * area * rinv
            a2 = a1 * rinv2
            out[:, t, 0] = a1 + dx * dx * a2
            out[:, t, 1] = dx * dy * a2
            out[:, t, 2] = dx * dz * a2
            out[:, t, 3] = a1 + dy * dy * a2
            out[:, t, 4] = dy * dz * a2
            out[:, t, 5] = a1 + dz * dz * a2
        else:
            rinv5 = rinv2 * rinv2 * rinv
            q = (3.0 / (4.0 * np.pi)) * w * (nx * dx + ny * dy + nz * dz) * rinv5
            out[:, t, 0] = dx * dx * q
            out[:, t, 1] = dx * dy * q
            out[:, t, 2] = dx * dz * q
            out[:, t, 3] = dy * dy * q
            out[:, t, 4] = dy * dz * q
            out[:, t, 5] = dz * dz * q
    return out


def stokes_singular_matrix(X0, p0, p1, single=True, stable=True):
    """Per-vesicle self-interaction matrix, (3 Ncoef) x (3 Ncoef), row = input density
    coefficient (c_in*Ncoef + k), column = output velocity coefficient (c_out*Ncoef + k')
    (src/SphericalHarmonics.cc:954-1180)."""
    nc = ncoef(p0)
    ng = ngrid(p0)
    X0 = np.asarray(X0, dtype=np.float64).reshape(-1, 3 * ng)
    nves = X0.shape[0]
    S0 = grid2shc(X0.reshape(-1), p0, p0)
    S = rotate_all(S0, p0, 3, stable)
    X, Xt, Xp = shc2grid(S, p0, p1, grads=True)
    trg = shc2pole(S, p0)
    K = singular_kernel(X, Xt, Xp, trg, p1, single=single)
    K1 = shc2grid_transpose(K.reshape(-1), p1, p0)
    K2 = rotate_transpose(K1, p0, 12, stable).reshape(nves, p0 + 1, p0, 2, 6, nc)
    # Rearrange (:1090-1172): target grid point of rotation (t, j), pole 0 -> (lat t, lon j),
    # pole 1 -> (lat p0-t, lon p0+j).
    M1 = np.zeros((nves, 3, nc, 3, p0 + 1, 2 * p0))
    for ci in range(3):
        for co in range(3):
            comp = SYM[ci, co]
            M1[:, ci, :, co, :, :p0] = np.transpose(K2[:, :, :, 0, comp, :], (0, 3, 1, 2))
            M1[:, ci, :, co, ::-1, p0:] = np.transpose(K2[:, :, :, 1, comp, :], (0, 3, 1, 2))
    SL = grid2shc(M1.reshape(-1), p0, p0)
    return SL.reshape(nves, 3 * nc, 3 * nc)


def area_element(X, p):
    """|X_theta x X_phi| on the order-p grid (src/StokesVelocity.cc:252-273)."""
    ng = ngrid(p)
    S = grid2shc(X, p, p)
    _, Xt, Xp = shc2grid(S, p, p, grads=True)
    Xt = Xt.reshape(-1, 3, ng)
    Xp = Xp.reshape(-1, 3, ng)
    n = np.cross(Xt, Xp, axis=1)
    return np.sqrt((n * n).sum(axis=1))


def smooth_weights_grid(p):
    return np.repeat(legendre_weights(p), 2 * p)


def self_apply(SL, f, p):
    """vel_self = SHC2Grid(Grid2SHC(f) . SL) (src/StokesVelocity.cc:397-451)."""
    nc = ncoef(p)
    F = grid2shc(f, p, p).reshape(-1, 3 * nc)
    V = np.einsum("vi,vij->vj", F, SL)
    return shc2grid(V.reshape(-1), p, p)
