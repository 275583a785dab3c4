"""CPU oracle (test infrastructure only): surface geometry, interfacial forces, BiCGStab
and the globally implicit step, restated from the reference in numpy. Only tests/,
bench.py's cpu_baseline leg and __graft_entry__.smoke() may use it, as the checker.

Formulas follow (reference file:line):
  first forms, normal, div/grad coefficients   Surface::updateFirstForms  src/Surface.cc:212-262
  mean and Gaussian curvature                  Surface::updateAll          src/Surface.cc:264-323
  surface gradient / divergence                Surface::grad / div         src/Surface.cc:325-379
  linearised mean curvature                    Surface::linearizedMeanCurv src/Surface.cc:530-569
  bending, linear bending, tension forces      InterfacialForce            src/InterfacialForce.cc:21-125
  bending coefficient -kappa                   VesicleProperties::update   src/VesicleProps.cc:39-41
  gravity traction (explicit and linearised)   InterfacialForce::gravityForce src/InterfacialForce.cc:127-184
  area, volume, centres                        Surface::area/volume/getCenters src/Surface.cc:378-440
  surface quadrature                           GaussLegendreIntegrator     src/GLIntegrator.cc:33-80
  implicit matvec (solve for velocity)         ImplicitMatvecPhysical      src/InterfacialVelocity.cc:922-979
  right-hand side                              AssembleRhsVel              src/InterfacialVelocity.cc:716-771
  BiCGStab (preconditioned)                    BiCGStab::operator()        src/BiCGStab.cc:45-138
Derivatives come from the SphericalHarmonics tables of oracle/sh.py: u is the latitude
direction (the Legendre derivative), v the longitude direction (the Fourier derivative),
as SHTrans::FirstDerivatives / backward_du / backward_dv use them (src/SHTrans.cc:133-170).
  low-pass filter (opt-in, filter_freq)        SHTrans::lowPassFilter      src/SHTrans.cc:8-32, :172-180
Deliberate differences from the reference (the GPU path makes the same choices): forces
are evaluated at order p (the reference upsamples to params.upsample_freq), and by default
no low-pass filter is applied to curvatures, gradients and divergences. geometry(X, p,
filter_freq=f) turns the reference's filter on (coefficients of degree above f zeroed, the
reference's default f = 2p/3) for H, K, grad, div and the linearised curvature, which is
how the reference's own known answers for them are reproduced.
"""
import numpy as np

from . import sh
from . import stokes


def _d2_table(p):
    """Second latitude derivative of the normalised Legendre functions at the p nodes,
    per m block like sh.mat_legendre(p, p): P_uu = cot(theta) P_u - (n(n+1) - m^2/sin^2) P."""
    x = sh.legendre_nodes(p)
    s = np.sqrt(1.0 - x * x)
    cot = x / s
    P = sh.mat_legendre(p, p)
    D = sh.mat_legendre_grad(p, p)
    out = []
    for m in range(p + 1):
        n = np.arange(m, p + 1)[:, None]
        out.append(cot[None, :] * D[m] - (n * (n + 1) - (m * m) / (s * s)[None, :]) * P[m])
    return out


def _fourier_d2(p):
    j = np.arange(2 * p)
    M = np.zeros((2 * p, 2 * p))
    for k in range(1, p):
        M[2 * k - 1] = -sh.SQRT2PI * k * k * np.cos(j * k * np.pi / p)
        M[2 * k] = -sh.SQRT2PI * k * k * np.sin(j * k * np.pi / p)
    M[2 * p - 1] = -sh.SQRT2PI * p * p * np.cos(j * p * np.pi / p)
    return M


def synth(S, p, kind):
    """Coefficients -> grid derivative at order p: kind in '', 'u', 'v', 'uu', 'uv', 'vv'."""
    S = np.asarray(S, dtype=np.float64).reshape(-1, sh.ncoef(p))
    nf = S.shape[0]
    nu = kind.count("u")
    nv = kind.count("v")
    L = [sh.mat_legendre(p, p), sh.mat_legendre_grad(p, p), _d2_table(p)][nu]
    F = [sh.mat_fourier(p, p), sh.mat_fourier_grad(p, p), _fourier_d2(p)][nv]
    off = sh.block_offsets(p)
    B = np.zeros((nf, p + 1, 2 * p))
    for jf in range(2 * p):
        m = (jf + 1) // 2
        B[:, :, jf] = S[:, off[jf]:off[jf + 1]] @ L[m]
    return (B @ F).reshape(nf, -1)


def integrals(X, p):
    """Per vesicle: area = int W, volume = int (x.n)/3 W, centre = int (|x|^2/2) n W / volume,
    with the Gauss-Legendre surface weights w_i (2 pi / 2p) / sin(theta_i)
    (Surface::area / volume / getCenters, src/Surface.cc:378-440; GaussLegendreIntegrator,
    src/GLIntegrator.cc:33-80)."""
    geo = geometry(X, p)
    q = geo["W"] * sh.smooth_weights_grid(p)[None, :]
    Xv = geo["X"]
    area = q.sum(1)
    vol = ((Xv * geo["n"]).sum(1) / 3.0 * q).sum(1)
    cen = ((0.5 * (Xv * Xv).sum(1))[:, None, :] * geo["n"] * q[:, None, :]).sum(2) / vol[:, None]
    return area, vol, cen


def lowpass(f, p, freq):
    """Zero the coefficients of degree > freq of scalar fields f [..][ng]
    (SHTrans::lowPassFilter with filter_coeff_, src/SHTrans.cc:22-29, :172-180)."""
    if freq is None:
        return f
    return sh.low_pass(np.reshape(f, -1), p, freq).reshape(np.shape(f))


def geometry(X, p, filter_freq=None):
    """Per point: normalised E, F, G (divided by W^2), W, normal, cu, cv, H, K. With
    filter_freq set, H, K and the derived operators of this geometry are low-pass filtered
    as the reference's Surface does."""
    ng = sh.ngrid(p)
    X = np.asarray(X, dtype=np.float64).reshape(-1, 3, ng)
    nv = X.shape[0]
    S = sh.grid2shc(X.reshape(-1), p, p)
    d = {k: synth(S, p, k).reshape(nv, 3, ng) for k in ("u", "v", "uu", "uv", "vv")}
    xu, xv = d["u"], d["v"]
    E = (xu * xu).sum(1)
    F = (xu * xv).sum(1)
    G = (xv * xv).sum(1)
    W2 = E * G - F * F
    W = np.sqrt(W2)
    # the reference differentiates in theta (SHTrans::backward_du with d1legTrans, d/dtheta)
    # where u here is -d/dtheta, so its normal x_theta x x_phi / W is -(x_u x x_v) / W:
    # outward, and H of a sphere of radius R is -1/R
    n = -np.cross(xu, xv, axis=1) / W[:, None, :]
    En, Fn, Gn = E / W2, F / W2, G / W2
    cu = Gn[:, None] * xu - Fn[:, None] * xv
    cv = En[:, None] * xv - Fn[:, None] * xu
    L = (d["uu"] * n).sum(1)
    M = (d["uv"] * n).sum(1)
    N = (d["vv"] * n).sum(1)
    H = lowpass(0.5 * (Gn * L + En * N) - Fn * M, p, filter_freq)
    K = lowpass((L * N - M * M) / W2, p, filter_freq)
    return dict(p=p, E=En, F=Fn, G=Gn, W=W, n=n, cu=cu, cv=cv, H=H, K=K, X=X, filter_freq=filter_freq)


def grad(f, geo):
    """Surface gradient of a scalar field [nv][ng] -> [nv][3][ng]."""
    p = geo["p"]
    f = np.asarray(f, dtype=np.float64).reshape(geo["H"].shape)
    S = sh.grid2shc(f.reshape(-1), p, p)
    fu = synth(S, p, "u").reshape(f.shape)
    fv = synth(S, p, "v").reshape(f.shape)
    return lowpass(fu[:, None] * geo["cu"] + fv[:, None] * geo["cv"], p, geo.get("filter_freq"))


def div(Fv, geo):
    """Surface divergence of a vector field [nv][3][ng] -> [nv][ng]."""
    p = geo["p"]
    Fv = np.asarray(Fv, dtype=np.float64).reshape(geo["n"].shape)
    S = sh.grid2shc(Fv.reshape(-1), p, p)
    Fu = synth(S, p, "u").reshape(Fv.shape)
    Fvv = synth(S, p, "v").reshape(Fv.shape)
    return lowpass((Fu * geo["cu"]).sum(1) + (Fvv * geo["cv"]).sum(1), p, geo.get("filter_freq"))


def lin_mean_curv(xn, geo):
    """Linearised mean curvature of the displacement field xn on the current surface."""
    p = geo["p"]
    xn = np.asarray(xn, dtype=np.float64).reshape(geo["n"].shape)
    S = sh.grid2shc(xn.reshape(-1), p, p)
    nrm = geo["n"]
    duu = (synth(S, p, "uu").reshape(xn.shape) * nrm).sum(1)
    duv = (synth(S, p, "uv").reshape(xn.shape) * nrm).sum(1)
    dvv = (synth(S, p, "vv").reshape(xn.shape) * nrm).sum(1)
    return lowpass(0.5 * (geo["G"] * duu - 2.0 * geo["F"] * duv + geo["E"] * dvv), p, geo.get("filter_freq"))


def bending_of(h, geo, kappa):
    """-kappa (Lap_s h + 2 h (H^2 - K)) n  (InterfacialForce::bendingForce / linearBendingForce,
    src/InterfacialForce.cc:21-90, scaled by bending_coeff = -bending_modulus,
    src/VesicleProps.cc:39-41): with the outward normal and H = -1/R on a sphere this is the
    restoring traction, which lowers the bending energy of a relaxing vesicle."""
    lap = div(grad(h, geo), geo)
    s = lap + 2.0 * h * (geo["H"] ** 2 - geo["K"])
    return -kappa * s[:, None] * geo["n"]


def bending_force(geo, kappa):
    return bending_of(geo["H"], geo, kappa)


def lin_bending_force(xn, geo, kappa):
    return bending_of(lin_mean_curv(xn, geo), geo, kappa)


def tensile_force(sigma, geo):
    sigma = np.asarray(sigma, dtype=np.float64).reshape(geo["H"].shape)
    return 2.0 * (geo["H"] * sigma)[:, None] * geo["n"] + grad(sigma, geo)


def gravity_force(x, geo, excess_density, g):
    """Traction jump of gravity, excess_density (g . x) n (InterfacialForce::gravityForce,
    src/InterfacialForce.cc:127-160); x is a vector field [nv][3][ng] (the positions in
    the explicit jump, the displacement in the linearised one)."""
    gx = np.einsum("c,vcn->vn", np.asarray(g, dtype=np.float64), x)
    return excess_density * gx[:, None, :] * geo["n"]


def shear_flow(X, rate):
    """u = (rate * y, 0, 0)."""
    X = np.asarray(X).reshape(-1, 3, X.size // 3 if X.ndim == 1 else X.shape[-1])
    u = np.zeros_like(X)
    u[:, 0] = rate * X[:, 1]
    return u


class ImplicitStep:
    """Globally implicit step solving for the velocity (pseudospectral form):
        u - S[f(dt u, sigma)] = u_inf + S[f_b(x)],     -div S[f] = div(u_inf + S[f_b])
    with f(y, sigma) = lin_bending(y) + tension(sigma).

    With a viscosity contrast lambda (scalar or per vesicle; VesicleProps.cc:27-49) the
    operator becomes (ImplicitApply, src/InterfacialVelocity.cc:934-966)
        (1 + lambda)/2 u - S[f] - D[(1 - lambda) u],   -div(S[f] + D[(1 - lambda) u])
    and the right-hand side is unchanged (AssembleRhsVel, :717-745)."""

    def __init__(self, X, p, kappa, dt, shear_rate, SL=None, excess_density=0.0, gravity=(0.0, 0.0, -1.0),
                 filter_freq=None, viscosity_contrast=None):
        self.p = p
        self.X = np.asarray(X, dtype=np.float64)
        self.geo = geometry(self.X, p, filter_freq)
        self.kappa, self.dt, self.rate = kappa, dt, shear_rate
        self.drho, self.g = excess_density, np.asarray(gravity, dtype=np.float64)
        self.SL = SL if SL is not None else sh.stokes_singular_matrix(self.X, p, 2 * p)
        self.nv, _, self.ng = self.geo["n"].shape
        lam = np.broadcast_to(np.asarray(1.0 if viscosity_contrast is None else viscosity_contrast, np.float64),
                              (self.nv,)).copy()
        self.contrast = bool(np.any(np.abs(lam - 1.0) > 1e-12))  # has_contrast (VesicleProps.cc:45-49)
        self.vel_coeff = (0.5 + 0.5 * lam)[:, None, None]
        self.dl_coeff = (1.0 - lam)[:, None, None]
        self._DL = None

    def stokes_dl(self, g):
        if self._DL is None:
            self._DL = sh.stokes_singular_matrix(self.X, self.p, 2 * self.p, single=False)
        return stokes.stokes_velocity_dl(self.X, g.reshape(-1), self.p, DL=self._DL)

    def stokes(self, f):
        return sh.self_apply(self.SL, f.reshape(-1), self.p) + stokes.far_velocity(self.X, f.reshape(-1), self.p)

    def split(self, z):
        nu = self.nv * 3 * self.ng
        return z[:nu].reshape(self.nv, 3, self.ng), z[nu:].reshape(self.nv, self.ng)

    def matvec(self, z):
        u, sig = self.split(z)
        f = lin_bending_force(self.dt * u, self.geo, self.kappa) + tensile_force(sig, self.geo)
        if self.drho:
            f = f + gravity_force(self.dt * u, self.geo, self.drho, self.g)
        Sf = self.stokes(f).reshape(u.shape)
        if self.contrast:
            Sf = Sf + self.stokes_dl(self.dl_coeff * u).reshape(u.shape)
            return np.concatenate([(self.vel_coeff * u - Sf).reshape(-1), (-div(Sf, self.geo)).reshape(-1)])
        return np.concatenate([(u - Sf).reshape(-1), (-div(Sf, self.geo)).reshape(-1)])

    def precond_scales(self):
        """Degree-diagonal spectral preconditioner (ConfigurePrecond, src/InterfacialVelocity.cc:
        664-713): position block 1/|1 - dt n^3| (kept within [1e-10, 1e3], else 1), tension
        block (4n^2-1)(2n+3) / ((n+1)(2n^2+2n-1) n), 1 for n = 0."""
        p = self.p
        deg = np.concatenate([np.arange((jf + 1) // 2, p + 1) for jf in range(2 * p)]).astype(float)
        b = 1.0 / np.abs(1.0 - self.dt * deg ** 3)
        b = np.where(np.abs(b) < 1e3, b, 1.0)
        b = np.where(np.abs(b) > 1e-10, b, 1.0)
        n = np.maximum(deg, 1.0)
        e = (4 * n * n - 1) * (2 * n + 3) / (n + 1) / (2 * n * n + 2 * n - 1) / n
        e = np.where(deg == 0, 1.0, e)
        e = np.where(np.abs(e) > 1e-10, e, 1.0)
        return b, e

    def precond(self, z):
        """SHC2Grid(scale(Grid2SHC(z))) per block (ImplicitPrecond, pseudospectral form,
        src/InterfacialVelocity.cc:1055-1109)."""
        b, e = self.precond_scales()
        p = self.p
        u, sig = self.split(z)
        Su = sh.grid2shc(u.reshape(-1), p, p).reshape(-1, sh.ncoef(p)) * b[None, :]
        Ss = sh.grid2shc(sig.reshape(-1), p, p).reshape(-1, sh.ncoef(p)) * e[None, :]
        return np.concatenate([sh.shc2grid(Su.reshape(-1), p, p), sh.shc2grid(Ss.reshape(-1), p, p)])

    # --- Galerkin form (the reference's default, params.pseudospectral = false): unknowns
    # are SH coefficients; ImplicitApply maps them to the grid, applies the physical
    # matvec and maps back (src/InterfacialVelocity.cc:982-1052).
    def to_grid(self, c):
        nc = sh.ncoef(self.p)
        k = self.nv * 3 * nc
        return np.concatenate([sh.shc2grid(c[:k], self.p, self.p), sh.shc2grid(c[k:], self.p, self.p)])

    def to_coef(self, z):
        u, sig = self.split(z)
        return np.concatenate([sh.grid2shc(u.reshape(-1), self.p, self.p), sh.grid2shc(sig.reshape(-1), self.p, self.p)])

    def matvec_sh(self, c):
        return self.to_coef(self.matvec(self.to_grid(c)))

    def precond_sh(self, c):
        b, e = self.precond_scales()
        return c * np.concatenate([np.tile(b, 3 * self.nv), np.tile(e, self.nv)])

    def solve(self, x0=None, tol=1e-8, max_iter=300, precond=False):
        """BiCGStab on the Galerkin system; returns (grid solution [u; sigma], code, iters, relres)."""
        b = self.to_coef(self.rhs())
        c0 = np.zeros_like(b) if x0 is None else self.to_coef(np.asarray(x0, dtype=np.float64))
        c, code, it, rr = bicgstab(self.matvec_sh, b, c0, tol, max_iter, self.precond_sh if precond else None)
        return self.to_grid(c), code, it, rr

    def rhs(self):
        fb = bending_force(self.geo, self.kappa)
        if self.drho:
            fb = fb + gravity_force(self.X.reshape(self.nv, 3, self.ng), self.geo, self.drho, self.g)
        v = shear_flow(self.X.reshape(self.nv, 3, self.ng), self.rate) + self.stokes(fb).reshape(self.nv, 3, self.ng)
        return np.concatenate([v.reshape(-1), div(v, self.geo).reshape(-1)])


class PolyImplicitStep:
    """The implicit step of a polydisperse suspension: vesicles in runs of equal SH order (the
    grouping of a polydisperse StokesVelocity), forces of each vesicle at its own order, and the
    single layer over every point (each run's self part plus the all-pairs far field across
    runs). Grid vectors are [u (per-vesicle [3][ng_v] blocks); sigma (per-vesicle [ng_v])];
    coefficient vectors are, run after run, [u coefficients; sigma coefficients] of the run
    (the layout of ImplicitStep.to_coef for each run)."""

    def __init__(self, X, orders, kappa, dt, shear_rate, excess_density=0.0, gravity=(0.0, 0.0, -1.0),
                 viscosity_contrast=None):
        X = np.asarray(X, dtype=np.float64).reshape(-1)
        orders = [int(q) for q in orders]
        self.runs = []  # (p, first vesicle, vesicles, first point)
        pt = 0
        for v, q in enumerate(orders):
            if not self.runs or self.runs[-1][0] != q:
                self.runs.append([q, v, 0, pt])
            self.runs[-1][2] += 1
            pt += sh.ngrid(q)
        self.N = pt
        lam = np.broadcast_to(np.asarray(1.0 if viscosity_contrast is None else viscosity_contrast, np.float64),
                              (len(orders),)).copy()
        self.contrast = bool(np.any(np.abs(lam - 1.0) > 1e-12))
        self.steps = [ImplicitStep(X[3 * r[3]:3 * (r[3] + r[2] * sh.ngrid(r[0]))], r[0], kappa, dt, shear_rate,
                                   excess_density=excess_density, gravity=gravity,
                                   viscosity_contrast=lam[r[1]:r[1] + r[2]]) for r in self.runs]
        self.X = X
        self.off = np.concatenate([[0], np.cumsum([sh.ngrid(q) for q in orders])]).astype(np.int64)

    def stokes_dl(self, gs):
        """Double layer of per-run densities gs[r] ([nv][3][ng]) -> per-run velocities: each
        run's DL matrices plus the far double layer over every point of the other vesicles."""
        D = np.concatenate([stokes.far_density(st.X, g.reshape(-1), st.p) for st, g in zip(self.steps, gs)])
        nrm = np.concatenate([stokes.unit_normal(st.X, st.p) for st in self.steps])
        farv = stokes.far_dl(self.X, nrm, D, self.off)
        out = []
        for r, st, g in zip(self.runs, self.steps, gs):
            ng = sh.ngrid(r[0])
            if st._DL is None:
                st._DL = sh.stokes_singular_matrix(st.X, st.p, 2 * st.p, single=False)
            fv = farv[r[3]:r[3] + r[2] * ng].reshape(r[2], ng, 3).transpose(0, 2, 1)
            out.append(sh.self_apply(st._DL, g.reshape(-1), st.p).reshape(r[2], 3, ng) + fv)
        return out

    def stokes(self, fs):
        """Single layer of per-run tractions fs[r] ([nv][3][ng]) -> per-run velocities."""
        D = np.concatenate([stokes.far_density(st.X, f.reshape(-1), st.p) for st, f in zip(self.steps, fs)])
        farv = stokes.far(self.X, D, self.off)  # [N][3]
        out = []
        for r, (st, f) in zip(self.runs, zip(self.steps, fs)):
            ng = sh.ngrid(r[0])
            fv = farv[r[3]:r[3] + r[2] * ng].reshape(r[2], ng, 3).transpose(0, 2, 1)
            out.append(sh.self_apply(st.SL, f.reshape(-1), st.p).reshape(r[2], 3, ng) + fv)
        return out

    def split(self, z):
        us, ss = [], []
        for r in self.runs:
            n = r[2] * sh.ngrid(r[0])
            us.append(z[3 * r[3]:3 * (r[3] + n)].reshape(r[2], 3, -1))
            ss.append(z[3 * self.N + r[3]:3 * self.N + r[3] + n].reshape(r[2], -1))
        return us, ss

    def join(self, us, ss):
        return np.concatenate([np.concatenate([u.reshape(-1) for u in us]), np.concatenate([q.reshape(-1) for q in ss])])

    def matvec(self, z):
        us, ss = self.split(z)
        fs = []
        for st, u, sig in zip(self.steps, us, ss):
            f = lin_bending_force(st.dt * u, st.geo, st.kappa) + tensile_force(sig, st.geo)
            if st.drho:
                f = f + gravity_force(st.dt * u, st.geo, st.drho, st.g)
            fs.append(f)
        Sf = self.stokes(fs)
        if self.contrast:  # (1 + lambda)/2 u - S[f] - D[(1 - lambda) u] over the suspension
            Df = self.stokes_dl([st.dl_coeff * u for st, u in zip(self.steps, us)])
            Sf = [v + w for v, w in zip(Sf, Df)]
            return self.join([st.vel_coeff * u - v for st, u, v in zip(self.steps, us, Sf)],
                             [-div(v, st.geo) for st, v in zip(self.steps, Sf)])
        return self.join([u - v for u, v in zip(us, Sf)], [-div(v, st.geo) for st, v in zip(self.steps, Sf)])

    def rhs(self):
        fs = []
        for st in self.steps:
            fb = bending_force(st.geo, st.kappa)
            if st.drho:
                fb = fb + gravity_force(st.X.reshape(st.nv, 3, st.ng), st.geo, st.drho, st.g)
            fs.append(fb)
        Sf = self.stokes(fs)
        vs = [shear_flow(st.X.reshape(st.nv, 3, st.ng), st.rate) + v for st, v in zip(self.steps, Sf)]
        return self.join(vs, [div(v, st.geo) for st, v in zip(self.steps, vs)])

    def to_coef(self, z):
        us, ss = self.split(z)
        return np.concatenate([st.to_coef(np.concatenate([u.reshape(-1), q.reshape(-1)]))
                               for st, u, q in zip(self.steps, us, ss)])

    def to_grid(self, c):
        us, ss, k = [], [], 0
        for r, st in zip(self.runs, self.steps):
            n = 4 * r[2] * sh.ncoef(r[0])
            g = st.to_grid(c[k:k + n])
            k += n
            us.append(g[:3 * st.nv * st.ng])
            ss.append(g[3 * st.nv * st.ng:])
        return self.join(us, ss)

    def matvec_sh(self, c):
        return self.to_coef(self.matvec(self.to_grid(c)))

    def solve(self, x0=None, tol=1e-8, max_iter=300):
        b = self.to_coef(self.rhs())
        c0 = np.zeros_like(b) if x0 is None else self.to_coef(np.asarray(x0, dtype=np.float64))
        c, code, it, rr = bicgstab(self.matvec_sh, b, c0, tol, max_iter)
        return self.to_grid(c), code, it, rr


def bicgstab(A, b, x0, tol, max_iter, P=None):
    """Preconditioned BiCGStab, the reference's iteration (src/BiCGStab.cc:45-138).
    Returns (x, status, iterations, relres); status 100 success, 101 max iterations,
    102 rho breakdown, 103 omega breakdown, 104 NaN residual (BiCGSReturn)."""
    P = P or (lambda y: y.copy())
    x = x0.copy()
    normb = np.linalg.norm(b)
    normb = 1.0 if normb == 0.0 else normb
    r = b - A(x)
    rt = r.copy()
    resid = np.linalg.norm(r) / normb
    if resid <= tol:
        return x, 100, 0, resid
    rho2 = alpha = omega = 1.0
    p = v = None
    for i in range(1, max_iter + 1):
        if resid != resid:
            return x, 104, i, resid
        rho1 = rt @ r
        if rho1 == 0:
            return x, 102, i, np.linalg.norm(r) / normb
        if i == 1:
            p = r.copy()
        else:
            beta = (rho1 / rho2) * (alpha / omega)
            p = r + beta * (p - omega * v)
        ph = P(p)
        v = A(ph)
        alpha = rho1 / (rt @ v)
        s = r - alpha * v
        resid = np.linalg.norm(s) / normb
        if resid < tol:
            x = x + alpha * ph
            return x, 100, i, resid
        shat = P(s)
        t = A(shat)
        omega = (t @ s) / (t @ t)
        x = x + alpha * ph + omega * shat
        r = s - omega * t
        rho2 = rho1
        resid = np.linalg.norm(r) / normb
        if resid < tol:
            return x, 100, i, resid
        if omega == 0:
            return x, 103, i, np.linalg.norm(r) / normb
    return x, 101, max_iter, resid
