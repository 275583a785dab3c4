"""Seeded synthetic suspensions (no datasets are involved).

Shapes follow x(theta, phi) = c + R(theta, phi) * e(theta, phi): e is the unit-sphere
point scaled by the semi-axes, R = scale * (1 + amp * q / max|q|) with
q = sum_{1<=n<=deg} a_nm Y_nm, a_nm ~ U(-1, 1), in the reference's real SH basis
sqrt(2 pi) P_n^m(cos theta) {cos, sin}(m phi). The amplitude is the max-norm of the
relative perturbation, so R stays within scale * [1 - amp, 1 + amp]. Grid: Gauss-Legendre latitudes (ascending cos theta) x uniform
longitudes j*pi/p, i.e. the reference's (p+1) x 2p grid. Densities are i.i.d. N(0,1).
Seeds are 1000 + the configuration index.
"""
import numpy as np


def gl_nodes(p):
    return np.polynomial.legendre.leggauss(p + 1)[0]


def _legendre_all(x, deg):
    """Normalised associated Legendre functions P_n^m(x) for n <= deg, dict[(n, m)]."""
    u = np.sqrt(np.maximum(1.0 - x * x, 0.0))
    P = {}
    pmm = np.full_like(x, 1.0 / np.sqrt(4.0 * np.pi))
    for m in range(deg + 1):
        if m > 0:
            pmm = -pmm * u * np.sqrt((2.0 * m + 1.0) / (2.0 * m))
        P[(m, m)] = pmm
        a_prev, a_cur = np.zeros_like(x), pmm
        for n in range(m + 1, deg + 1):
            a = np.sqrt((2.0 * n - 1) * (2 * n + 1) / ((n - m) * (n + m)))
            b = np.sqrt((2.0 * n + 1) * (n + m - 1) * (n - m - 1) / ((n - m) * (n + m) * (2 * n - 3))) if n > 1 else 0.0
            a_new = x * a * a_cur - b * a_prev
            a_prev, a_cur = a_cur, a_new
            P[(n, m)] = a_new
    return P


def shape(p, center, semi_axes=(1.0, 1.0, 1.0), scale=1.0, deg=4, amp=0.05, rng=None):
    """One vesicle surface, AxisMajor [3][(p+1)*2p]."""
    x = gl_nodes(p)
    th = np.arccos(x)[:, None]
    ph = (np.pi * np.arange(2 * p) / p)[None, :]
    R = np.ones((p + 1, 2 * p))
    if deg > 0 and amp > 0:
        P = _legendre_all(x, deg)
        s2p = np.sqrt(2.0 * np.pi)
        q = np.zeros((p + 1, 2 * p))
        for n in range(1, deg + 1):
            for m in range(0, n + 1):
                q += rng.uniform(-1, 1) * s2p * P[(n, m)][:, None] * np.cos(m * ph)
                if m > 0:
                    q += rng.uniform(-1, 1) * s2p * P[(n, m)][:, None] * np.sin(m * ph)
        R += amp * q / np.abs(q).max()
    a, b, c = semi_axes
    e = np.stack([a * np.sin(th) * np.cos(ph), b * np.sin(th) * np.sin(ph), c * np.cos(th) + 0 * ph])
    X = np.asarray(center, dtype=np.float64)[:, None, None] + scale * R[None] * e
    return X.reshape(3, -1)


def lattice_centers(n, spacing):
    """Centres of an n x n x n (or nx x ny x nz for a tuple n) lattice."""
    nx, ny, nz = (n, n, n) if np.isscalar(n) else n
    axes = [np.arange(k) * spacing for k in (nx, ny, nz)]
    return np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, 3)


def suspension(nves_side, p, spacing, semi_axes=(1.0, 1.0, 1.0), deg=4, amp=0.05, jitter=0.0, min_sep=0.0,
               seed=0):
    """Vesicles on an n^3 lattice (optionally jittered with rejection on min_sep)."""
    rng = np.random.default_rng(seed)
    C = lattice_centers(nves_side, spacing)
    nv = C.shape[0]
    shapes = [shape(p, np.zeros(3), semi_axes, 1.0, deg, amp, rng) for _ in range(nv)]
    if jitter > 0:
        C = C + rng.uniform(-jitter, jitter, size=C.shape)
        if min_sep > 0:
            from scipy.spatial import cKDTree
            for _ in range(50):
                X = np.stack([s + c[:, None] for s, c in zip(shapes, C)])
                pts = X.transpose(0, 2, 1).reshape(-1, 3)
                owner = np.repeat(np.arange(nv), X.shape[2])
                tree = cKDTree(pts)
                pairs = tree.query_pairs(min_sep, output_type="ndarray")
                bad = pairs[owner[pairs[:, 0]] != owner[pairs[:, 1]]]
                if bad.size == 0:
                    break
                offenders = np.unique(owner[bad.ravel()])
                C[offenders] = lattice_centers(nves_side, spacing)[offenders] + rng.uniform(
                    -jitter, jitter, size=(offenders.size, 3)) * 0.5
    X = np.stack([s + c[:, None] for s, c in zip(shapes, C)])
    f = rng.standard_normal(X.shape)
    return np.ascontiguousarray(X.reshape(-1)), np.ascontiguousarray(f.reshape(-1))


CONFIGS = {
    # 8 vesicles, p=12, ellipsoids (1,1,0.5) + deg<=4 amp 0.05 perturbation, 2x2x2 lattice spacing 3.
    "c1_8ves_p12": dict(nves_side=2, p=12, spacing=3.0, semi_axes=(1.0, 1.0, 0.5), deg=4, amp=0.05, seed=1000),
    # 512 vesicles, p=16, unit spheres + deg<=6 amp 0.1, jittered 8x8x8 lattice spacing 2.5, min sep 0.2.
    "c2_512ves_p16": dict(nves_side=8, p=16, spacing=2.5, semi_axes=(1.0, 1.0, 1.0), deg=6, amp=0.1, jitter=0.15,
                          min_sep=0.2, seed=1001),
    # 256 vesicles, p=16, spheres + deg<=4 amp 0.05 on a jittered 8x8x4 lattice: the
    # implicit-step workload (shear u = (y, 0, 0), bending modulus 0.05, dt 0.01).
    "c4_256ves_p16": dict(nves_side=(8, 8, 4), p=16, spacing=2.5, semi_axes=(1.0, 1.0, 1.0), deg=4, amp=0.05,
                          jitter=0.15, min_sep=0.2, seed=1003),
    # 64-vesicle cut of the C2 suspension (4x4x4 lattice): the small case for profiler captures.
    "c2s_64ves_p16": dict(nves_side=4, p=16, spacing=2.5, semi_axes=(1.0, 1.0, 1.0), deg=6, amp=0.1, jitter=0.15,
                          min_sep=0.2, seed=1001),
}


POLYDISPERSE = {
    # 4096 vesicles, p ~ U{8,12,16,24}, radii ~ U[0.7,1.3], SH-perturbed ellipsoids, 20% volume fraction
    "c3_4096ves_poly": dict(n_ves=4096, seed=1002),
    # 2048 vesicles, p ~ U{12,16}, radii ~ U[0.7,1.3], 25% volume fraction: the sedimentation
    # workload (gravity -z, excess density 1, bending modulus 0.05, dt 0.01)
    "c5_2048ves_sed": dict(n_ves=2048, orders=(12, 16), radius=(0.7, 1.3), volume_fraction=0.25, seed=1004),
}


def make(name):
    cfg = dict(CONFIGS[name])
    p = cfg["p"]
    X, f = suspension(**cfg)
    return X, f, p


def poisson_disk_centers(radii, volume_fraction, gap, rng, max_tries=200000):
    """Random sequential addition of non-overlapping spheres (radius r_i + gap/2 each) in a
    cube sized for the given volume fraction of the bare spheres."""
    vol = (4.0 / 3.0) * np.pi * np.sum(np.asarray(radii) ** 3)
    L = (vol / volume_fraction) ** (1.0 / 3.0)
    cell = 2.0 * (np.max(radii) + gap)
    nc = max(1, int(L / cell))
    grid = {}
    centers = np.zeros((len(radii), 3))
    order = np.argsort(-np.asarray(radii))  # place large ones first
    tries = 0
    for i in order:
        r = radii[i]
        while True:
            tries += 1
            if tries > max_tries:
                raise RuntimeError("could not place all spheres; lower the volume fraction")
            c = rng.uniform(r, L - r, size=3)
            key = tuple(np.minimum((c / cell).astype(int), nc - 1))
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        for j in grid.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                            if np.sum((centers[j] - c) ** 2) < (r + radii[j] + gap) ** 2:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                centers[i] = c
                grid.setdefault(key, []).append(i)
                break
    return centers, L


def polydisperse(n_ves, orders=(8, 12, 16, 24), radius=(0.7, 1.3), volume_fraction=0.2, deg=4, amp=0.05,
                 semi_axes=(1.0, 1.0, 0.8), gap=0.2, seed=1002):
    """Vesicles with p ~ U(orders) and radii ~ U(radius); SH-perturbed ellipsoids; centres
    by random sequential addition at the given volume fraction. Returned sorted by order
    (runs of equal p contiguous): (X, f, orders)."""
    rng = np.random.default_rng(seed)
    ps = np.sort(rng.choice(np.asarray(orders), size=n_ves))
    radii = rng.uniform(radius[0], radius[1], size=n_ves)
    ext = radii * (1.0 + amp) * max(semi_axes)
    centers, _ = poisson_disk_centers(ext, volume_fraction * (np.mean(ext ** 3) / np.mean(radii ** 3)), gap, rng)
    Xs, fs = [], []
    for v in range(n_ves):
        Xs.append(shape(int(ps[v]), centers[v], semi_axes, radii[v], deg, amp, rng).reshape(-1))
        fs.append(rng.standard_normal(3 * 2 * ps[v] * (ps[v] + 1)))
    return np.concatenate(Xs), np.concatenate(fs), ps.astype(np.int32)
