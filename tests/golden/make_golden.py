"""Generate the golden fixtures in tests/golden/ from the reference's own CPU code
(oracle/_ref, built from the reference sources by oracle/ref/Makefile). Run in a tree
where the reference is available:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import reflib  # noqa: E402
from ves3d_b200 import workloads  # noqa: E402


def ellipsoid_pair(p):
    x = np.polynomial.legendre.leggauss(p + 1)[0]
    th = np.arccos(x)[:, None]
    ph = (np.pi * np.arange(2 * p) / p)[None, :]
    X = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), 0.5 * np.cos(th) + 0 * ph]).reshape(3, -1)
    return np.concatenate([X, X + np.array([3.0, 0.3, -0.2])[:, None]]).reshape(-1)


def _reference_root():
    """The reference tree, from VES3D_DIR (the variable the reference itself reads)."""
    root = os.environ.get("VES3D_DIR")
    if not root:
        raise SystemExit("set VES3D_DIR to the reference source tree")
    return root


def dumbbell(reference_root=None):
    """The reference's dumbbell test surface (entry 0 of precomputed/shape_gallery_6.txt,
    AxisMajor [3][7][12] at p = 6) and SurfaceTest's known answers for it (area and volume,
    test/SurfaceTest.cc:72, :79; curvature, gradients and Laplacians, :91-116). The
    reference test compares magnitudes (MaxAbs)."""
    reference_root = reference_root or _reference_root()
    vals = []
    with open(os.path.join(reference_root, "precomputed", "shape_gallery_6.txt")) as fh:
        started = False
        for line in fh:
            line = line.strip()
            if line.startswith("#"):
                if started:
                    break
                started = "dumbbell" in line
                continue
            if started and line:
                vals.append(float(line))
    p = 6
    X = np.asarray(vals[: 3 * 2 * p * (p + 1)])
    assert X.size == 3 * 2 * p * (p + 1), X.size
    # test/SurfaceTest.cc:72,79 (area, volume, 5e-8), :91 (max |H|, 8e-8), :98-116 (max |grad|
    # and max |div grad| of the coordinate fields x, y, z, 1e-7), :138-150 (Lap X . n 1e-7,
    # H - Lap X . n / 2 and H + div n / 2, 1e-6); the reference's surface filters at 2p/3
    np.savez_compressed(os.path.join(HERE, "ref_dumbbell_p6.npz"), p=p, X=X, area=16.2179377312307,
                        volume=5.24886489292959, rtol=5e-8, max_abs_H=1.376627062, rtol_H=8e-8,
                        max_abs_grad=np.array([1.01100423438481, 1.011004234384816, 1.004308085588217]),
                        max_abs_lap=np.array([2.239995450856133, 2.239995450856133, 1.777133873450119]),
                        rtol_grad=1e-7, max_abs_lap_dot_n=2.428980517523748,
                        max_abs_H_minus_half_lap_dot_n=0.348685011112687,
                        max_abs_H_plus_half_div_n=0.2437253515, rtol_mixed=1e-6)


def streamable(ref_stream=None):
    """The reference's own Streamable ASCII output (oracle/_ref/ref_stream, built from
    src/Array.cc, Scalars.cc, Vectors.cc by oracle/ref/Makefile): a Vectors of 2 vectors at
    p = 4 and a Scalars, written as its checkpoints are (scientific, 16 digits)."""
    import subprocess
    ref_stream = ref_stream or os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle", "_ref", "ref_stream")
    out = os.path.join(HERE, "ref_stream_p4.txt")
    subprocess.check_call([ref_stream, "pack", "4", "2", out], env=dict(os.environ, VES3D_DIR=_reference_root()))


def double_layer():
    """The reference's double layer: the DL self matrix of vesicle 0 and the DL self velocity
    of two ellipsoids at p = 6 (StokesSingularInteg with DLMatrix), and the far double layer
    of an 8-vesicle p = 6 suspension from DirectStokesDoubleLayerKernel over all points as
    one surface minus its per-vesicle sums, with unit normals from the reference's
    SHC2Grid derivatives and densities times its area element and weights."""
    reflib.set_threads(os.cpu_count() or 1)
    p = 6
    X = ellipsoid_pair(p)
    g = np.random.default_rng(16).standard_normal(X.size)
    _, DL = reflib.singular_matrices(X, p, 2 * p, sl=False, dl=True)
    n = 3 * p * (p + 2)
    vel_self = reflib.self_apply(DL, g, p)
    Xs, _ = workloads.suspension(2, p, 3.0, semi_axes=(1.0, 1.0, 0.6), deg=4, amp=0.05, seed=17)
    gs = np.random.default_rng(18).standard_normal(Xs.size)
    ng = 2 * p * (p + 1)
    nv = Xs.size // (3 * ng)
    _, Xt, Xp = reflib.shc2grid(reflib.grid2shc(Xs, p, p), p, p, grads=True)
    nrm = np.cross(Xt.reshape(nv, 3, ng), Xp.reshape(nv, 3, ng), axis=1)
    nrm = (nrm / np.sqrt((nrm * nrm).sum(axis=1))[:, None, :]).reshape(-1)
    area, qw = reflib.area_weights(Xs, p)
    den = (gs.reshape(nv, 3, ng) * (area.reshape(nv, 1, ng) * qw.reshape(1, 1, ng))).reshape(-1)

    def whole(A):
        return np.ascontiguousarray(A.reshape(nv, 3, ng).transpose(1, 0, 2).reshape(-1))

    allp = reflib.direct_stokes_dl(nv * ng, nv * ng, 1, 0, nv * ng, None, whole(Xs), whole(Xs), whole(nrm), whole(den))
    allp = allp.reshape(3, nv, ng).transpose(1, 0, 2).reshape(-1)
    own = reflib.direct_stokes_dl(ng, ng, nv, 0, ng, None, Xs, Xs, nrm, den)
    np.savez_compressed(os.path.join(HERE, "ref_p6_double_layer.npz"), p=p, X=X, g=g, DL0=DL[: n * n],
                        vel_self=vel_self, Xs=Xs, gs=gs, far_dl=allp - own)


def noise_floor():
    """The reference's own noise floor on the self part, and the p = 24 case: the self
    velocity of the 8-vesicle p = 12 suspension and of one perturbed ellipsoid at p = 24
    (p_up = 48) from the reference built twice, differing only in its GEMM loop order
    (libves3d_ref.so with OpenBLAS, libves3d_ref_naive.so with plain loops). The two
    reference builds disagree at the level of MatRotate's sqrt(1 - x^2) rounding at the
    poles, which is the bar an independent restatement can meet against the reference."""
    reflib.set_threads(os.cpu_count() or 1)
    out = {}
    X, f, p = workloads.make("c1_8ves_p12")
    SL, _ = reflib.singular_matrices(X, p, 2 * p)
    out["c1_vel_self"] = reflib.self_apply(SL, f, p)
    out["c1_vel_self_naive"] = reflib.self_apply(reflib.naive_singular_matrices(X, p, 2 * p), f, p)
    X24, f24 = workloads.suspension(1, 24, 3.0, semi_axes=(1.0, 1.0, 0.6), deg=4, amp=0.05, seed=2424)
    SL, _ = reflib.singular_matrices(X24, 24, 48)
    out["p24_X"], out["p24_f"] = X24, f24
    out["p24_vel_self"] = reflib.self_apply(SL, f24, 24)
    out["p24_vel_self_naive"] = reflib.self_apply(reflib.naive_singular_matrices(X24, 24, 48), f24, 24)
    np.savez_compressed(os.path.join(HERE, "ref_noise_floor_p12_p24.npz"), **out)


def move_pole():
    """The reference's MovePole in its Direct scheme at p = 6 (src/MovePole.cc:166-180:
    rot_mat = CircShift(all_rot_mats[trg_i], trg_j np), results = rot_mat . arr, the gemm in
    column-major BLAS terms) on its own precomputed rotations
    (precomputed/all_rot_mats_6_double.txt), applied to grid functions of degree < p: the
    coordinate functions of a perturbed ellipsoid and three functions of random
    coefficients up to degree p - 1. Also the matrix of latitude 2, for AggregateRotation."""
    from oracle import sh
    p = 6
    npt = 2 * p * (p + 1)
    path = os.path.join(_reference_root(), "precomputed", "all_rot_mats_6_double.txt")
    M = np.loadtxt(path).ravel()[: (p + 1) * npt * npt].reshape(p + 1, npt, npt)  # [lat][col][row]
    X, _ = workloads.suspension(1, p, 3.0, semi_axes=(1.0, 1.0, 0.6), deg=4, amp=0.05, seed=66)
    rng = np.random.default_rng(67)
    S = rng.standard_normal((3, sh.ncoef(p)))
    deg = np.concatenate([np.arange((jf + 1) // 2, p + 1) for jf in range(2 * p)])
    S[:, deg >= p] = 0.0  # degree < p
    F = np.concatenate([X.reshape(3, npt), sh.shc2grid(S.reshape(-1), p, p).reshape(3, npt)])
    lat = np.arange(npt) // (2 * p)
    lon = np.arange(npt) % (2 * p)
    targets = np.array([(0, 0), (2, 3), (2, 9), (5, 5), (3, 11), (6, 2), (1, 7)])
    out = []
    for i, j in targets:
        A = M[i].T  # A[row][col]
        Aj = A[:, lat * 2 * p + (lon - j) % (2 * p)]  # CircShift of the columns per latitude block
        out.append(F @ Aj.T)
    np.savez_compressed(os.path.join(HERE, "ref_movepole_p6.npz"), p=p, F=F, targets=targets,
                        rotated=np.array(out), mat_lat2=M[2].ravel())


def main():
    import sys
    if "--noise-floor" in sys.argv:  # the newest fixtures alone
        noise_floor()
        return
    if "--move-pole" in sys.argv:
        move_pole()
        return
    dumbbell()
    streamable()
    double_layer()
    noise_floor()
    move_pole()
    assert reflib.available(), "build oracle/_ref first (make -C oracle/ref)"
    reflib.set_threads(os.cpu_count() or 1)
    # p = 6: two ellipsoids; quadrature rules, transforms, the self matrix of vesicle 0
    p = 6
    X = ellipsoid_pair(p)
    f = np.random.default_rng(6).standard_normal(X.size)
    SL, _ = reflib.singular_matrices(X, p, 2 * p)
    n = 3 * p * (p + 2)
    S = reflib.grid2shc(X, p, p)
    Xu, Xt, Xp = reflib.shc2grid(S, p, 2 * p, grads=True)
    vel_self = reflib.self_apply(SL, f, p)
    vel_far, _ = reflib.far_sl(X, f, p)
    np.savez_compressed(os.path.join(HERE, "ref_p6_two_ellipsoids.npz"), p=p, X=X, f=f,
                        nodes=reflib.legendre_nodes(p), weights=reflib.legendre_weights(p),
                        sing_weights=reflib.singular_weights(2 * p), shc=S, up=Xu, up_theta=Xt, up_phi=Xp,
                        SL0=SL[: n * n], vel_self=vel_self, vel_far=vel_far)
    # the 8-vesicle p = 12 suspension (seed 1000): full velocity and its far part
    X, f, p = workloads.make("c1_8ves_p12")
    vel, _ = reflib.stokes_velocity_sl(X, f, p, 2 * p)
    far, _ = reflib.far_sl(X, f, p)
    np.savez_compressed(os.path.join(HERE, "ref_c1_8ves_p12.npz"), p=p, X=X, f=f, vel=vel, vel_far=far)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
