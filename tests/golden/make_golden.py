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


def dumbbell(reference_root="/root/reference"):
    """The reference's dumbbell test surface (entry 0 of precomputed/shape_gallery_6.txt,
    AxisMajor [3][7][12] at p = 6) and SurfaceTest's known answers for it
    (test/SurfaceTest.cc:72, :79, relative tolerance 5e-8)."""
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
    np.savez_compressed(os.path.join(HERE, "ref_dumbbell_p6.npz"), p=p, X=X, area=16.2179377312307,
                        volume=5.24886489292959, rtol=5e-8)


def main():
    dumbbell()
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
