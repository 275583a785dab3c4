"""Learned initial guess of the globally implicit step.

The reference starts each BiCGStab/GMRES solve of the implicit step from the previous
step's solution (InterfacialVelocity::AssembleInitial, src/InterfacialVelocity.cc:874-919).
This module adds a per-vesicle network that predicts the solution [u; sigma] of a vesicle
from its own shape:

    features  SH coefficients of the vesicle's x, y, z with degree 0 removed (3 nc)
    targets   SH coefficients of [u - u_inf; sigma] (4 nc), u_inf = (rate * y, 0, 0)
    network   MLP (BF16 tensor-core training and inference kernels of the library)

The guess that starts the solve is the residual-minimising combination of the candidates
(learned and, when there is one, the previous step's solution), so the true residual of
the solver's own system decides what the network contributes; a useless or broken
network gets weight ~0 and the fallback candidate wins.

Training data come from the method itself: implicit steps of seeded suspensions solved
by the library's BiCGStab (generate_dataset). Weights are stored in a versioned binary
file (LearnedGuess.save / load).
"""
import ctypes
import os
import struct
import time

import numpy as np

from ._lib import check, lib
from .stokes_velocity import StokesVelocity, ncoef


class MLP:
    """x -> [Linear -> ReLU] x (n_layers - 1) -> Linear on the GPU (BF16 operands, FP32
    accumulation and master weights, Adam). Host float32 arrays in and out."""

    def __init__(self, n_in, n_hidden, n_layers, n_out, seed=0):
        h = ctypes.c_void_p()
        check(lib().ves3d_mlp_create(int(n_in), int(n_hidden), int(n_layers), int(n_out), int(seed),
                                     ctypes.byref(h)), "mlp_create")
        self._h = h
        self.n_in, self.n_hidden, self.n_layers, self.n_out = int(n_in), int(n_hidden), int(n_layers), int(n_out)

    @property
    def dims(self):
        return [(self.n_in if l == 0 else self.n_hidden, self.n_out if l == self.n_layers - 1 else self.n_hidden)
                for l in range(self.n_layers)]

    def close(self):
        if getattr(self, "_h", None):
            lib().ves3d_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _f32(a, shape=None):
        a = np.ascontiguousarray(a, dtype=np.float32)
        if shape is not None and a.shape != shape:
            a = a.reshape(shape)
        return a

    def num_params(self):
        return int(lib().ves3d_mlp_num_params(self._h))

    def get_params(self):
        out = np.empty(self.num_params(), dtype=np.float32)
        check(lib().ves3d_mlp_get_params(self._h, out.ctypes.data), "mlp_get_params")
        return out

    def set_params(self, params):
        params = self._f32(params).reshape(-1)
        if params.size != self.num_params():
            raise ValueError("parameter vector has the wrong size")
        check(lib().ves3d_mlp_set_params(self._h, params.ctypes.data), "mlp_set_params")

    def set_scaling(self, in_shift=None, in_scale=None, out_shift=None, out_scale=None):
        arrs = [None if a is None else self._f32(a).reshape(-1) for a in (in_shift, in_scale, out_shift, out_scale)]
        for a, n in zip(arrs, (self.n_in, self.n_in, self.n_out, self.n_out)):
            if a is not None and a.size != n:
                raise ValueError("scaling vector has the wrong size")
        check(lib().ves3d_mlp_set_scaling(self._h, *[None if a is None else a.ctypes.data for a in arrs]),
              "mlp_set_scaling")
        self._keep = arrs

    def forward(self, X):
        X = self._f32(X)
        B = X.shape[0]
        Y = np.empty((B, self.n_out), dtype=np.float32)
        check(lib().ves3d_mlp_forward(self._h, X.ctypes.data, B, Y.ctypes.data, 0), "mlp_forward")
        return Y

    def gradients(self, X, T):
        X, T = self._f32(X), self._f32(T)
        g = np.empty(self.num_params(), dtype=np.float32)
        loss = ctypes.c_double(0)
        check(lib().ves3d_mlp_gradients(self._h, X.ctypes.data, T.ctypes.data, X.shape[0], g.ctypes.data,
                                        ctypes.byref(loss), 0), "mlp_gradients")
        return loss.value, g

    def train_step(self, X, T, lr):
        X, T = self._f32(X), self._f32(T)
        loss = ctypes.c_double(0)
        check(lib().ves3d_mlp_train_step(self._h, X.ctypes.data, T.ctypes.data, X.shape[0], ctypes.c_float(lr),
                                         ctypes.byref(loss), 0), "mlp_train_step")
        return loss.value


MAGIC = b"V3DGUESS"
VERSION = 1
_HEADER = struct.Struct("<8sIIIIIIdddQ")  # magic, version, p, n_in, n_hidden, n_layers, n_out, dt, kappa, rate, n_train


class LearnedGuess:
    """Per-vesicle learned guess for one SH order and one set of implicit-step parameters."""

    def __init__(self, p, dt, kappa, shear_rate, n_hidden=256, n_layers=4, seed=0):
        self.p = int(p)
        self.dt, self.kappa, self.shear_rate = float(dt), float(kappa), float(shear_rate)
        nc = ncoef(self.p)
        self.net = MLP(3 * nc, n_hidden, n_layers, 4 * nc, seed)
        self.scaling = (np.zeros(3 * nc, np.float32), np.ones(3 * nc, np.float32), np.zeros(4 * nc, np.float32),
                        np.ones(4 * nc, np.float32))
        self.n_train = 0

    def close(self):
        self.net.close()

    # ---- persistence -------------------------------------------------------------------
    def save(self, path):
        n = self.net
        with open(path, "wb") as fh:
            fh.write(_HEADER.pack(MAGIC, VERSION, self.p, n.n_in, n.n_hidden, n.n_layers, n.n_out, self.dt,
                                  self.kappa, self.shear_rate, self.n_train))
            for a in self.scaling:
                fh.write(np.ascontiguousarray(a, dtype="<f4").tobytes())
            fh.write(np.ascontiguousarray(n.get_params(), dtype="<f4").tobytes())

    @classmethod
    def load(cls, path):
        with open(path, "rb") as fh:
            raw = fh.read()
        magic, ver, p, n_in, n_hid, n_layers, n_out, dt, kappa, rate, n_train = _HEADER.unpack_from(raw, 0)
        if magic != MAGIC or ver != VERSION:
            raise ValueError(f"{path}: not a version-{VERSION} learned-guess file")
        g = cls(p, dt, kappa, rate, n_hid, n_layers)
        if (g.net.n_in, g.net.n_out) != (n_in, n_out):
            raise ValueError(f"{path}: sizes do not match SH order {p}")
        off = _HEADER.size
        arrs = []
        for n in (n_in, n_in, n_out, n_out):
            arrs.append(np.frombuffer(raw, dtype="<f4", count=n, offset=off).astype(np.float32))
            off += 4 * n
        params = np.frombuffer(raw, dtype="<f4", offset=off).astype(np.float32)
        g.net.set_params(params)
        g.set_scaling(*arrs)
        g.n_train = n_train
        return g

    def set_scaling(self, in_shift, in_scale, out_shift, out_scale):
        self.scaling = tuple(np.asarray(a, np.float32) for a in (in_shift, in_scale, out_shift, out_scale))
        self.net.set_scaling(*self.scaling)

    def matches(self, p, dt, kappa, shear_rate):
        return (self.p == p and np.isclose(self.dt, dt) and np.isclose(self.kappa, kappa)
                and np.isclose(self.shear_rate, shear_rate))

    # ---- training ----------------------------------------------------------------------
    def fit_scaling(self, F, T):
        """Inputs: per-feature mean and 1 / std (std floored at 1e-3 of the largest);
        outputs: per-feature mean, one scale per block (u coefficients, sigma
        coefficients) so the loss weighs coefficients like the solution norm does."""
        nc = ncoef(self.p)
        mu_in = F.mean(0)
        sd_in = F.std(0)
        sd_in = np.maximum(sd_in, 1e-3 * sd_in.max())
        mu_out = T.mean(0)
        sd_out = np.empty(T.shape[1])
        for a, b in ((0, 3 * nc), (3 * nc, 4 * nc)):
            sd_out[a:b] = max(float(np.sqrt(np.mean((T[:, a:b] - mu_out[a:b]) ** 2))), 1e-30)
        self.set_scaling(mu_in, 1.0 / sd_in, mu_out, sd_out)

    def fit(self, F, T, epochs=200, batch=256, lr=1e-3, lr_min=1e-5, seed=0, val=None, log=None):
        """Minibatch Adam with cosine learning-rate decay; returns the loss history."""
        F = np.ascontiguousarray(F, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        self.fit_scaling(F, T)
        rng = np.random.default_rng(seed)
        n = F.shape[0]
        steps_per_epoch = max(1, n // batch)
        total = epochs * steps_per_epoch
        hist = []
        k = 0
        for ep in range(epochs):
            perm = rng.permutation(n)
            acc = 0.0
            for s in range(steps_per_epoch):
                idx = perm[s * batch:(s + 1) * batch]
                cur = lr_min + 0.5 * (lr - lr_min) * (1 + np.cos(np.pi * k / total))
                acc += self.net.train_step(F[idx], T[idx], cur)
                k += 1
            rec = {"epoch": ep, "train_loss": acc / steps_per_epoch}
            if val is not None and (ep % 10 == 9 or ep == epochs - 1):
                rec["val_rel_err"] = self.relative_error(*val)
            hist.append(rec)
            if log and (ep % 10 == 9 or ep == epochs - 1):
                log(rec)
        self.n_train = n
        return hist

    def predict(self, F):
        return self.net.forward(F)

    def relative_error(self, F, T):
        """|prediction - T| / |T| over the whole set (Frobenius)."""
        P = self.predict(F)
        return float(np.linalg.norm(P - T) / max(np.linalg.norm(T), 1e-300))

    # ---- use in the solve --------------------------------------------------------------
    def guess(self, sv):
        """Grid field [u; sigma] predicted for the surfaces currently set on sv."""
        if sv.sh_order != self.p:
            raise ValueError("the network was trained for another SH order")
        return sv.guess_from_targets(self.predict(sv.guess_features()))


def initial_guess(sv, learned=None, previous=None):
    """The guess the implicit solve starts from: the residual-minimising combination of the
    learned guess and the previous step's solution (whichever exist). Returns (x0, info);
    x0 is None when there is no candidate (zero guess)."""
    cands, names = [], []
    if learned is not None:
        t0 = time.perf_counter()
        cands.append(learned.guess(sv))
        names.append("learned")
        t_pred = time.perf_counter() - t0
    if previous is not None:
        cands.append(np.asarray(previous, np.float64))
        names.append("previous")
    if not cands:
        return None, {}
    t0 = time.perf_counter()
    x0, w, r = sv.implicit_combine(cands)
    info = {"candidates": names, "weights": w.tolist(), "relres": dict(zip(names, r[:-1].tolist())),
            "relres_combined": float(r[-1]), "combine_s": time.perf_counter() - t0}
    if learned is not None:
        info["predict_s"] = t_pred
    return x0, info


def generate_dataset(configs, steps, p=16, dt=0.01, kappa=0.05, shear_rate=1.0, tol=1e-7, max_iter=800,
                     device=-1, log=None):
    """Run the implicit method on seeded suspensions and collect (features, targets) per
    vesicle and step. configs: list of workloads.suspension keyword dicts (p is set here).
    Each suspension takes `steps` implicit steps (x += dt u), the first from a zero guess,
    the rest from the previous solution. Returns (F, T, stats)."""
    from . import workloads
    Fs, Ts, stats = [], [], []
    for cfg in configs:
        cfg = dict(cfg, p=p)
        X, _ = workloads.suspension(**cfg)
        N = X.size // 3
        sv = StokesVelocity(p, 2 * p, precision="fp64", device=device)
        sv.set_implicit_params(dt, kappa, shear_rate)
        prev = None
        for k in range(steps):
            sv.SetSrcCoord(X)
            t0 = time.perf_counter()
            x, it, rr, code = sv.implicit_solve(x0=prev, tol=tol, max_iter=max_iter)
            el = time.perf_counter() - t0
            if code != 100:
                raise RuntimeError(f"implicit solve did not converge (code {code}, relres {rr:.2e})")
            Fs.append(sv.guess_features())
            Ts.append(sv.guess_targets(x))
            stats.append({"seed": cfg.get("seed"), "step": k, "iterations": it, "relres": rr, "s": el})
            if log:
                log(stats[-1])
            X = X + dt * x[:3 * N]
            prev = x
        sv.close()
    return np.concatenate(Fs), np.concatenate(Ts), stats


# ---- the C4 network: training on the method's own solves, evaluation -------------------
C4_PARAMS = dict(p=16, dt=0.01, kappa=0.05, shear_rate=1.0)
# training suspensions: the 256-vesicle workload's distribution (spheres + deg <= 4 amp 0.05
# perturbations, jittered lattice spacing 2.5) cut to 4 x 4 x 2 lattices, seeds disjoint
# from the workload's
TRAIN_SUSPENSION = dict(nves_side=(4, 4, 2), spacing=2.5, semi_axes=(1.0, 1.0, 1.0), deg=4, amp=0.05, jitter=0.15,
                        min_sep=0.2)
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "guess_c4_p16.bin")


def train_c4(n_systems=48, steps=3, epochs=300, seed0=20000, log=print, out=None):
    """Generate training data with the method (FP64 implicit solves to 1e-7) and fit the
    network; returns (LearnedGuess, report)."""
    cp = C4_PARAMS
    t0 = time.perf_counter()
    cfgs = [dict(TRAIN_SUSPENSION, seed=seed0 + s) for s in range(n_systems)]
    F, T, stats = generate_dataset(cfgs, steps, p=cp["p"], dt=cp["dt"], kappa=cp["kappa"],
                                   shear_rate=cp["shear_rate"], tol=1e-7)
    t_data = time.perf_counter() - t0
    nval = max(1, F.shape[0] // 8)
    g = LearnedGuess(cp["p"], cp["dt"], cp["kappa"], cp["shear_rate"])
    t0 = time.perf_counter()
    hist = g.fit(F[nval:], T[nval:], epochs=epochs, batch=256, lr=1e-3, val=(F[:nval], T[:nval]), log=log)
    t_fit = time.perf_counter() - t0
    rep = {"samples": int(F.shape[0]), "validation_samples": nval, "systems": n_systems, "steps": steps,
           "data_s": t_data, "fit_s": t_fit, "params": g.net.num_params(),
           "solve_iterations_mean": float(np.mean([s["iterations"] for s in stats])),
           "val_rel_err": hist[-1].get("val_rel_err"), "train_loss": hist[-1]["train_loss"],
           "mean_predictor_val_rel_err": float(np.linalg.norm(T[:nval] - T[nval:].mean(0)) / np.linalg.norm(T[:nval]))}
    if out:
        g.save(out)
    return g, rep


def evaluate_steps(learned, X, p, steps=3, precision="fp64", tol=1e-8, max_iter=1000, device=-1, stream=None,
                   timer=None):
    """Implicit steps of suspension X, each solved from four starts: zero (step 1 only),
    previous solution, residual-minimising combination of the previous two solutions
    (no network), and the same plus the learned guess. The trajectory follows the
    previous-guess solution. Returns per-step records."""
    cp = C4_PARAMS
    sv = StokesVelocity(p, 2 * p, precision=precision, device=device)
    if stream is not None:
        sv.set_stream(stream)
    sv.set_implicit_params(cp["dt"], cp["kappa"], cp["shear_rate"])
    N = X.size // 3
    hist = []
    recs = []
    for k in range(steps):
        sv.SetSrcCoord(X)
        rec = {"step": k + 1}
        variants = []
        if not hist:
            variants = [("zero", None), ("learned", "L")]
        else:
            variants = [("previous", "P"), ("previous+history", "PH"), ("previous+history+learned", "PHL")]
        x_next = None
        for name, kind in variants:
            t0 = time.perf_counter()
            tm = timer() if timer else None
            if kind is None:
                x0, info = None, {}
            elif kind == "P":
                x0, info = hist[-1], {}
            else:
                prev = hist[-1] if hist else None
                cands = []
                if "L" in kind:
                    cands.append(learned.guess(sv))
                if prev is not None:
                    cands.append(prev)
                if "H" in kind and len(hist) > 1:
                    cands.append(hist[-2])
                x0, w, r = sv.implicit_combine(cands)
                info = {"weights": [float(v) for v in w], "candidate_relres": [float(v) for v in r[:-1]],
                        "start_relres": float(r[-1])}
            x, it, rr, code = sv.implicit_solve(x0=x0, tol=tol, max_iter=max_iter)
            el = time.perf_counter() - t0
            d = {"iterations": it, "relres": rr, "code": code, "wall_s": el}
            if tm is not None:
                d["device_ms"] = tm()
            if precision == "mixed":
                d["fp64_residual_evaluations"] = sv.solver_stats()["outer"]
            d.update(info)
            rec[name] = d
            if kind in (None, "P"):
                x_next = x
        recs.append(rec)
        hist.append(x_next)
        X = X + cp["dt"] * x_next[:3 * N]
    sv.close()
    return recs


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train / evaluate the learned initial guess of the implicit step")
    ap.add_argument("--systems", type=int, default=48)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--eval-steps", type=int, default=3)
    ap.add_argument("--eval-only", action="store_true")
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)
    from . import workloads
    if a.eval_only:
        g, rep = LearnedGuess.load(a.out), {}
    else:
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        g, rep = train_c4(a.systems, a.steps, a.epochs, log=lambda r: print(json.dumps(r), flush=True), out=a.out)
        print(json.dumps({"training": rep}), flush=True)
    X, _, p = workloads.make("c4_256ves_p16")
    recs = evaluate_steps(g, X, p, steps=a.eval_steps)
    for r in recs:
        print(json.dumps(r), flush=True)
    if a.report:
        with open(a.report, "w") as fh:
            json.dump({"training": rep, "evaluation": recs}, fh, indent=1)


if __name__ == "__main__":
    main()
