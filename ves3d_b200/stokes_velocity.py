"""Host-side mirror of the reference's StokesVelocity operator contract
(include/StokesVelocity.h:16-44, src/StokesVelocity.cc:11-539), backed by the CUDA
library through its C ABI.

    sv = StokesVelocity(sh_order, sh_order_up)          # StokesVelocity(p, p_up)
    sv.SetSrcCoord(S)                                    # AxisMajor [n_ves][3][(p+1)2p]
    sv.SetDensitySL(f)                                   # same layout
    vel = sv()                                           # operator()()

Arrays are numpy float64 (host) or torch float64 CUDA tensors (device, passed by
pointer without a copy). Errors raise Ves3dError with the library's message.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib


def _ptr(a):
    """(pointer, is_device, n_elems) of a contiguous float64 numpy array or CUDA tensor."""
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise ValueError("expected a C-contiguous float64 array")
        return a.ctypes.data, 0, a.size
    try:
        import torch
    except ImportError:  # pragma: no cover
        torch = None
    if torch is not None and isinstance(a, torch.Tensor):
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise ValueError("expected a contiguous float64 tensor")
        return a.data_ptr(), 1 if a.is_cuda else 0, a.numel()
    raise TypeError(f"unsupported array type {type(a)}")


def ngrid(p):
    return 2 * p * (p + 1)


def ncoef(p):
    return p * (p + 2)


class StokesVelocity:
    """Stokes velocity (single layer, and double layer when a density is set) of a suspension
    of vesicles at their own surface points."""

    def __init__(self, sh_order, sh_order_up=-1, precision="fp64", device=-1):
        prec = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}[precision]
        h = ctypes.c_void_p()
        check(lib().ves3d_sv_create(int(sh_order), int(sh_order_up), prec, int(device), ctypes.byref(h)),
              "StokesVelocity")
        self._h = h
        self.sh_order = int(sh_order)
        self.sh_order_up = int(sh_order_up) if sh_order_up > 0 else 2 * int(sh_order)
        self.n_ves = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().ves3d_sv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- reference API names -------------------------------------------------
    def SetSrcCoord(self, S, sh_order_up_self=-1, sh_order_up=-1):
        if (sh_order_up_self > 0 and sh_order_up_self != self.sh_order_up) or \
                (sh_order_up > 0 and sh_order_up != self.sh_order_up):
            raise ValueError("changing the upsample order needs a new operator")
        p, dev, n = _ptr(S)
        ng = ngrid(self.sh_order)
        if n % (3 * ng):
            raise ValueError(f"surface size {n} is not a multiple of 3*{ng}")
        self.n_ves = n // (3 * ng)
        check(lib().ves3d_sv_set_src_coord(self._h, p, self.n_ves, dev), "SetSrcCoord")

    def SetDensitySL(self, f, add_repul=False):
        if add_repul:
            raise NotImplementedError("repulsion needs the near-singular module, which is not on this path")
        p, dev, n = _ptr(f)
        if n != self.n_ves * 3 * ngrid(self.sh_order):
            raise ValueError("density size does not match the surfaces")
        check(lib().ves3d_sv_set_density_sl(self._h, p, dev), "SetDensitySL")

    def SetDensityDL(self, g):
        """Double-layer density (same layout as the surfaces), or None to turn the double
        layer off; while set, the evaluation adds its velocity."""
        if g is None:
            check(lib().ves3d_sv_set_density_dl(self._h, None, 0), "SetDensityDL")
            return
        p, dev, n = _ptr(g)
        if n != self.n_ves * 3 * ngrid(self.sh_order):
            raise ValueError("density size does not match the surfaces")
        check(lib().ves3d_sv_set_density_dl(self._h, p, dev), "SetDensityDL")

    def __call__(self, out=None):
        if out is None:
            out = np.empty(self.n_ves * 3 * ngrid(self.sh_order))
        p, dev, n = _ptr(out)
        if n != self.n_ves * 3 * ngrid(self.sh_order):
            raise ValueError("output size does not match the surfaces")
        check(lib().ves3d_sv_eval(self._h, p, dev), "StokesVelocity()")
        return out

    # --- extras ----------------------------------------------------------------
    def setup(self):
        check(lib().ves3d_sv_setup(self._h), "setup")

    def self_matrix(self):
        n = 3 * ncoef(self.sh_order)
        out = np.empty((self.n_ves, n, n))
        check(lib().ves3d_sv_get_self_matrix(self._h, out.ctypes.data, 0), "self_matrix")
        return out

    def SetTrgCoord(self, T):
        """Off-surface targets, [M][3] (numpy or CUDA tensor), or None for the surface points.
        eval_targets() returns their velocities (accurate away from the surfaces: no
        near-singular correction)."""
        if T is None:
            check(lib().ves3d_sv_set_trg_coord(self._h, None, 0, 0), "SetTrgCoord")
            self.n_trg = 0
            return
        p, dev, n = _ptr(T)
        if n % 3:
            raise ValueError("targets must be [M][3]")
        check(lib().ves3d_sv_set_trg_coord(self._h, p, n // 3, dev), "SetTrgCoord")
        self.n_trg = n // 3

    def eval_targets(self, out=None):
        if out is None:
            out = np.empty(3 * getattr(self, "n_trg", 0))
        p, dev, n = _ptr(out)
        check(lib().ves3d_sv_eval_trg(self._h, p, dev), "eval_targets")
        return out

    def set_order_up(self, sh_order_up):
        """The self part's upsampling order; the self matrices are rebuilt on next use."""
        check(lib().ves3d_sv_set_order_up(self._h, int(sh_order_up)), "set_order_up")
        self._sync_order()

    def _sync_order(self):
        o = ctypes.c_int()
        check(lib().ves3d_sv_get_order_up(self._h, ctypes.byref(o)), "get_order_up")
        self.sh_order_up = o.value

    def MonitorError(self, tol):
        """StokesVelocity::MonitorError: the double layer of density 1 against its exact value;
        returns (total, [self, near (0), far]) and adapts the self upsampling order."""
        err = np.zeros(3)
        tot = ctypes.c_double()
        check(lib().ves3d_sv_monitor_error(self._h, float(tol), err.ctypes.data, ctypes.byref(tot)), "MonitorError")
        self._sync_order()
        return tot.value, err

    def dl_matrix(self):
        """The double-layer self matrices [n_ves][3 Ncoef][3 Ncoef] (a double-layer density
        must be set)."""
        n = 3 * ncoef(self.sh_order)
        out = np.empty((self.n_ves, n, n))
        check(lib().ves3d_sv_get_dl_matrix(self._h, out.ctypes.data, 0), "dl_matrix")
        return out

    def parts(self):
        n = self.n_ves * 3 * ngrid(self.sh_order)
        a, b = np.empty(n), np.empty(n)
        check(lib().ves3d_sv_get_parts(self._h, a.ctypes.data, b.ctypes.data, 0), "parts")
        return a, b

    def stage_times(self):
        ms = (ctypes.c_float * 4)()
        check(lib().ves3d_sv_stage_times(self._h, ms), "stage_times")
        return {"setup_ms": ms[0], "self_apply_ms": ms[1], "far_ms": ms[2], "eval_ms": ms[3]}

    def set_near_singular(self, on=True):
        """Near-singular correction of the off-surface targets (NearSingular): with it on,
        eval_targets() is accurate up to the surfaces."""
        check(lib().ves3d_sv_set_near_singular(self._h, 1 if on else 0), "set_near_singular")

    def near_info(self):
        """(r_near, number of corrected (target, vesicle) pairs) of the last evaluation."""
        r = ctypes.c_double()
        n = ctypes.c_long()
        check(lib().ves3d_sv_near_info(self._h, ctypes.byref(r), ctypes.byref(n)), "near_info")
        return r.value, n.value

    def far_dl_ms(self):
        """Device ms of the far double layer's kernels in the last evaluation (0 without
        a double-layer density)."""
        ms = ctypes.c_float()
        check(lib().ves3d_sv_far_dl_time(self._h, ctypes.byref(ms)), "far_dl_time")
        return ms.value

    def device_buffer(self, which):
        ptr = ctypes.c_void_p()
        n = ctypes.c_size_t()
        check(lib().ves3d_sv_device_buffer(self._h, int(which), ctypes.byref(ptr), ctypes.byref(n)), "device_buffer")
        return ptr.value, n.value

    def eval_resident(self):
        check(lib().ves3d_sv_eval_resident(self._h), "eval_resident")

    def capture_eval(self):
        """Record the resident evaluation (device density buffer -> device velocity
        buffer) as a CUDA graph; relaunch it with launch_eval_graph()."""
        check(lib().ves3d_sv_capture_eval(self._h), "capture_eval")

    def launch_eval_graph(self):
        """Launch the captured evaluation asynchronously on the context's stream."""
        check(lib().ves3d_sv_launch_eval_graph(self._h), "launch_eval_graph")

    def set_stream(self, stream_ptr):
        check(lib().ves3d_sv_set_stream(self._h, stream_ptr), "set_stream")

    # --- surface geometry, tractions, implicit step ---------------------------------------
    OPS = {"geometry": 0, "grad": 1, "div": 2, "lin_mean_curv": 3, "lin_bending": 4, "bending": 5,
           "tension": 6, "implicit_matvec": 7, "implicit_rhs": 8, "gravity": 9}

    def set_implicit_params(self, dt, kappa, shear_rate):
        check(lib().ves3d_sv_set_implicit_params(self._h, float(dt), float(kappa), float(shear_rate)),
              "set_implicit_params")

    def set_gravity(self, excess_density, g=(0.0, 0.0, -1.0)):
        """Excess density of the vesicles and the gravity field (sedimentation)."""
        check(lib().ves3d_sv_set_gravity(self._h, float(excess_density), *[float(c) for c in g]), "set_gravity")

    def set_viscosity_contrast(self, lam):
        """Viscosity contrast of the implicit step: one value, one per vesicle, or None."""
        if lam is None:
            check(lib().ves3d_sv_set_viscosity_contrast(self._h, None, 0), "set_viscosity_contrast")
            return
        a = np.ascontiguousarray(np.atleast_1d(np.asarray(lam, dtype=np.float64)))
        check(lib().ves3d_sv_set_viscosity_contrast(self._h, a.ctypes.data, a.size), "set_viscosity_contrast")

    def set_surface_filter(self, filter_freq=-1):
        """The reference Surface's low-pass filter on H, K, gradients, divergences and the
        linearised curvature: 0 off (default), -1 degrees <= 2p/3, n > 0 degrees <= n."""
        check(lib().ves3d_sv_set_surface_filter(self._h, int(filter_freq)), "set_surface_filter")

    def surface_op(self, op, field=None):
        ng = ngrid(self.sh_order)
        N = self.n_ves * ng
        sizes = {0: 15 * N, 1: 3 * N, 2: N, 3: N, 4: 3 * N, 5: 3 * N, 6: 3 * N, 7: 4 * N, 8: 4 * N, 9: 3 * N}
        code = self.OPS[op] if isinstance(op, str) else int(op)
        out = np.empty(sizes[code])
        if field is None:
            ptr = None
        else:
            field = np.ascontiguousarray(field, dtype=np.float64).reshape(-1)
            ptr = field.ctypes.data
        check(lib().ves3d_sv_surface_op(self._h, code, ptr, out.ctypes.data, 0), f"surface_op({op})")
        return out

    PRECONDS = {"none": 0, "diag_spectral": 1, "self_block": 2}

    def set_precond(self, scheme):
        """Preconditioner of implicit_solve: "none", "diag_spectral" (the reference's
        ImplicitPrecond) or "self_block" (per-vesicle inverse of the isolated operator)."""
        code = self.PRECONDS[scheme] if isinstance(scheme, str) else int(scheme)
        check(lib().ves3d_sv_set_precond(self._h, code), "set_precond")

    def set_precond_refresh(self, every):
        """Rebuild the preconditioner only every `every` surface updates (lagged
        preconditioner; the solve still meets its tolerance on the true residual)."""
        check(lib().ves3d_sv_set_precond_refresh(self._h, int(every)), "set_precond_refresh")

    def precond_info(self):
        """Device time of the last preconditioner build (total, operator assembly, LU) and
        the bytes the preconditioner holds."""
        ms, nb, age = (ctypes.c_double * 3)(), ctypes.c_size_t(0), ctypes.c_int(0)
        check(lib().ves3d_sv_precond_info(self._h, ms, ctypes.byref(nb), ctypes.byref(age)), "precond_info")
        return {"setup_ms": ms[0], "assembly_ms": ms[1], "factor_ms": ms[2], "bytes": nb.value, "age": age.value}

    def integrals(self):
        """Per vesicle (area, volume, centre [n_ves][3]) of the current surfaces."""
        a, v, c = np.empty(self.n_ves), np.empty(self.n_ves), np.empty((self.n_ves, 3))
        check(lib().ves3d_sv_integrals(self._h, a.ctypes.data, v.ctypes.data, c.ctypes.data, 0), "integrals")
        return a, v, c

    def solver_stats(self):
        o, i = ctypes.c_int(0), ctypes.c_int(0)
        check(lib().ves3d_sv_solver_stats(self._h, ctypes.byref(o), ctypes.byref(i)), "solver_stats")
        return {"outer": o.value, "inner": i.value}

    def implicit_solve(self, x0=None, tol=1e-8, max_iter=200):
        """Solve the implicit system for [u; sigma]; returns (x, iterations, relres, code)."""
        N = self.n_ves * ngrid(self.sh_order)
        x = np.empty(4 * N)
        t = ctypes.c_double(tol)
        it = ctypes.c_int(max_iter)
        code = ctypes.c_int(0)
        p0 = None
        if x0 is not None:
            x0 = np.ascontiguousarray(x0, dtype=np.float64).reshape(-1)
            p0 = x0.ctypes.data
        check(lib().ves3d_sv_implicit_solve(self._h, p0, x.ctypes.data, ctypes.byref(t), ctypes.byref(it),
                                            ctypes.byref(code), 0), "implicit_solve")
        return x, it.value, t.value, code.value

    # ---- initial guesses ---------------------------------------------------------------
    def guess_features(self):
        """[n_ves][3 nc] float32: SH coefficients of the positions, degree 0 removed."""
        out = np.empty((self.n_ves, 3 * ncoef(self.sh_order)), dtype=np.float32)
        check(lib().ves3d_sv_guess_features(self._h, out.ctypes.data, 0), "guess_features")
        return out

    def guess_targets(self, x):
        """[n_ves][4 nc] float32: SH coefficients of [u - u_inf; sigma] of the grid field x."""
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        out = np.empty((self.n_ves, 4 * ncoef(self.sh_order)), dtype=np.float32)
        check(lib().ves3d_sv_guess_targets(self._h, x.ctypes.data, out.ctypes.data, 0), "guess_targets")
        return out

    def guess_from_targets(self, tgt):
        """Grid field [u; sigma] from target coefficients (inverse of guess_targets)."""
        tgt = np.ascontiguousarray(tgt, dtype=np.float32).reshape(-1)
        x0 = np.empty(4 * self.n_ves * ngrid(self.sh_order))
        check(lib().ves3d_sv_guess_from_targets(self._h, tgt.ctypes.data, x0.ctypes.data, 0), "guess_from_targets")
        return x0

    def implicit_combine(self, candidates):
        """Residual-minimising combination of candidate guesses (grid fields [u; sigma]).
        Returns (x0, weights, relres): relres[i] is candidate i's own relative residual,
        relres[-1] that of x0."""
        cands = [np.ascontiguousarray(c, dtype=np.float64).reshape(-1) for c in candidates]
        n = len(cands)
        arr = (ctypes.c_void_p * n)(*[c.ctypes.data for c in cands])
        x0 = np.empty_like(cands[0])
        w = np.zeros(n)
        r = np.zeros(n + 1)
        check(lib().ves3d_sv_implicit_combine(self._h, n, arr, x0.ctypes.data,
                                              w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                              r.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0),
              "implicit_combine")
        return x0, w, r


class SHTrans:
    """SHTrans (include/SHTrans.h:21-63) on CUDA float64 tensors: grid functions
    [n_fun][(p+1) 2p], coefficients function-major [n_fun][p(p+2)]. filter_freq -1 means
    2p/3; filter_exponent is lowPassFilterPoly's exponent (the reference's default 4)."""

    def __init__(self, sh_order, filter_freq=-1, filter_exponent=4.0, stream=None):
        self.p = int(sh_order)
        self.filter_freq = int(filter_freq)
        self.filter_exponent = float(filter_exponent)
        self.stream = stream

    def _nfun(self, t, per):
        p_, dev, n = _ptr(t)
        if not dev or n % per:
            raise ValueError("expected a CUDA float64 tensor of whole functions")
        return p_, n // per

    def forward(self, grid, shc):
        g, n = self._nfun(grid, ngrid(self.p))
        c, _ = self._nfun(shc, ncoef(self.p))
        check(lib().ves3d_sht_forward(g, n, self.p, self.p, c, self.stream), "SHTrans.forward")

    def backward(self, shc, grid):
        c, n = self._nfun(shc, ncoef(self.p))
        g, _ = self._nfun(grid, ngrid(self.p))
        check(lib().ves3d_sht_backward(c, n, self.p, self.p, g, None, None, self.stream), "SHTrans.backward")

    def backward_d2(self, shc, uu=None, vv=None, uv=None):
        """backward_d2u / d2v / duv: second derivatives (u latitude, v longitude) into the
        given grid tensors (any of them None)."""
        c, n = self._nfun(shc, ncoef(self.p))
        outs = []
        for t in (uu, vv, uv):
            if t is None:
                outs.append(None)
            else:
                g, m = self._nfun(t, ngrid(self.p))
                if m != n:
                    raise ValueError("output does not hold one grid function per coefficient vector")
                outs.append(g)
        check(lib().ves3d_sht_backward_d2(c, n, self.p, *outs, self.stream), "SHTrans.backward_d2")

    def ScaleFreq(self, shc_in, scale, shc_out):
        a, n = self._nfun(shc_in, ncoef(self.p))
        b, _ = self._nfun(shc_out, ncoef(self.p))
        sc, _, _ = _ptr(scale)
        check(lib().ves3d_sht_scale_freq(a, n, self.p, sc, b, self.stream), "SHTrans.ScaleFreq")

    def RotateAll(self, shc, out):
        """SphericalHarmonics::RotateAll: vector fields [n][3][p(p+2)] -> every rotation
        [n][p+1][p][3][p(p+2)] (grid point (t, j) to the pole; MovePole's (t, j) slice)."""
        a, n = self._nfun(shc, 3 * ncoef(self.p))
        b, m = self._nfun(out, 3 * ncoef(self.p))
        if m != n * self.p * (self.p + 1):
            raise ValueError("output must hold p(p+1) rotations of every vector field")
        check(lib().ves3d_sht_rotate_all(a, n, self.p, b, self.stream), "SHTrans.RotateAll")

    def lowPassFilter(self, grid_in, grid_out):
        a, n = self._nfun(grid_in, ngrid(self.p))
        b, _ = self._nfun(grid_out, ngrid(self.p))
        check(lib().ves3d_sht_lowpass(a, n, self.p, self.filter_freq, 0.0, b, self.stream), "lowPassFilter")

    def lowPassFilterPoly(self, grid_in, grid_out):
        a, n = self._nfun(grid_in, ngrid(self.p))
        b, _ = self._nfun(grid_out, ngrid(self.p))
        check(lib().ves3d_sht_lowpass(a, n, self.p, self.filter_freq, self.filter_exponent, b, self.stream),
              "lowPassFilterPoly")


class PolydisperseStokesVelocity:
    """Single-layer velocity of a suspension whose vesicles have different SH orders.
    Arrays are the per-vesicle AxisMajor blocks concatenated in vesicle order; vesicles of
    equal order must be contiguous."""

    def __init__(self, precision="fp64", device=-1):
        prec = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}[precision]
        h = ctypes.c_void_p()
        check(lib().ves3d_svp_create(prec, int(device), ctypes.byref(h)), "PolydisperseStokesVelocity")
        self._h = h
        self.orders = None

    def close(self):
        if getattr(self, "_h", None):
            lib().ves3d_svp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def npoints(self):
        return int(sum(ngrid(p) for p in self.orders))

    def SetSrcCoord(self, S, orders):
        self.orders = np.ascontiguousarray(orders, dtype=np.int32)
        p, dev, n = _ptr(S)
        if n != 3 * self.npoints():
            raise ValueError("surface size does not match the orders")
        check(lib().ves3d_svp_set_src_coord(self._h, p, self.orders.ctypes.data, self.orders.size, dev),
              "SetSrcCoord")

    def SetDensitySL(self, f):
        p, dev, n = _ptr(f)
        if n != 3 * self.npoints():
            raise ValueError("density size does not match the surfaces")
        check(lib().ves3d_svp_set_density_sl(self._h, p, dev), "SetDensitySL")

    def SetDensityDL(self, g):
        """Double-layer density (same layout as SetDensitySL), or None to switch it off."""
        if g is None:
            check(lib().ves3d_svp_set_density_dl(self._h, None, 0), "SetDensityDL")
            return
        p, dev, n = _ptr(g)
        if n != 3 * self.npoints():
            raise ValueError("density size does not match the surfaces")
        check(lib().ves3d_svp_set_density_dl(self._h, p, dev), "SetDensityDL")

    def set_viscosity_contrast(self, lam):
        """Viscosity contrast of the implicit step: one value, one per vesicle, or None."""
        if lam is None:
            check(lib().ves3d_svp_set_viscosity_contrast(self._h, None, 0), "set_viscosity_contrast")
            return
        a = np.ascontiguousarray(np.atleast_1d(np.asarray(lam, dtype=np.float64)))
        check(lib().ves3d_svp_set_viscosity_contrast(self._h, a.ctypes.data, a.size), "set_viscosity_contrast")

    def setup(self):
        check(lib().ves3d_svp_setup(self._h), "setup")

    def __call__(self, out=None):
        if out is None:
            out = np.empty(3 * self.npoints())
        p, dev, n = _ptr(out)
        check(lib().ves3d_svp_eval(self._h, p, dev), "StokesVelocity()")
        return out

    def capture_eval(self):
        """Record the evaluation (self parts + far field) as a CUDA graph."""
        check(lib().ves3d_svp_capture_eval(self._h), "capture_eval")

    def launch_eval_graph(self, out=None):
        """Relaunch the captured evaluation (after SetDensitySL with new densities)."""
        if out is None:
            out = np.empty(3 * self.npoints())
        p, dev, n = _ptr(out)
        check(lib().ves3d_svp_launch_eval_graph(self._h, p, dev), "launch_eval_graph")
        return out

    def stage_times(self):
        ms = (ctypes.c_float * 4)()
        check(lib().ves3d_svp_stage_times(self._h, ms), "stage_times")
        return {"setup_ms": ms[0], "self_ms": ms[1], "far_ms": ms[2], "eval_ms": ms[3]}

    # ---- implicit step -----------------------------------------------------------------
    def set_implicit_params(self, dt, kappa, shear_rate):
        check(lib().ves3d_svp_set_implicit_params(self._h, float(dt), float(kappa), float(shear_rate)),
              "set_implicit_params")

    def set_gravity(self, excess_density, g=(0.0, 0.0, -1.0)):
        check(lib().ves3d_svp_set_gravity(self._h, float(excess_density), *[float(c) for c in g]), "set_gravity")

    def set_surface_filter(self, filter_freq=-1):
        check(lib().ves3d_svp_set_surface_filter(self._h, int(filter_freq)), "set_surface_filter")

    def set_precond(self, scheme, refresh_every=1):
        """"none", "diag_spectral" or "self_block" for every order group, rebuilt every
        refresh_every surface updates."""
        code = StokesVelocity.PRECONDS[scheme] if isinstance(scheme, str) else int(scheme)
        check(lib().ves3d_svp_set_precond(self._h, code, int(refresh_every)), "set_precond")

    def solver_stats(self):
        o, i = ctypes.c_int(0), ctypes.c_int(0)
        check(lib().ves3d_svp_solver_stats(self._h, ctypes.byref(o), ctypes.byref(i)), "solver_stats")
        return {"outer": o.value, "inner": i.value}

    def implicit_solve(self, x0=None, tol=1e-8, max_iter=200):
        """Solve the implicit system of the whole suspension for [u; sigma] (u: the
        per-vesicle [3][ng] blocks of all points, then sigma); returns (x, iterations,
        relres, code)."""
        x = np.empty(4 * self.npoints())
        t = ctypes.c_double(tol)
        it = ctypes.c_int(max_iter)
        code = ctypes.c_int(0)
        p0 = None
        if x0 is not None:
            x0 = np.ascontiguousarray(x0, dtype=np.float64).reshape(-1)
            if x0.size != x.size:
                raise ValueError("x0 size does not match the surfaces")
            p0 = x0.ctypes.data
        check(lib().ves3d_svp_implicit_solve(self._h, p0, x.ctypes.data, ctypes.byref(t), ctypes.byref(it),
                                             ctypes.byref(code), 0), "implicit_solve")
        return x, it.value, t.value, code.value

    def implicit_combine(self, candidates):
        """Residual-minimising combination of candidate guesses (grid vectors [u; sigma] of
        the whole suspension), e.g. the last two solutions. Returns (x0, weights, relres)."""
        cands = [np.ascontiguousarray(c, dtype=np.float64).reshape(-1) for c in candidates]
        n = len(cands)
        if any(c.size != 4 * self.npoints() for c in cands):
            raise ValueError("candidate size does not match the surfaces")
        arr = (ctypes.c_void_p * n)(*[c.ctypes.data for c in cands])
        x0 = np.empty_like(cands[0])
        w = np.zeros(n)
        r = np.zeros(n + 1)
        check(lib().ves3d_svp_implicit_combine(self._h, n, arr, x0.ctypes.data,
                                               w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                               r.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0),
              "implicit_combine")
        return x0, w, r
