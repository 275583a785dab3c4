"""C-ABI library: loads without a GPU, exports every symbol of include/ves3d_b200.h,
and its host-built FP64 tables match the oracle. CPU only (no compute calls)."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import sh
from tests.helpers import rel_err
from ves3d_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "ves3d_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ves3d_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert {s[0] for s in _lib.SIGNATURES} == set(names)


def test_status_without_gpu_is_an_error_not_a_crash():
    from tests.conftest import cuda_available
    if cuda_available():
        pytest.skip("GPU present")
    h = ctypes.c_void_p()
    st = _lib.lib().ves3d_sv_create(12, 24, 0, -1, ctypes.byref(h))
    assert st == 5  # VES3D_ERR_NODEV
    assert b"CUDA" in _lib.lib().ves3d_last_error() or b"device" in _lib.lib().ves3d_last_error()


def test_argument_errors():
    h = ctypes.c_void_p()
    assert _lib.lib().ves3d_sv_create(1, 0, 0, -1, ctypes.byref(h)) == 1
    assert _lib.lib().ves3d_sv_create(12, 6, 0, -1, ctypes.byref(h)) == 1
    assert _lib.lib().ves3d_sv_create(12, 24, 7, -1, ctypes.byref(h)) == 1
    assert _lib.lib().ves3d_sv_eval(None, None, 0) == 1


def test_argument_errors_of_the_implicit_and_filter_entry_points():
    """Null contexts and out-of-range arguments come back as VES3D_ERR_ARG (1) with a
    message, before any device work: the polydisperse implicit step, the guess
    combination, the Surface filter and the SHTrans filters."""
    L = _lib.lib()
    d = ctypes.c_double(1e-8)
    i = ctypes.c_int(10)
    assert L.ves3d_svp_set_implicit_params(None, 0.01, 0.05, 1.0) == 1
    assert L.ves3d_svp_set_gravity(None, 1.0, 0.0, 0.0, -1.0) == 1
    assert L.ves3d_svp_set_precond(None, 2, 1) == 1
    assert L.ves3d_svp_set_surface_filter(None, -1) == 1
    assert L.ves3d_svp_implicit_solve(None, None, None, ctypes.byref(d), ctypes.byref(i), ctypes.byref(i), 0) == 1
    assert L.ves3d_svp_implicit_combine(None, 2, None, None, None, None, 0) == 1
    assert L.ves3d_svp_solver_stats(None, ctypes.byref(i), ctypes.byref(i)) == 1
    assert L.ves3d_sv_set_surface_filter(None, -1) == 1
    out = np.empty(16 * 18)
    assert L.ves3d_sht_filter_coeffs(0, -1, 0.0, out.ctypes.data) == 1
    assert L.ves3d_sht_filter_coeffs(16, -2, 0.0, out.ctypes.data) == 1
    assert L.ves3d_sht_filter_coeffs(16, -1, 0.0, None) == 1
    assert b"coeff" in L.ves3d_last_error()
    assert L.ves3d_sht_lowpass(None, 1, 16, -1, 0.0, None, None) == 1
    assert L.ves3d_sht_backward_d2(None, 1, 6, None, None, None, None) == 1
    assert L.ves3d_sht_backward_d2(out.ctypes.data, 1, 6, None, None, None, None) == 1
    assert L.ves3d_sht_backward_d2(out.ctypes.data, 1, 0, out.ctypes.data, None, None, None) == 1
    assert L.ves3d_sht_scale_freq(None, 1, 16, None, None, None) == 1
    assert L.ves3d_sht_lowpass(out.ctypes.data, -1, 16, -1, 0.0, out.ctypes.data, None) == 1
    # targets, self order and monitor
    assert L.ves3d_sv_set_trg_coord(None, None, 0, 0) == 1
    assert L.ves3d_sv_eval_trg(None, None, 0) == 1
    assert L.ves3d_sv_set_order_up(None, 24) == 1
    assert L.ves3d_sv_monitor_error(None, 1e-6, None, None) == 1
    # double layer and viscosity contrast
    assert L.ves3d_sv_set_viscosity_contrast(None, None, 0) == 1
    assert L.ves3d_sv_set_density_dl(None, None, 0) == 1
    assert L.ves3d_sv_get_dl_matrix(None, None, 0) == 1
    assert L.ves3d_cuda_stokes_double_layer_f64(4, 4, 1, 0, 4, None, None, None, None, None, None, None) == 1
    z = out.ctypes.data
    assert L.ves3d_cuda_stokes_double_layer_f64(4, 4, 1, 0, 5, z, z, z, z, z, None, None) == 1
    assert L.ves3d_cuda_stokes_double_layer_f64(4, 4, 1, 3, 2, z, z, z, z, z, None, None) == 1
    # Device primitives
    assert L.ves3d_dev_axpy(1.0, None, None, 4, None, None) == 1
    assert L.ves3d_dev_transpose(out.ctypes.data, 2, 2, out.ctypes.data, None) == 1
    assert L.ves3d_dev_reduce(None, 0, None, None, 4, 1, None, None) == 1
    assert L.ves3d_dev_gemm(b"X", b"N", 2, 2, 2, 1.0, None, 2, None, 2, 0.0, None, 2, None) == 1
    assert L.ves3d_dev_gemm(b"N", b"N", -1, 2, 2, 1.0, None, 2, None, 2, 0.0, None, 2, None) == 1


@pytest.mark.parametrize("p,p1", [(6, 12), (12, 24), (16, 32)])
def test_host_tables_match_oracle(p, p1):
    T = _lib.tables_export
    assert rel_err(T(p, p1, "nodes0"), sh.legendre_nodes(p)) < 1e-14
    assert rel_err(T(p, p1, "nodes1"), sh.legendre_nodes(p1)) < 1e-14
    assert rel_err(T(p, p1, "smooth_w0"), sh.legendre_weights(p)) < 1e-13
    assert rel_err(T(p, p1, "sing_w"), sh.singular_weights(p1)) < 1e-13
    mr = T(p, p1, "mr")
    blocks = np.concatenate([b.reshape(-1) for b in sh.mat_rotate(p)])
    assert rel_err(mr, blocks) < 1e-13
    # Legendre synthesis tables per coefficient vs the oracle's per-m blocks
    leg = T(p, p1, "syn1_leg").reshape(sh.ncoef(p), p1 + 1)
    Ml = sh.mat_legendre(p, p1)
    rows = []
    for jf in range(2 * p):
        m = (jf + 1) // 2
        rows.append(Ml[m])
    assert rel_err(leg, np.concatenate(rows)) < 1e-13
    four = T(p, p1, "syn1_four").reshape(2 * p, 2 * p1)
    assert rel_err(four, sh.mat_fourier(p, p1)) < 1e-14
