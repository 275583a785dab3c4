"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle on the same
seeded inputs. Tolerance for the plain FP64 form: 1e-12 relative, max-norm."""
import ctypes

import numpy as np
import pytest

from oracle import sh, stokes
from tests.helpers import ellipsoid_pair, rel_err, small_suspension, unit_sphere
from ves3d_b200 import _lib
from ves3d_b200.stokes_velocity import StokesVelocity

pytestmark = pytest.mark.gpu
TOL = 1e-12


def torch_cuda(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("p,p1", [(6, 6), (6, 12), (12, 24), (16, 32), (12, 9)])
def test_sht_forward_backward(p, p1):
    import torch
    rng = np.random.default_rng(p + 7 * p1)
    nf = 7
    X = rng.standard_normal(nf * sh.ngrid(p))
    dX = torch_cuda(X)
    dS = torch.empty(nf * sh.ncoef(p1), dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().ves3d_sht_forward(dX.data_ptr(), nf, p, p1, dS.data_ptr(), None), "fwd")
    assert rel_err(dS.cpu().numpy(), sh.grid2shc(X, p, p1)) < TOL
    if p1 >= p:
        S = rng.standard_normal(nf * sh.ncoef(p))
        dS0 = torch_cuda(S)
        n = nf * sh.ngrid(p1)
        outs = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(3)]
        _lib.check(_lib.lib().ves3d_sht_backward(dS0.data_ptr(), nf, p, p1, *[o.data_ptr() for o in outs], None), "bwd")
        ref = sh.shc2grid(S, p, p1, grads=True)
        for o, r in zip(outs, ref):
            assert rel_err(o.cpu().numpy(), r) < TOL


def test_self_matrix_matches_oracle():
    p = 6
    X = ellipsoid_pair(p)
    with StokesVelocity(p, 2 * p) as sv:
        sv.SetSrcCoord(X)
        SL = sv.self_matrix()
    ref = sh.stokes_singular_matrix(X, p, 2 * p)
    assert rel_err(SL, ref) < TOL


@pytest.mark.parametrize("nside,p,seed", [(1, 6, 1), (2, 6, 2), (2, 12, 3)])
def test_stokes_velocity_matches_oracle(nside, p, seed):
    X, f = small_suspension(nside, p, seed)
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        vel = sv()
        vself, vfar = sv.parts()
    SL = sh.stokes_singular_matrix(X, p, 2 * p)
    ref_self = sh.self_apply(SL, f, p)
    ref_far = stokes.far_velocity(X, f, p)
    assert rel_err(vself, ref_self) < TOL
    if nside > 1:
        assert rel_err(vfar, ref_far) < TOL
    else:
        assert np.abs(vfar).max() == 0.0  # one vesicle: nothing is far
    assert rel_err(vel, ref_self + ref_far) < TOL


def test_c1_config_vs_oracle():
    from ves3d_b200 import workloads
    X, f, p = workloads.make("c1_8ves_p12")
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        vel = sv()
    ref = stokes.stokes_velocity_sl(X, f, p)
    assert rel_err(vel, ref) < TOL


def test_sphere_identity_gpu():
    p = 12
    X = unit_sphere(p)
    f = np.zeros((3, sh.ngrid(p)))
    f[0] = 1.0
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f.reshape(-1))
        v = sv().reshape(3, -1)
    assert np.abs(v[0] - 2.0 / 3.0).max() < 1e-10
    assert np.abs(v[1:]).max() < 1e-10


def test_device_pointers_and_resident_eval():
    import torch
    p = 6
    X, f = small_suspension(2, p, 9)
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(torch_cuda(X))
        sv.SetDensitySL(torch_cuda(f))
        out = torch.empty(X.size, dtype=torch.float64, device="cuda")
        sv(out)
        host = sv()
    assert np.array_equal(out.cpu().numpy(), host)
    assert rel_err(host, stokes.stokes_velocity_sl(X, f, p)) < TOL


def test_repeated_eval_is_deterministic():
    p = 6
    X, f = small_suspension(2, p, 11)
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        a = sv()
        b = sv()
        sv.SetDensitySL(2.0 * f)
        c = sv()
    assert np.array_equal(a, b)
    assert rel_err(c, 2.0 * a) < 1e-14


def test_cuda_stokes_matches_direct_stokes():
    rng = np.random.default_rng(3)
    ns, src_m, trg_m = 3, 150, 140
    S = rng.standard_normal(3 * ns * src_m)
    T = rng.standard_normal(3 * ns * trg_m)
    D = rng.standard_normal(3 * ns * src_m)
    Q = rng.uniform(0.5, 1.5, src_m)
    dS, dT, dD, dQ = map(torch_cuda, (S, T, D, Q))
    import torch
    dU = torch.zeros(3 * ns * trg_m, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().ves3d_cuda_stokes_f64(src_m, trg_m, ns, 7, 131, dT.data_ptr(), dS.data_ptr(),
                                                  dD.data_ptr(), dU.data_ptr(), dQ.data_ptr(), None), "cuda_stokes")
    torch.cuda.synchronize()
    # oracle with trg stride != src stride: run per surface
    ref = np.zeros((ns, 3, trg_m))
    for v in range(ns):
        Sv = S.reshape(ns, 3, src_m)[v]
        Dv = D.reshape(ns, 3, src_m)[v]
        Tv = T.reshape(ns, 3, trg_m)[v]
        for t in range(7, 131):
            r = Sv - Tv[:, t:t + 1]
            d = Dv * Q
            rr = np.sqrt((r * r).sum(0))
            cc = (r * d).sum(0) / rr ** 2
            ref[v, :, t] = ((d + cc * r) / rr).sum(1) / (8 * np.pi)
    assert rel_err(dU.cpu().numpy(), ref.reshape(-1)) < TOL


def test_interaction_handle_matches_alltoall():
    rng = np.random.default_rng(4)
    np_ = 517
    src = rng.standard_normal(3 * np_)
    den = rng.standard_normal(3 * np_)
    src[9:12] = src[0:3]
    pot = np.empty(3 * np_)
    ctx = ctypes.c_void_p()
    L = _lib.lib()
    L.ves3d_stokes_alltoall_f64(src.ctypes.data, den.ctypes.data, np_, pot.ctypes.data, ctypes.byref(ctx))
    L.ves3d_stokes_alltoall_f64(src.ctypes.data, den.ctypes.data, np_, pot.ctypes.data, ctypes.byref(ctx))
    L.ves3d_interaction_free(ctypes.byref(ctx))
    assert ctx.value is None
    assert rel_err(pot, stokes.alltoall(src, den)) < TOL


def test_state_errors():
    with StokesVelocity(6) as sv:
        assert _lib.lib().ves3d_sv_eval(sv._h, None, 0) == 1  # null output: ERR_ARG
        out = np.empty(10)
        assert _lib.lib().ves3d_sv_eval(sv._h, out.ctypes.data, 0) == 4  # no surfaces: ERR_STATE
    with StokesVelocity(6) as sv:
        X, f = small_suspension(1, 6, 1)
        sv.SetSrcCoord(X)
        with pytest.raises(_lib.Ves3dError, match="ERR_STATE"):
            sv()


def test_c1_vs_reference_golden():
    """GPU FP64 against the reference's own output (tests/golden): far part to the 1e-12
    bar of the plain form, full velocity within the reference's self-part noise floor."""
    import os
    g = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_c1_8ves_p12.npz")))
    p = int(g["p"])
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(g["X"])
        sv.SetDensitySL(g["f"])
        vel = sv()
        _, far = sv.parts()
    assert rel_err(far, g["vel_far"]) < TOL
    assert rel_err(vel, g["vel"]) < 5e-9


@pytest.mark.parametrize("p", [4, 8, 12, 16])
def test_fused_build_matches_oracle(p):
    """Self matrices from the fused per-rotation build (FP64 tensor cores)."""
    X = ellipsoid_pair(p)
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        SL = sv.self_matrix()
    assert rel_err(SL, sh.stokes_singular_matrix(X, p, 2 * p)) < TOL


def test_fused_equals_unfused(monkeypatch):
    p = 12
    X, f = small_suspension(2, p, 31)
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        A = sv.self_matrix()
    monkeypatch.setenv("VES3D_FUSED_BUILD", "0")
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        B = sv.self_matrix()
    assert rel_err(A, B) < 1e-13


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_captured_eval_graph_matches_eager(precision):
    """The CUDA graph of the resident evaluation, relaunched on new densities written into
    the density buffer, gives bitwise the eager evaluation's self and far parts (every
    reduction runs in a fixed order)."""
    import torch
    p = 8
    X, f = small_suspension(2, p, 71, spacing=2.7)
    rng = np.random.default_rng(3)
    with StokesVelocity(p, precision=precision) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        sv.capture_eval()
        for _ in range(2):
            g = rng.standard_normal(X.size)
            sv.SetDensitySL(torch.from_numpy(g).cuda())  # device copy into the density buffer
            sv.launch_eval_graph()
            torch.cuda.synchronize()
            self_g, far_g = sv.parts()
            vel = sv()  # eager evaluation of the same density
            self_e, far_e = sv.parts()
            assert np.array_equal(self_g, self_e) and np.array_equal(far_g, far_e)
            assert np.allclose(vel, self_e + far_e, rtol=0, atol=1e-14 * np.abs(vel).max())


def test_far_field_autotuner():
    """With the launch-shape autotuner on, the first evaluation times every candidate and
    caches the fastest; results agree with the default shape to rounding and repeat
    bitwise once tuned."""
    p = 8
    X, f = small_suspension(2, p, 72, spacing=2.7)
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        v_default = sv()
        _lib.set_autotune(True)
        try:
            v1 = sv()
            v2 = sv()
            rep = _lib.autotune_report()
        finally:
            _lib.set_autotune(False)
    assert any(k.startswith("f64:N=%d:" % (X.size // 3)) for k in rep), rep
    for e in rep.values():
        assert e["waves"] in (4, 8, 16) and e["threads"] in (256, 384) and e["ms"] > 0
    assert rel_err(v1, v_default) < 1e-13
    assert np.array_equal(v1, v2)


@pytest.mark.parametrize("shape", [(4, 256, 2), (16, 384, 2), (8, 256, 2)])
def test_far_field_launch_shapes_agree(shape):
    """Every launch shape the autotuner may pick (segments, threads per CTA) computes the
    same far field as the default one to rounding, and matches the oracle to 1e-12."""
    p = 8
    X, f = small_suspension(2, p, 73, spacing=2.7)
    with StokesVelocity(p) as sv:
        sv.SetSrcCoord(X)
        sv.SetDensitySL(f)
        v0 = sv()
        _lib.set_far_shape(*shape)
        try:
            sv.SetDensitySL(f)
            v1 = sv()
        finally:
            _lib.set_far_shape(0)
    assert rel_err(v1, v0) < 1e-13
    assert rel_err(v1, stokes.stokes_velocity_sl(X, f, p, 2 * p)) < 1e-12
