"""The rest of the reference's operator boundary on the GPU: MovePole (include/MovePole.h),
Device<GPU>::AggregateRotation (include/Device.h:234-237), the single-precision
cuda_stokes (src/CudaKernels.cu:751-761) and the Surface mirror, through the C ABI
(ctypes) and through the C++03 mirror (tests/cpp/device_api_test.cc). Checked against the
oracle and against the reference's own precomputed rotations (tests/golden)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from oracle import sh, stokes, surface as su
from tests.helpers import rel_err, small_suspension
from ves3d_b200 import _lib

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "ref_movepole_p6.npz")


def _cuda(a, dtype=np.float64):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def _move_pole(F, p, i, j):
    import torch
    dF = _cuda(F)
    dY = torch.empty_like(dF)
    _lib.check(_lib.lib().ves3d_move_pole(dF.data_ptr(), F.size // (2 * p * (p + 1)), p, int(i), int(j),
                                          dY.data_ptr(), None), "move_pole")
    return dY.cpu().numpy().reshape(F.shape)


def test_move_pole_matches_reference_direct_scheme():
    """The reference's Direct MovePole on its precomputed p = 6 rotations, functions of
    degree < p, targets on both halves of the longitudes (1e-12)."""
    g = dict(np.load(GOLDEN))
    p, F = int(g["p"]), g["F"]
    for (i, j), ref in zip(g["targets"], g["rotated"]):
        assert rel_err(_move_pole(F, p, i, j), ref) < 1e-12


@pytest.mark.parametrize("p", [6, 12, 16])
def test_move_pole_matches_oracle_every_point_at_pole(p):
    """Full band (degree p included) against the oracle's rotation, and the target point at
    the x = -1 pole of the rotated coordinates."""
    X, f = small_suspension(1, p, 90 + p)
    F = np.concatenate([X.reshape(3, -1), f.reshape(3, -1)])
    for i, j in [(0, 0), (p // 2, 1), (p, p - 1), (1, p), (p - 1, 2 * p - 1)]:
        got = _move_pole(F, p, i, j)
        assert rel_err(got, sh.move_pole(F, p, i, j).reshape(F.shape)) < 1e-12
        poles = sh.shc2pole(sh.grid2shc(got[:3].reshape(-1), p, p), p).reshape(3, 2)
        assert np.abs(poles[:, 0] - F[:3, i * 2 * p + j]).max() < 1e-12 * np.abs(F[:3]).max()


def test_move_pole_argument_errors():
    one = _cuda(np.zeros(84))
    L = _lib.lib()
    assert L.ves3d_move_pole(one.data_ptr(), 1, 6, 7, 0, one.data_ptr(), None) == 1  # trg_i > p
    assert L.ves3d_move_pole(one.data_ptr(), 1, 6, 0, 12, one.data_ptr(), None) == 1  # trg_j >= 2p


def test_aggregate_rotation_matches_reference_semantics():
    """Device::AggregateRotation with the reference's latitude-2 rotation: every longitude
    against the restatement of Device<CPU>::AggregateRotation and, for the golden targets of
    that latitude, against the reference's Direct MovePole."""
    import torch
    g = dict(np.load(GOLDEN))
    p, F = int(g["p"]), g["F"]
    npt, nlong, nf = 2 * p * (p + 1), 2 * p, F.shape[0]
    dM, dF = _cuda(g["mat_lat2"]), _cuda(F)
    dR = torch.zeros(nlong * nf * npt, dtype=torch.float64, device="cuda")
    vec = (ctypes.c_void_p * 1)(dF.data_ptr())
    res = (ctypes.c_void_p * nlong)(*[dR.data_ptr() + jj * nf * npt * 8 for jj in range(nlong)])
    n_sub = (ctypes.c_int * 1)(nf)
    _lib.check(_lib.lib().ves3d_dev_aggregate_rotation(p, p + 1, nlong, 1, n_sub, dM.data_ptr(), vec, None, res, 1,
                                                       None), "aggregate_rotation")
    got = dR.cpu().numpy().reshape(nlong, nf, npt)
    assert rel_err(got, sh.aggregate_rotation(g["mat_lat2"], p + 1, nlong, F)) < 1e-13
    for (i, j), ref in zip(g["targets"], g["rotated"]):
        if i == 2:
            assert rel_err(got[j], ref) < 1e-12


def _stokes32(X, f, qw, p, head, tail, use_q=True):
    import torch
    ng = 2 * p * (p + 1)
    nv = X.size // (3 * ng)
    dX, dD = _cuda(X, np.float32), _cuda(f, np.float32)
    dQ = _cuda(qw, np.float32) if use_q else None
    dU = torch.zeros(X.size, dtype=torch.float32, device="cuda")
    _lib.check(_lib.lib().ves3d_cuda_stokes_f32(ng, ng, nv, head, tail, dX.data_ptr(), dX.data_ptr(), dD.data_ptr(),
                                                dU.data_ptr(), dQ.data_ptr() if use_q else None, None), "stokes_f32")
    torch.cuda.synchronize()
    return dU.cpu().numpy().astype(np.float64)


def test_cuda_stokes_float_overload():
    """cuda_stokes on float arrays against the FP64 oracle of DirectStokes (FP32 inputs:
    tolerance 2e-6 relative); Q = NULL is unit weights."""
    p = 12
    X, f = small_suspension(2, p, 71)
    ng = 2 * p * (p + 1)
    nv = X.size // (3 * ng)
    qw = sh.smooth_weights_grid(p)
    X32 = X.astype(np.float32).astype(np.float64)
    f32 = f.astype(np.float32).astype(np.float64)
    q32 = qw.astype(np.float32).astype(np.float64)
    got = _stokes32(X, f, qw, p, 0, ng)
    ref = stokes.direct_stokes(ng, ng, nv, 0, ng, q32, X32, X32, f32)
    assert rel_err(got, ref) < 2e-6
    got1 = _stokes32(X, f, qw, p, 5, ng - 3, use_q=False)
    ref1 = stokes.direct_stokes(ng, ng, nv, 5, ng - 3, np.ones(ng), X32, X32, f32)
    assert rel_err(got1, ref1) < 2e-6


# ---- the C++03 mirror ------------------------------------------------------------------
def build_device_api_test(tmpdir):
    exe = os.path.join(str(tmpdir), "device_api_test")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cmd = ["g++", "-std=gnu++03", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(cuda, "include"), os.path.join(ROOT, "tests", "cpp", "device_api_test.cc"), "-o", exe, "-L",
           os.path.join(ROOT, "ves3d_b200"), "-lves3d_b200", "-L", os.path.join(cuda, "lib64"), "-lcudart",
           "-Wl,-rpath," + os.path.join(ROOT, "ves3d_b200")]
    subprocess.check_call(cmd)
    return exe


def _run(exe, mode, tmp_path, payload):
    fin, fout = tmp_path / f"{mode}.in", tmp_path / f"{mode}.out"
    with open(fin, "wb") as fh:
        for part in payload:
            fh.write(part.tobytes())
    subprocess.run([exe, mode, str(fin), str(fout)], check=True)
    return fout


def test_cpp_move_pole_and_aggregate_rotation(tmp_path):
    exe = build_device_api_test(tmp_path)
    g = dict(np.load(GOLDEN))
    p, F = int(g["p"]), g["F"]
    trg = g["targets"].astype(np.int32)
    out = _run(exe, "movepole", tmp_path, [np.array([p, F.shape[0], len(trg)], np.int32), trg.ravel(), F])
    got = np.fromfile(out, dtype=np.float64).reshape(len(trg), *F.shape)
    assert rel_err(got, g["rotated"]) < 1e-12
    out = _run(exe, "aggregate", tmp_path, [np.array([p, F.shape[0]], np.int32), g["mat_lat2"], F])
    got = np.fromfile(out, dtype=np.float64).reshape(2 * p, *F.shape)
    assert rel_err(got, sh.aggregate_rotation(g["mat_lat2"], p + 1, 2 * p, F)) < 1e-13


def test_cpp_direct_stokes_float(tmp_path):
    exe = build_device_api_test(tmp_path)
    p = 8
    X, f = small_suspension(2, p, 72)
    ng = 2 * p * (p + 1)
    nv = X.size // (3 * ng)
    qw = sh.smooth_weights_grid(p)
    out = _run(exe, "stokes32", tmp_path, [np.array([ng, ng, nv, 0, ng, 1], np.int32), X.astype(np.float32),
                                           X.astype(np.float32), f.astype(np.float32), qw.astype(np.float32)])
    got = np.fromfile(out, dtype=np.float32).astype(np.float64)
    c = lambda a: a.astype(np.float32).astype(np.float64)  # noqa: E731
    assert rel_err(got, stokes.direct_stokes(ng, ng, nv, 0, ng, c(qw), c(X), c(X), c(f))) < 2e-6


def test_cpp_surface_matches_oracle(tmp_path):
    """Surface's geometry, integrals and differential operators through the C++ mirror."""
    exe = build_device_api_test(tmp_path)
    p = 8
    X, _ = small_suspension(2, p, 73)
    ng = 2 * p * (p + 1)
    nv = X.size // (3 * ng)
    out = _run(exe, "surface", tmp_path, [np.array([p, nv], np.int32), X])
    r = np.fromfile(out, dtype=np.float64)
    sizes = [3 * nv * ng, nv * ng, nv * ng, nv * ng, nv, nv, 3 * nv, 3 * nv * ng, nv * ng, nv * ng]
    parts = np.split(r, np.cumsum(sizes)[:-1])
    geo = su.geometry(X, p)
    area, vol, cen = su.integrals(X, p)
    fx = X.reshape(nv, 3, ng)[:, 0]
    refs = [geo["n"], geo["W"], geo["H"], geo["K"], area, vol, cen, su.grad(fx, geo), su.div(X, geo),
            su.lin_mean_curv(X, geo)]
    for got, ref in zip(parts, refs):
        assert rel_err(got, np.asarray(ref).reshape(-1)) < 1e-11
