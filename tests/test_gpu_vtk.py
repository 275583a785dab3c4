"""GPU: SHC2Pole and WriteVTK, whose surfaces are taken to the output order on the GPU,
against the same files written from the oracle's Grid2SHC / SHC2Grid / SHC2Pole.
Tolerance 1e-12 relative (max-norm) on points and values; the mesh bit for bit."""
import os
import subprocess

import numpy as np
import pytest

from oracle import sh
from tests.helpers import rel_err, small_suspension
from ves3d_b200 import vtk

pytestmark = pytest.mark.gpu
TOL = 1e-12


def oracle_file(path, X, V, p0, p1, period):
    S = sh.grid2shc(X, p0, p0)
    X1, Xp = sh.shc2grid(S, p0, p1), sh.shc2pole(S, p0)
    V1 = Vp = None
    if V is not None:
        T = sh.grid2shc(V, p0, p0)
        V1, Vp = sh.shc2grid(T, p0, p1), sh.shc2pole(T, p0)
    vtk.write_grid(X1, Xp, p1, path, V1, Vp, period=period)
    return vtk.read_vtp(path + "_000000.vtp")


def same_file(a, b):
    assert a["header"] == b["header"]
    assert rel_err(b["points"], a["points"]) < TOL
    if a["value"] is None:
        assert b["value"] is None
    else:
        assert rel_err(b["value"], a["value"]) < TOL
    assert np.array_equal(a["connectivity"], b["connectivity"])
    assert np.array_equal(a["offsets"], b["offsets"])


@pytest.mark.parametrize("p", [2, 6, 12, 16])
def test_shc2pole_matches_oracle(p):
    import torch
    rng = np.random.default_rng(p)
    nf = 11
    S = rng.standard_normal(nf * sh.ncoef(p))
    dP = torch.empty(nf * 2, dtype=torch.float64, device="cuda")
    vtk.SHC2Pole(torch.from_numpy(S).cuda(), p, dP)
    assert rel_err(dP.cpu().numpy(), sh.shc2pole(S, p)) < TOL


@pytest.mark.parametrize("p0,p1,on_device,field,period", [(6, 12, False, True, 0.0), (12, 12, True, True, 2.5),
                                                          (8, 16, True, False, 0.0), (6, 4, False, False, 2.5)])
def test_write_vtk_matches_oracle(tmp_path, p0, p1, on_device, field, period):
    import torch
    X, f = small_suspension(2, p0, p0 + p1)
    V = f if field else None
    ref = oracle_file(str(tmp_path / "ref"), X, V, p0, p1, period)
    S, v = X, V
    if on_device:
        S = torch.from_numpy(X).cuda()
        v = torch.from_numpy(V).cuda() if field else None
    vtk.WriteVTK(S, p0, p1, str(tmp_path / "gpu"), period=period, v=v, rank=0, n_ranks=1)
    same_file(ref, vtk.read_vtp(str(tmp_path / "gpu_000000.vtp")))
    assert vtk.read_pvtp(str(tmp_path / "gpu.pvtp")) == ["gpu_000000.vtp"]


def test_cpp_write_vtk_matches_oracle(tmp_path):
    """The C++ mirror's WriteVTK (host vectors, the reference's signature)."""
    from tests.test_cpp_api import build_api_test
    exe = build_api_test(tmp_path)
    p0, p1 = 6, 12
    X, f = small_suspension(2, p0, 7)
    nv = X.size // (3 * 2 * p0 * (p0 + 1))
    fin = tmp_path / "in.bin"
    with open(fin, "wb") as fh:
        fh.write(np.array([p0, nv], dtype=np.int32).tobytes())
        fh.write(X.tobytes())
        fh.write(f.tobytes())
    subprocess.run([exe, "--vtk", str(fin), str(p1), str(tmp_path / "cpp")], check=True)
    assert os.path.exists(tmp_path / "cpp.pvtp")
    same_file(oracle_file(str(tmp_path / "ref"), X, f, p0, p1, 0.0), vtk.read_vtp(str(tmp_path / "cpp_000000.vtp")))
