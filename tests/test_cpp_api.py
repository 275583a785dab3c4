"""The C++ mirror of the reference API (include/ves3d_b200.hpp) compiles as C++03 against
the C ABI and runs: built here with g++ (CPU), evaluated on the GPU against the oracle."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "ves3d_b200")


def build_api_test(tmpdir):
    exe = os.path.join(str(tmpdir), "api_test")
    cmd = ["g++", "-std=gnu++03", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "api_test.cc"), "-o", exe, "-L", LIBDIR, "-lves3d_b200",
           "-Wl,-rpath," + LIBDIR]
    subprocess.check_call(cmd)
    return exe


def test_cpp_api_builds_as_cpp03_and_links(tmp_path):
    exe = build_api_test(tmp_path)
    out = subprocess.run([exe, "--version"], capture_output=True, text=True, check=True).stdout
    assert int(out.strip()) >= 1


def test_cpp_shtrans_filters_match_oracle(tmp_path):
    """SHTrans's filter coefficients through the C++ mirror (host only) against the oracle,
    with the reference constructor's defaults (filter_freq -1 = 2p/3, exponent 4)."""
    from oracle import sh
    exe = build_api_test(tmp_path)
    for p, freq, e in ((6, -1, 4.0), (12, 5, 2.5), (16, -1, 4.0)):
        out = subprocess.run([exe, "--filter", str(p), str(freq), str(e)], capture_output=True, text=True,
                             check=True).stdout.split("\n")
        hard = np.array(out[0].split(), dtype=float)
        poly = np.array(out[1].split(), dtype=float)
        f_out, e_out = out[2].split()
        assert int(f_out) == (2 * p // 3 if freq == -1 else freq) and float(e_out) == e
        assert np.array_equal(hard, sh.filter_coeffs(p, freq))
        assert np.abs(poly - sh.filter_coeffs(p, freq, e)).max() < 1e-15


@pytest.mark.gpu
def test_cpp_api_matches_oracle(tmp_path):
    from oracle import stokes, surface as su
    from tests.helpers import rel_err, small_suspension
    exe = build_api_test(tmp_path)
    p = 6
    X, f = small_suspension(2, p, 81, spacing=2.7)
    nv = X.size // (3 * 2 * p * (p + 1))
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(fin, "wb") as fh:
        fh.write(np.array([p, nv], dtype=np.int32).tobytes())
        fh.write(X.tobytes())
        fh.write(f.tobytes())
    subprocess.run([exe, str(fin), str(fout)], check=True)
    res = np.fromfile(fout, dtype=np.float64)
    vel, x = res[: X.size], res[X.size:]
    assert rel_err(vel, stokes.stokes_velocity_sl(X, f, p, 2 * p)) < 1e-12
    step = su.ImplicitStep(X, p, 0.05, 0.01, 1.0)
    b = step.to_coef(step.rhs())
    r = b - step.matvec_sh(step.to_coef(x))
    assert np.linalg.norm(r) / np.linalg.norm(b) < 3e-9


def test_cpp_device_api_builds_as_cpp03_and_links(tmp_path):
    """The device-pointer callers (MovePole, AggregateRotation, float DirectStokes, Surface)
    compile as C++03 against the mirror header and link (no GPU needed)."""
    from tests.test_gpu_boundary import build_device_api_test
    assert os.path.exists(build_device_api_test(tmp_path))
