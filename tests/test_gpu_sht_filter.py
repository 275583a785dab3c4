"""SHTrans's frequency filters and ScaleFreq on the GPU (ves3d_sht_lowpass,
ves3d_sht_scale_freq) against the oracle's restatement (oracle/sh.py low_pass, scale_freq),
FP64, 1e-12 relative; the hard filter is pinned to the reference's dumbbell known answers
through the oracle's curvature and operator tests."""
import numpy as np
import pytest

from oracle import sh
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("p,freq,exponent", [(6, -1, None), (12, -1, 4.0), (16, 9, None), (16, -1, 2.5), (7, 3, 4.0)])
def test_low_pass_matches_oracle(p, freq, exponent):
    import torch
    from ves3d_b200.stokes_velocity import SHTrans
    rng = np.random.default_rng(p * 100 + (freq % 97))
    X = rng.standard_normal(5 * 2 * p * (p + 1))
    ref = sh.low_pass(X, p, freq, exponent)
    sht = SHTrans(p, filter_freq=freq, filter_exponent=exponent or 4.0)
    dX = torch.from_numpy(X).cuda()
    out = torch.empty_like(dX)
    (sht.lowPassFilter if exponent is None else sht.lowPassFilterPoly)(dX, out)
    assert rel_err(out.cpu().numpy(), ref) < 1e-12
    # in place, and a filtered field is a fixed point of the hard filter
    (sht.lowPassFilter if exponent is None else sht.lowPassFilterPoly)(dX, dX)
    assert rel_err(dX.cpu().numpy(), ref) < 1e-12
    if exponent is None:
        again = torch.empty_like(dX)
        sht.lowPassFilter(dX, again)
        assert rel_err(again.cpu().numpy(), ref) < 1e-12


def test_scale_freq_matches_oracle():
    import torch
    from ves3d_b200.stokes_velocity import SHTrans
    p = 12
    rng = np.random.default_rng(3)
    S = rng.standard_normal(4 * p * (p + 2))
    scale = rng.standard_normal(p * (p + 2))
    sht = SHTrans(p)
    dS, dsc = torch.from_numpy(S).cuda(), torch.from_numpy(scale).cuda()
    out = torch.empty_like(dS)
    sht.ScaleFreq(dS, dsc, out)
    assert np.array_equal(out.cpu().numpy(), sh.scale_freq(S, p, scale))


@pytest.mark.parametrize("p", [6, 8, 12])
def test_rotate_all_matches_oracle(p):
    """SphericalHarmonics::RotateAll (the rotation behind MovePole) through the C ABI against
    the oracle's restatement, every rotation of three vector fields, 1e-12 relative."""
    import torch
    from ves3d_b200.stokes_velocity import SHTrans
    rng = np.random.default_rng(p)
    S = rng.standard_normal(3 * 3 * p * (p + 2))
    ref = sh.rotate_all(S, p, 3)
    out = torch.empty(ref.size, dtype=torch.float64, device="cuda")
    SHTrans(p).RotateAll(torch.from_numpy(S).cuda(), out)
    assert rel_err(out.cpu().numpy(), ref) < 1e-12


@pytest.mark.parametrize("p", [6, 12, 16])
def test_second_derivatives_match_oracle(p):
    """ves3d_sht_backward_d2 (SHTrans::backward_d2u / d2v / duv) against the oracle's
    synthesis of second derivatives (oracle/surface.py synth), 1e-12 relative."""
    import torch
    from oracle import surface as su
    from ves3d_b200.stokes_velocity import SHTrans
    rng = np.random.default_rng(p + 3)
    nf = 5
    S = rng.standard_normal(nf * sh.ncoef(p))
    outs = {k: torch.empty(nf * sh.ngrid(p), dtype=torch.float64, device="cuda") for k in ("uu", "vv", "uv")}
    SHTrans(p).backward_d2(torch.from_numpy(S).cuda(), **outs)
    for k, t in outs.items():
        assert rel_err(t.cpu().numpy(), su.synth(S, p, k).reshape(-1)) < 1e-12, k
    only = torch.empty(nf * sh.ngrid(p), dtype=torch.float64, device="cuda")
    SHTrans(p).backward_d2(torch.from_numpy(S).cuda(), vv=only)  # one output alone
    assert torch.equal(only, outs["vv"])
