"""B-spline shift family on the GPU against the reference (golden vectors from
its own shift.py) and the oracle.  Bound: rel L2 <= 1e-5."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import holo_oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.mark.parametrize("key", ["complex64_a", "complex64_b", "float32_a", "float32_b"])
def test_shift_family_matches_reference(golden, key):
    from holotomocupy_b200 import Shift
    g = golden("shift")
    G = lambda k: torch.from_numpy(g[f"{key}_{k}"]).cuda()
    R = lambda k: g[f"{key}_{k}"]
    n, npsi, nz, nzpsi, nt = [int(v) for v in g[f"{key}_dims"]]
    s = Shift(n, npsi, nz, nzpsi, key.split("_")[0])
    c = s.coeff(G("psi"))
    assert rel_l2(c.cpu().numpy(), R("coeff")) < TOL
    c = torch.from_numpy(R("coeff")).cuda()   # isolate each operator from coeff's rounding
    checks = {
        "S": s.S(c, G("r"), G("m")),
        "Sadj": s.Sadj(G("g"), G("r"), G("m")),
        "curlyS": s.curlyS(G("psi"), G("r"), G("m")),
        "dS": s.dcurlySc(c, G("r"), G("m"), G("c1"), G("d1")),
        "d2S": s.d2curlySc(c, G("r"), G("m"), G("c1"), G("d1"), G("c2"), G("d2")),
    }
    o1, o2 = s.dcurlySadjc(c, G("r"), G("m"), G("g"))
    checks["dSadj1"], checks["dSadj2"] = o1, o2
    for k, v in checks.items():
        v = v.cpu().numpy()
        assert v.shape == R(k).shape and v.dtype == R(k).dtype, k
        assert rel_l2(v, R(k)) < TOL, (k, rel_l2(v, R(k)))


@pytest.mark.parametrize("tag", ["a", "b", "c", "d"])
def test_back_projection_shift_matches_reference(golden, tag):
    """Sback, coeffback, curlySback (shift.py:84-96, 138-153) against the
    reference's outputs and the FP64 oracle.  The back-filter's symbol dips
    to ~0.1 at m = 1.55, so its checks use 1e-5 against the FP32 reference
    and the same bound against FP64."""
    from holotomocupy_b200 import Shift
    g = golden("sback")
    R = lambda k: g[f"sb_{tag}_{k}"]
    G = lambda k: torch.from_numpy(R(k)).cuda()
    n, npsi, nz, nzpsi, nt = [int(v) for v in R("dims")]
    s = Shift(n, npsi, nz, nzpsi, "complex64")
    o = O.Shift(n, npsi, nz, nzpsi, "complex64", "complex128")
    m = R("m") if R("m").ndim else float(R("m"))
    sb = s.Sback(G("g"), G("r"), m).cpu().numpy()
    assert sb.shape == R("Sback").shape and sb.dtype == np.complex64
    assert rel_l2(sb, R("Sback")) < TOL
    assert rel_l2(sb, o.Sback(R("g"), R("r"), R("m"))) < TOL
    if tag != "d":
        cb = s.coeffback(G("psi"), m).cpu().numpy()
        assert rel_l2(cb, R("coeffback")) < TOL
        assert rel_l2(cb, o.coeffback(R("psi"), R("m"))) < TOL
        csb = s.curlySback(G("g"), G("r"), torch.tensor(R("m")).cuda()).cpu().numpy()
        assert rel_l2(csb, R("curlySback")) < TOL
        assert rel_l2(csb, o.curlySback(R("g"), R("r"), R("m"))) < TOL


@pytest.mark.parametrize("m", [0.001, 0.3, 0.93, 1.0, 2.5, 3.5])
def test_sback_over_magnifications_matches_oracle(m):
    """Sback with one magnification per call from 0.001 (candidate ranges too
    wide for the register-held column taps; the reference's windows then reach
    no cell) to 3.5, shifts of a few pixels, against the FP64 oracle's
    restatement of the reference's scatter (1e-5)."""
    from holotomocupy_b200 import Shift
    rng = np.random.default_rng(int(1000 * m))
    n, npsi, nz, nzpsi, nt = 40, 48, 32, 36, 3
    g = (rng.standard_normal((nt, nz, n)) + 1j * rng.standard_normal((nt, nz, n))).astype("complex64")
    r = rng.uniform(-3, 3, (nt, 2)).astype("float32")
    s = Shift(n, npsi, nz, nzpsi, "complex64")
    o = O.Shift(n, npsi, nz, nzpsi, "complex64", "complex128")
    sb = s.Sback(torch.from_numpy(g).cuda(), torch.from_numpy(r).cuda(), m).cpu().numpy()
    ref = o.Sback(g, r, np.float32(m))
    if not np.any(ref):   # m = 0.001: windows of +-2m reach no cell, in the reference as here
        assert not np.any(sb)
    else:
        # at m = 0.3 a cell takes a few taps of small weight, and FP32 rounding
        # alone puts any FP32 evaluation ~1.5e-5 from FP64 (the FP32 oracle too)
        tol = 5e-5 if m < 0.5 else TOL
        assert rel_l2(sb, ref) < tol, rel_l2(sb, ref)


@pytest.mark.parametrize("mag", [1.0, 0.8, 1.25, 0.0])
def test_adjoint_and_oracle(mag):
    from holotomocupy_b200 import Shift
    n = nz = 96
    npsi = nzpsi = 128
    nt = 3
    rng = np.random.default_rng(int(mag * 100))
    s = Shift(n, npsi, nz, nzpsi, "complex64")
    o = O.Shift(n, npsi, nz, nzpsi, "complex64", "complex64")
    c = (rng.standard_normal((nt, nzpsi, npsi)) + 1j * rng.standard_normal((nt, nzpsi, npsi))).astype("complex64")
    gimg = (rng.standard_normal((nt, nz, n)) + 1j * rng.standard_normal((nt, nz, n))).astype("complex64")
    r = rng.uniform(-5, 5, (nt, 2)).astype("float32")
    m = np.full(nt, mag, "float32")
    ct, gt = torch.from_numpy(c).cuda(), torch.from_numpy(gimg).cuda()
    Sc = s.S(ct, torch.from_numpy(r).cuda(), torch.from_numpy(m).cuda())
    STg = s.Sadj(gt, torch.from_numpy(r).cuda(), torch.from_numpy(m).cuda())
    assert rel_l2(Sc.cpu().numpy(), o.S(c, r, m)) < TOL
    assert rel_l2(STg.cpu().numpy(), o.Sadj(gimg, r, m)) < TOL
    lhs = np.vdot(gimg.astype(np.complex128), Sc.cpu().numpy().astype(np.complex128))
    rhs = np.vdot(STg.cpu().numpy().astype(np.complex128), c.astype(np.complex128))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5
    o1, o2 = s.dcurlySadjc(ct, torch.from_numpy(r).cuda(), torch.from_numpy(m).cuda(), gt)
    p1, p2 = o.dcurlySadjc(c, r, m, gimg)
    assert rel_l2(o1.cpu().numpy(), p1) < TOL
    assert rel_l2(o2.cpu().numpy(), p2) < TOL


def test_coeff_large_against_fp64():
    from holotomocupy_b200 import Shift
    n = 512
    rng = np.random.default_rng(1)
    psi = (rng.standard_normal((2, n, n)) + 1j * rng.standard_normal((2, n, n))).astype("complex64")
    s = Shift(n, n, n, n, "complex64")
    o = O.Shift(n, n, n, n, "complex64", "complex128")
    assert rel_l2(s.coeff(torch.from_numpy(psi).cuda()).cpu().numpy(), o.coeff(psi.astype(np.complex128))) < TOL
