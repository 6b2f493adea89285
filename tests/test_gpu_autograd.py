"""Differentiable operators (holotomocupy_b200.autograd): the backward passes
are the adjoint kernels; checked against the adjoint identity, against
central finite differences of the FP64 oracle, against the reference's own
BH gradient (golden vectors from rec_mpi.py's gradients_cascade) and against
the fused cascade at 256^3 x 360 angles (and 900 angles in chunks).

Bounds: backward vs adjoint kernel rel <= 1e-6 (same kernels); directional
derivatives vs FP64 central differences (step 1e-3 relative) rel <= 1e-4;
gradients vs the reference rel L2 <= 1e-5; autograd vs fused cascade
rel L2 <= 1e-4 (different FP32 summation orders)."""
import types

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import holo_oracle as O

pytestmark = pytest.mark.gpu


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _args(n, ntheta, ndist, niter=1):
    return types.SimpleNamespace(
        energy=17.1, detector_pixelsize=1.4760147601476e-6 * 2 * 2048 / n, focustodetectordistance=1.217,
        z1=(np.array([5.110, 5.464, 6.879, 9.817]) * 1e-3 + 3.135e-3)[:ndist],
        theta=np.linspace(0, np.pi, ntheta, endpoint=False).astype("float32"), ndist=ndist, ntheta=ntheta,
        nz=n, n=n, nzobj=n, nobj=n, obj_dtype="complex64", mask=0.9, lam_prbfit=0.0, rho=[1, 0.05, 0.02],
        niter=niter, nchunk=max(n, ntheta), vis_step=-1, err_step=-1, start_iter=0)


def _redot(a, b):
    a, b = a.to(torch.complex128), b.to(torch.complex128)
    return float(torch.sum(a.real * b.real + a.imag * b.imag))


def test_linear_backwards_are_the_adjoints():
    from holotomocupy_b200 import Propagation, Tomo
    from holotomocupy_b200.autograd import propagate, radon
    g = torch.Generator(device="cuda").manual_seed(3)
    cn = lambda *s: torch.randn(*s, dtype=torch.complex64, device="cuda", generator=g)
    n = 64
    tomo = Tomo(n, n, np.linspace(0, np.pi, 20, endpoint=False).astype("float32"), 0)
    x = cn(n, n, n).requires_grad_()
    w = cn(20, n, n)
    y = radon(x, tomo)
    (gx,) = torch.autograd.grad(_redot_t(y, w), x)
    assert rel_l2(gx.cpu().numpy(), tomo.RT(w).cpu().numpy()) < 1e-6
    prop = Propagation(n, n, 3, 2, 7.3e-11, 20e-9, [3e-3, 5e-3])
    x = cn(3, n, n).requires_grad_()
    w = cn(3, n, n)
    (gx,) = torch.autograd.grad(_redot_t(propagate(x, 1, prop), w), x)
    assert rel_l2(gx.cpu().numpy(), prop.DT(w, 1).cpu().numpy()) < 1e-6


def _redot_t(a, b):
    return torch.sum(a.real * b.real + a.imag * b.imag)


def test_shift_derivatives_against_fp64_central_differences():
    """d/dh Re<S(coeff(psi + h dpsi); pos + h dpos), w> from the backward pass
    against central differences of the FP64 oracle's curlyS."""
    from holotomocupy_b200 import Shift
    from holotomocupy_b200.autograd import shift
    n, B = 64, 6
    rng = np.random.default_rng(5)
    cn = lambda *s: (rng.standard_normal(s) + 1j * rng.standard_normal(s))
    psi = cn(B, n, n).astype("complex64")
    pos = rng.uniform(-3, 3, (B, 2)).astype("float32")
    mag = rng.uniform(0.9, 1.1, B).astype("float32")
    w = cn(B, n, n).astype("complex64")
    dpsi = cn(B, n, n).astype("complex64")
    dpos = rng.uniform(-1, 1, (B, 2)).astype("float32")
    sh = Shift(n, n, n, n, "complex64")
    tp, tq = cuda(psi).requires_grad_(), cuda(pos).requires_grad_()
    out = shift(tp, tq, cuda(mag), sh)
    gp, gq = torch.autograd.grad(_redot_t(out, cuda(w)), (tp, tq))
    osh = O.Shift(n, n, n, n, "complex64", dtype="complex128")
    f = lambda p, q: float(np.sum((np.conj(w.astype(np.complex128)) * osh.curlyS(p, q, mag.astype(np.float64))).real))
    for name, (d_psi, d_pos) in {"psi": (dpsi, 0 * dpos), "pos": (0 * dpsi, dpos)}.items():
        scale = np.linalg.norm(psi) / np.linalg.norm(d_psi) if name == "psi" else \
            np.linalg.norm(pos) / np.linalg.norm(d_pos)
        h = 1e-3 * scale
        p0, q0 = psi.astype(np.complex128), pos.astype(np.float64)
        fd = (f(p0 + h * d_psi, q0 + h * d_pos) - f(p0 - h * d_psi, q0 - h * d_pos)) / (2 * h)
        an = _redot(gp, cuda(d_psi)) + float(torch.sum(gq.double() * cuda(d_pos).double()))
        assert abs(an / fd - 1) < 1e-4, (name, an, fd)


def _golden_setup(g):
    from holotomocupy_b200.autograd import DataFidelity
    from holotomocupy_b200.rec import Rec
    n, ntheta, ndist, nobj = [int(v) for v in g["c_dims"]]
    rec = Rec(_args(n, ntheta, ndist))
    mag = (1 + rec.shrink_nd) / cuda(rec.norm_magnifications[None, :].astype("float32"))
    return rec, DataFidelity.from_rec(rec), mag.contiguous()


@pytest.mark.parametrize("chunk", [None, 4])
def test_fidelity_gradient_matches_reference_bh_gradient(golden, chunk):
    """Autograd through R-free data term (variable proj) against the
    reference's gradients_cascade on the same inputs (golden vectors)."""
    from holotomocupy_b200.autograd import DataFidelity
    g = golden("rec")
    rec, fid, mag = _golden_setup(g)
    if chunk:
        fid = DataFidelity.from_rec(rec, chunk=chunk)
    prb = cuda(g["c_prb"]).requires_grad_()
    proj = cuda(g["c_proj"]).requires_grad_()
    pos = cuda(g["c_pos"]).requires_grad_()
    F = fid(proj, prb, pos, mag, cuda(g["c_data"]), proj=True)
    assert abs(F.item() / float(g["c_F"]) - 1) < 1e-5
    gprb, gproj, gpos = torch.autograd.grad(F, (prb, proj, pos))
    r = rec.rho_sq
    assert rel_l2((gprb * r["prb"]).cpu().numpy(), g["c_grad_prb"]) < 1e-5
    assert rel_l2((gproj * r["obj"]).cpu().numpy(), g["c_grad_proj"]) < 1e-5
    assert rel_l2((gpos * r["pos"]).cpu().numpy(), g["c_grad_pos"]) < 1e-5


def test_fidelity_directional_derivative_against_fp64_central_differences():
    from holotomocupy_b200.autograd import DataFidelity
    from holotomocupy_b200.rec import Rec
    n, ntheta, ndist = 64, 8, 2
    args = _args(n, ntheta, ndist)
    rec = Rec(args)
    orc = O.Rec(args, "complex128")
    rng = np.random.default_rng(11)
    mag = rng.uniform(0.95, 1.05, (ntheta, ndist)).astype("float32")
    orc.eff_demagnifications[:] = mag
    cn = lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    x = {"prb": (1 + 0.1 * cn(ndist, n, n)).astype("complex64"), "proj": (0.05 * cn(ntheta, n, n)).astype("complex64"),
         "pos": rng.uniform(-3, 3, (ntheta, ndist, 2)).astype("float32")}
    v = {"prb": cn(ndist, n, n).astype("complex64"), "proj": cn(ntheta, n, n).astype("complex64"),
         "pos": rng.uniform(-1, 1, (ntheta, ndist, 2)).astype("float32")}
    data = (np.abs(rng.standard_normal((ntheta, ndist, n, n))) + 0.5).astype("float32")
    fid = DataFidelity.from_rec(rec)
    t = {k: cuda(a).requires_grad_() for k, a in x.items()}
    F = fid(t["proj"], t["prb"], t["pos"], cuda(mag), cuda(data), proj=True)
    gr = dict(zip(("prb", "proj", "pos"), torch.autograd.grad(F, (t["prb"], t["proj"], t["pos"]))))
    d64 = data.astype(np.float64)
    f = lambda y: orc.F0(orc.F1(orc.F2(orc.F3([y["prb"], y["proj"], y["pos"]]))), d64)
    for k in ("prb", "proj", "pos"):
        h = 1e-3 * np.linalg.norm(x[k]) / np.linalg.norm(v[k])
        up = {kk: a.astype(np.complex128 if np.iscomplexobj(a) else np.float64) for kk, a in x.items()}
        dn = dict(up)
        up[k] = up[k] + h * v[k]
        dn[k] = dn[k] - h * v[k]
        fd = (f(up) - f(dn)) / (2 * h)
        an = _redot(gr[k], cuda(v[k])) if k != "pos" else float(torch.sum(gr[k].double() * cuda(v[k]).double()))
        assert abs(an / fd - 1) < 1e-4, (k, an, fd)


def _phantom_problem(n, ntheta, ndist, pos_amp, seed):
    from holotomocupy_b200 import synthetic
    from holotomocupy_b200.rec import Rec
    args = _args(n, ntheta, ndist)
    rec = Rec(args)
    obj = synthetic.ellipsoid_phantom(n, 20, seed)
    prb = synthetic.random_probe(ndist, n, n, seed + 1)
    pos = synthetic.random_positions(ntheta, ndist, pos_amp, seed + 2)
    rec.eff_demagnifications[:] = (1 + rec.shrink_nd) / cuda(rec.norm_magnifications[None, :].astype("float32"))
    g = torch.Generator(device="cuda").manual_seed(seed + 4)
    # phases of ~0.1 rad (100x the phantom's) so that the object term weighs in
    rec.data.copy_(rec.forward_amplitudes(100 * obj, prb, pos))
    x = {"obj": 90 * obj, "prb": torch.ones_like(prb),
         "pos": pos + 0.5 * (2 * torch.rand(pos.shape, generator=g, device="cuda") - 1)}
    synthetic.noisy_amplitudes(rec.data, 1e4, seed + 3)
    return rec, x, rec.data


@pytest.mark.parametrize("ntheta,chunk", [(360, None), (360, 90), (900, 225)])
def test_autograd_matches_fused_cascade_at_256(ntheta, chunk):
    """256^3 object, 4 distances, 256^2 detector, positions +-3 px: the
    composed autograd gradient (object variable, through R) equals the fused
    cascade's (Rec.gradients), with and without angle-chunk recomputation."""
    from holotomocupy_b200.autograd import DataFidelity
    n, ndist = 256, 4
    rec, x, data = _phantom_problem(n, ntheta, ndist, 3.0, 31)
    vars = {"obj": x["obj"], "prb": x["prb"], "pos": x["pos"], "proj": rec.fwd_tomo(x["obj"])}
    grads = {k: torch.zeros_like(v) for k, v in vars.items()}
    rec.gradients(vars, grads)
    fid = DataFidelity.from_rec(rec, chunk=chunk)
    t = {k: x[k].clone().requires_grad_() for k in ("obj", "prb", "pos")}
    F = fid(t["obj"], t["prb"], t["pos"], rec.eff_demagnifications, data)
    gobj, gprb, gpos = torch.autograd.grad(F, (t["obj"], t["prb"], t["pos"]))
    r = rec.rho_sq
    assert rel_l2((gprb * r["prb"]).cpu().numpy(), grads["prb"].cpu().numpy()) < 1e-4
    assert rel_l2((gpos * r["pos"]).cpu().numpy(), grads["pos"].cpu().numpy()) < 1e-4
    assert rel_l2((gobj * r["obj"]).cpu().numpy(), grads["obj"].cpu().numpy()) < 1e-4
