"""The BH cascade and solver on the GPU against the reference (golden vectors
from its own rec_mpi.py), plus derivative (Taylor) checks of the cascade
functions, as in the reference's tests/holotomo3d/test_approximation.ipynb.

Bounds: cascade values rel <= 1e-5 against the reference; BH state after 4
iterations rel L2 <= 1e-5."""
import types

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def rec_args(n, ntheta, ndist, nobj, niter=1):
    return types.SimpleNamespace(
        energy=17.1, detector_pixelsize=1.4760147601476e-6 * 2 * 2048 / n,
        focustodetectordistance=1.217,
        z1=(np.array([5.110, 5.464, 6.879, 9.817]) * 1e-3 + 3.135e-3)[:ndist],
        theta=np.linspace(0, np.pi, ntheta, endpoint=False).astype("float32"),
        ndist=ndist, ntheta=ntheta, nz=n, n=n, nzobj=nobj, nobj=nobj,
        obj_dtype="complex64", mask=0.9, lam_prbfit=0.0, rho=[1, 0.05, 0.02],
        niter=niter, nchunk=max(nobj, ntheta), vis_step=-1, err_step=-1, start_iter=0)


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _cascade_setup(g):
    from holotomocupy_b200.rec import Rec
    n, ntheta, ndist, nobj = [int(v) for v in g["c_dims"]]
    rec = Rec(rec_args(n, ntheta, ndist, nobj))
    np.testing.assert_array_equal(rec.cl_prop.fker.cpu().numpy(), g["c_fker"])
    rec.data[:] = cuda(g["c_data"])
    rec.eff_demagnifications[:] = (1 + rec.shrink_nd) / cuda(rec.norm_magnifications[None, :].astype("float32"))
    v = {"prb": cuda(g["c_prb"]), "proj": cuda(g["c_proj"]), "pos": cuda(g["c_pos"])}
    gr = {k: cuda(g[f"c_g_{k}"]) for k in ("prb", "proj", "pos")}
    et = {k: cuda(g[f"c_e_{k}"]) for k in ("prb", "proj", "pos")}
    return rec, v, gr, et


def test_cascade_matches_reference(golden):
    g = golden("rec")
    rec, v, gr, et = _cascade_setup(g)
    assert abs(rec.min(v["prb"], None, v["pos"], v["proj"]) / float(g["c_F"]) - 1) < TOL
    assert abs(rec.hessian_cascade(v, gr, et) / float(g["c_h_ge"]) - 1) < TOL
    assert abs(rec.hessian_cascade(v, et, et) / float(g["c_h_ee"]) - 1) < TOL
    out = {k: torch.zeros_like(v[k]) for k in v}
    rec.gradients_cascade(v, out)
    for k in ("prb", "proj", "pos"):
        assert rel_l2(out[k].cpu().numpy(), g[f"c_grad_{k}"]) < TOL, k


def test_cascade_functions_match_reference(golden):
    """The operator-by-operator F/gF chain gives the same gradient as the fused pass."""
    g = golden("rec")
    rec, v, gr, et = _cascade_setup(g)
    x = [v["prb"], v["proj"], v["pos"]]
    y = rec.data
    for f in rec.gF:
        y = f(x, y)
    assert rel_l2((y[0] * rec.rho_sq["prb"]).cpu().numpy(), g["c_grad_prb"]) < TOL
    assert rel_l2((y[1] * rec.rho_sq["obj"]).cpu().numpy(), g["c_grad_proj"]) < TOL
    assert rel_l2((y[2] * rec.rho_sq["pos"]).cpu().numpy(), g["c_grad_pos"]) < TOL


def test_symmetric_hessian_is_the_polarised_quadratic_form(golden):
    g = golden("rec")
    rec, v, gr, et = _cascade_setup(g)
    c = rec._coeff_into(v["proj"], torch.empty_like(v["proj"]))
    rec._gradient_pass(c, v["pos"], v["prb"])
    co = lambda p: rec._coeff_into(p.contiguous(), torch.empty_like(p))
    y = (co(gr["proj"]), gr["pos"], gr["prb"])
    z = (co(et["proj"]), et["pos"], et["prb"])
    H = rec._hessian_pass(c, v["pos"], v["prb"], y, z).cpu().numpy()
    s = tuple((a + b).contiguous() for a, b in zip(y, z))
    d = tuple((a - b).contiguous() for a, b in zip(y, z))
    Hs = float(rec._hessian_pass(c, v["pos"], v["prb"], s)[0])
    Hd = float(rec._hessian_pass(c, v["pos"], v["prb"], d)[0])
    assert abs(H[3] - (Hs - Hd) / 4) <= 1e-4 * (abs(Hs) + abs(Hd))
    Hyy = float(rec._hessian_pass(c, v["pos"], v["prb"], y)[0])
    assert abs(H[0] / Hyy - 1) < 1e-6


def test_bh_matches_reference(golden):
    from holotomocupy_b200.rec import Rec
    g = golden("rec")
    n, ntheta, ndist, nobj, niter = [int(v) for v in g["bh_dims"]]
    rec = Rec(rec_args(n, ntheta, ndist, nobj, niter))
    rec.vars["obj"][:] = cuda(g["bh_obj_true"])
    rec.vars["prb"][:] = cuda(g["bh_prb_true"])
    rec.vars["pos"][:] = cuda(g["bh_pos_true"])
    rec.gen_sqrt_data(rec.vars, rec.data)
    assert rel_l2(rec.data.cpu().numpy(), g["bh_data"]) < TOL
    rec.vars["obj"][:] = 0
    rec.vars["prb"][:] = 1
    rec.vars["pos"][:] = cuda(g["bh_pos_true"] + g["bh_pos_err"])
    record = []
    rec.BH(record=record)
    tb = g["bh_topbottom"]
    ref_alpha = [tb[0, 0] / tb[0, 1]] + [tb[2 * i, 0] / tb[2 * i, 1] for i in range(1, niter)]
    ref_beta = [0.0] + [tb[2 * i - 1, 0] / tb[2 * i - 1, 1] for i in range(1, niter)]
    for (i, a, b), ra, rb in zip(record, ref_alpha, ref_beta):
        assert abs(a / ra - 1) < 1e-4, (i, a, ra)
        if rb:
            assert abs(b / rb - 1) < 1e-4, (i, b, rb)
    for k in ("obj", "prb", "pos", "proj"):
        assert rel_l2(rec.vars[k].cpu().numpy(), g[f"bh_{k}"]) < TOL, k


def _taylor(f_w, f_at, df, d2f, L):
    e1, e2, e3 = [], [], []
    for l in L:
        a = f_at(l)
        e1.append(float(torch.linalg.norm(f_w - a)) if torch.is_tensor(a) else abs(f_w - a))
        e2.append(float(torch.linalg.norm(f_w + df(l) - a)) if torch.is_tensor(a) else abs(f_w + df(l) - a))
        e3.append(float(torch.linalg.norm(f_w + df(l) + 0.5 * d2f(l) - a)) if torch.is_tensor(a)
                  else abs(f_w + df(l) + 0.5 * d2f(l) - a))
    return np.array(e1), np.array(e2), np.array(e3)


def test_taylor_orders():
    """tests/holotomo3d/test_approximation.ipynb cells 4-10 of the reference, asserted:
    halving the step divides the first-order residual by ~4 and the
    second-order residual by ~8."""
    from holotomocupy_b200.rec import Rec
    n, ntheta, ndist = 64, 4, 2
    args = rec_args(n, ntheta, ndist, n)
    args.theta = np.linspace(0, np.pi, ntheta).astype("float32")
    rec = Rec(args)
    rec.eff_demagnifications[:] = 1.0
    rng = np.random.default_rng(42)
    rc = lambda s, sc=1.0: cuda(((rng.standard_normal(s) + 1j * rng.standard_normal(s)) * sc).astype("complex64"))
    rf = lambda s, sc=1.0: cuda((rng.standard_normal(s) * sc).astype("float32"))
    prb, proj, pos = rc((ndist, n, n)), rf((ntheta, n, n), 0.1).to(torch.complex64), rf((ntheta, ndist, 2), 0.5)
    dprb, dproj, dpos = rc((ndist, n, n)), rf((ntheta, n, n), 0.1).to(torch.complex64), rf((ntheta, ndist, 2), 0.5)
    L = [0.08, 0.04]   # the reference notebook reads its ratios at steps 0.05-0.08
    # F3
    x3, dx3 = [prb, proj, pos], [dprb, dproj, dpos]
    sc = lambda l: [l * v for v in dx3]
    e1, e2, e3 = _taylor(rec.F3(x3)[1], lambda l: rec.F3([v + d for v, d in zip(x3, sc(l))])[1],
                         lambda l: rec.dF3(x3, sc(l), return_x=False)[1],
                         lambda l: rec.d2F_dF3(x3, sc(l), sc(l), [None] * 3)[1], L)
    assert 3.0 < e2[0] / e2[1] < 5.0 and 6.0 < e3[0] / e3[1] < 10.0
    # F2
    x22, dx22 = rf((ntheta, ndist, n, n), 0.1), rf((ntheta, ndist, n, n), 0.1)
    x2, dx2 = [prb, x22], [dprb, dx22]
    sc = lambda l: [l * v for v in dx2]
    e1, e2, e3 = _taylor(rec.F2(x2)[1], lambda l: rec.F2([v + d for v, d in zip(x2, sc(l))])[1],
                         lambda l: rec.dF2(x2, sc(l), return_x=False)[1],
                         lambda l: rec.d2F_dF2(x2, sc(l), sc(l), [None, None])[1], L)
    assert 3.0 < e2[0] / e2[1] < 5.0 and 6.0 < e3[0] / e3[1] < 10.0
    # F1 (bilinear: the second-order expansion is exact)
    x1 = [rc((ndist, n, n)), rc((ntheta, ndist, n, n))]
    dx1 = [rc((ndist, n, n)), rc((ntheta, ndist, n, n), 0.1)]
    sc = lambda l: [l * v for v in dx1]
    e1, e2, e3 = _taylor(rec.F1(x1), lambda l: rec.F1([v + d for v, d in zip(x1, sc(l))]),
                         lambda l: rec.dF1(x1, sc(l), return_x=False),
                         lambda l: rec.d2F_dF1(x1, sc(l), sc(l), [None, None]), L)
    assert 3.0 < e2[0] / e2[1] < 5.0 and e3[0] < 1e-5 * e1[0]
    # F0
    # F0 is a reduction evaluated in float64: build the perturbed points in float64 too
    data = (torch.abs(rf((ntheta, ndist, n, n))) + 0.1).double()
    # |x| has a kink at 0: keep the expansion point away from it (|x0| ~ 1)
    x0 = (1 + 0.3 * rc((ntheta, ndist, n, n))).to(torch.complex128)
    dx0 = rc((ntheta, ndist, n, n), 0.1).to(torch.complex128)
    e1, e2, e3 = _taylor(rec.F0(x0, data), lambda l: rec.F0(x0 + l * dx0, data),
                         lambda l: rec.dF0(x0, l * dx0, data), lambda l: rec.d2F_dF0(x0, l * dx0, l * dx0, None, data), L)
    assert 3.0 < e2[0] / e2[1] < 5.0 and 6.0 < e3[0] / e3[1] < 10.0


@pytest.mark.parametrize("n,nz", [(64, 64), (384, 384), (512, 512), (768, 96), (1024, 64)])
def test_cascade_at_large_magnifications_matches_oracle(n, nz):
    """Magnifications from 0 to 3.5; rows of n = 64, 384 and 768 samples
    (lines with a radix-3 stage), 512 (the 512-sample rows have their own
    kernels) and 1024, nz detector rows and as many object rows (short images
    at 768 and 1024 keep the FP64 oracle's volumes small).  Gradient and
    Hessian forms against the FP64 oracle (rel <= 1e-4)."""
    from oracle import holo_oracle as O
    from holotomocupy_b200.rec import Rec
    ntheta, ndist = 3, 2
    args = rec_args(n, ntheta, ndist, n)
    args.nz = args.nzobj = nz
    rec = Rec(args)
    orc = O.Rec(args, "complex128")
    eff = np.array([[1.0, 3.5], [0.5, 1.3], [2.9, 0.0]])
    rec.eff_demagnifications[:] = cuda(eff.astype("float32"))
    orc.eff_demagnifications[:] = eff.astype("float32")
    rng = np.random.default_rng(7)
    cn = lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    data = (np.abs(rng.standard_normal((ntheta, ndist, nz, n))) + 0.5).astype("float32")
    rec.data[:] = cuda(data)
    orc.data[:] = data

    def state(sc):
        return {"prb": (1 + 0.1 * cn(ndist, nz, n)).astype("complex64") if sc == 1 else
                (sc * cn(ndist, nz, n)).astype("complex64"),
                "proj": (0.05 * cn(ntheta, nz, n)).astype("complex64"),
                "pos": rng.uniform(-2, 2, (ntheta, ndist, 2)).astype("float32")}
    v, gr, et = state(1), state(0.1), state(0.1)
    g = lambda d: {k: cuda(x) for k, x in d.items()}
    o = lambda d: {k: x.astype("complex128") if np.iscomplexobj(x) else x.astype("float64") for k, x in d.items()}
    for a, b in ((gr, et), (et, et)):
        h = rec.hessian_cascade(g(v), g(a), g(b) if b is not a else g(a))
        ho = orc.hessian_cascade(o(v), o(a), o(b) if b is not a else o(a))
        assert abs(h / ho - 1) < 1e-4, (h, ho)
    out = {k: torch.zeros_like(x) for k, x in g(v).items()}
    rec.gradients_cascade(g(v), out)
    ref = {k: np.zeros_like(x) for k, x in o(v).items()}
    orc.gradients_cascade(o(v), ref)
    for k in ("prb", "proj", "pos"):
        assert rel_l2(out[k].cpu().numpy(), ref[k]) < 1e-4, k
    # the forward model alone: objective (min) and amplitudes (the gen_sqrt_data form)
    gv, ov = g(v), o(v)
    f = rec.min(gv["prb"], None, gv["pos"], gv["proj"])
    fo = orc.min(ov["prb"], None, ov["pos"], ov["proj"])
    assert abs(f / fo - 1) < 1e-4, (f, fo)
    from holotomocupy_b200 import _lib
    c = rec._coeff_into(gv["proj"], torch.empty_like(gv["proj"]))
    amp = torch.empty(ntheta, ndist, nz, n, dtype=torch.float32, device="cuda")
    _lib.call("ht_rec_forward", rec._h, _lib.ptr(c), _lib.ptr(gv["pos"]), _lib.ptr(rec.eff_demagnifications),
              _lib.ptr(gv["prb"]), None, _lib.ptr(amp), None, _lib.stream_ptr())
    y = [ov["prb"], ov["proj"], ov["pos"]]
    for i in range(1, len(orc.F))[::-1]:
        y = orc.F[i](y)
    assert rel_l2(amp.cpu().numpy(), np.abs(y)) < 1e-4


@pytest.mark.parametrize("mode", ["host", "graph"])
def test_bh_32_iterations_against_fp64_oracle(golden, mode):
    """32 BH iterations (FP32 bulk, FP64 reductions and step sizes) stay
    within rel L2 1e-4 of the FP64 oracle's BH on the golden problem
    (measured: obj 1.6e-5, prb 9e-8, pos 1.5e-7); the graph-replayed,
    device-scalar form gives the same state as the host-scalar one."""
    from oracle import holo_oracle as O
    from holotomocupy_b200.rec import Rec
    g = golden("rec")
    n, ntheta, ndist, nobj, _ = [int(v) for v in g["bh_dims"]]
    args = rec_args(n, ntheta, ndist, nobj, 32)
    rec = Rec(args)
    orc = O.Rec(args, "complex128")
    for r, put in ((rec, cuda), (orc, lambda a: a)):
        r.vars["obj"][:] = put(g["bh_obj_true"])
        r.vars["prb"][:] = put(g["bh_prb_true"])
        r.vars["pos"][:] = put(g["bh_pos_true"])
        r.gen_sqrt_data(r.vars, r.data)
        r.vars["obj"][:] = 0
        r.vars["prb"][:] = 1
        r.vars["pos"][:] = put(g["bh_pos_true"] + g["bh_pos_err"])
    rec.BH(mode=mode)
    orc.BH()
    for k in ("obj", "prb", "pos"):
        assert rel_l2(rec.vars[k].cpu().numpy(), orc.vars[k]) < 1e-4, k


def test_graph_history_beyond_the_default_room(golden):
    """BH(mode="graph") over more iterations than the device-side step-size
    history holds by default (4096) keeps every (alpha, beta) pair: the room
    is reserved before the iteration is recorded."""
    from holotomocupy_b200.rec import Rec
    g = golden("rec")
    n, ntheta, ndist, nobj, _ = [int(v) for v in g["bh_dims"]]
    niter = 4100
    rec = Rec(rec_args(n, ntheta, ndist, nobj, niter))
    rec.vars["obj"][:] = cuda(g["bh_obj_true"])
    rec.vars["prb"][:] = cuda(g["bh_prb_true"])
    rec.vars["pos"][:] = cuda(g["bh_pos_true"])
    rec.gen_sqrt_data(rec.vars, rec.data)
    rec.vars["obj"][:] = 0
    rec.vars["prb"][:] = 1
    rec.vars["pos"][:] = cuda(g["bh_pos_true"] + g["bh_pos_err"])
    record = []
    rec.BH(mode="graph", record=record)
    assert rec._hist_cap >= niter and int(rec._count.item()) == niter
    assert [r[0] for r in record] == list(range(niter))


@pytest.mark.parametrize("mode", ["host", "graph"])
def test_bh_real_object_against_fp64_oracle(golden, mode):
    """A real-valued (obj_dtype float32) object: 8 BH iterations on the golden
    problem (the real part of its object) stay within rel L2 1e-4 of the
    FP64 oracle's BH.  This iteration allocates temporaries, so
    mode="graph" iterates as "host" and records no graph."""
    from oracle import holo_oracle as O
    from holotomocupy_b200.rec import Rec
    g = golden("rec")
    n, ntheta, ndist, nobj, _ = [int(v) for v in g["bh_dims"]]
    args = rec_args(n, ntheta, ndist, nobj, 8)
    args.obj_dtype = "float32"
    rec = Rec(args)
    orc = O.Rec(args, "complex128")
    assert rec.vars["obj"].dtype == torch.float32 and not rec.graphable
    for r, put in ((rec, cuda), (orc, lambda a: a)):
        r.vars["obj"][:] = put(np.ascontiguousarray(g["bh_obj_true"].real))
        r.vars["prb"][:] = put(g["bh_prb_true"])
        r.vars["pos"][:] = put(g["bh_pos_true"])
        r.gen_sqrt_data(r.vars, r.data)
        r.vars["obj"][:] = 0
        r.vars["prb"][:] = 1
        r.vars["pos"][:] = put(g["bh_pos_true"] + g["bh_pos_err"])
    rec.BH(mode=mode)
    orc.BH()
    assert rec._graph is None
    for k in ("obj", "prb", "pos"):
        assert rel_l2(rec.vars[k].cpu().numpy(), orc.vars[k]) < 1e-4, k


def test_laplacian_terms_match_reference(golden):
    """gradient_laplacian, hessian_laplacian and the energy against the
    reference's own values (rec_mpi.py:402-496)."""
    from holotomocupy_b200.rec import Rec
    g = golden("lap")
    n, ntheta, ndist, nobj = [int(v) for v in g["l_dims"]]
    args = rec_args(n, ntheta, ndist, nobj)
    args.lam_laplacian = float(g["l_lam"])
    rec = Rec(args)
    rec.vars["obj"][:] = cuda(g["l_u"])
    rec.etas["obj"][:] = cuda(g["l_e"])
    gr = cuda(g["l_g0"]).clone()
    rec.gradient_laplacian(gr)
    assert rel_l2((gr - cuda(g["l_g0"])).cpu().numpy(), g["l_g"] - g["l_g0"]) < TOL
    h = rec.hessian_laplacian(cuda(g["l_d1"]))
    assert abs(h / float(g["l_h"]) - 1) < TOL
    e = rec._lap_energy()
    assert abs(e / float(g["l_energy"]) - 1) < TOL
    # the forms' and the energy's block sums are added in a fixed order: a second call repeats them bit for bit
    assert rec.hessian_laplacian(cuda(g["l_d1"])) == h and rec._lap_energy() == e


@pytest.mark.parametrize("mode", ["host", "graph"])
def test_bh_with_laplacian_matches_reference(golden, mode):
    """4 BH iterations with lam_laplacian > 0 against the reference's run."""
    from holotomocupy_b200.rec import Rec
    gr = golden("rec")
    g = golden("lap")
    n, ntheta, ndist, nobj, niter = [int(v) for v in g["lbh_dims"]]
    args = rec_args(n, ntheta, ndist, nobj, niter)
    args.lam_laplacian = float(g["lbh_lam"])
    rec = Rec(args)
    rec.vars["obj"][:] = cuda(gr["bh_obj_true"])
    rec.vars["prb"][:] = cuda(gr["bh_prb_true"])
    rec.vars["pos"][:] = cuda(gr["bh_pos_true"])
    rec.gen_sqrt_data(rec.vars, rec.data)
    rec.vars["obj"][:] = 0
    rec.vars["prb"][:] = 1
    rec.vars["pos"][:] = cuda(gr["bh_pos_true"] + gr["bh_pos_err"])
    record = []
    rec.BH(record=record, mode=mode)
    tb = g["lbh_topbottom"]
    ref_alpha = [tb[0, 0] / tb[0, 1]] + [tb[2 * i, 0] / tb[2 * i, 1] for i in range(1, niter)]
    for (i, a, b), ra in zip(record, ref_alpha):
        assert abs(a / ra - 1) < 1e-4, (i, a, ra)
    for k in ("obj", "prb", "pos", "proj"):
        assert rel_l2(rec.vars[k].cpu().numpy(), g[f"lbh_{k}"]) < TOL, k


def _prbfit_rec(g, niter=1):
    from holotomocupy_b200.rec import Rec
    n, ntheta, ndist, nobj = [int(v) for v in g["p_dims"]]
    args = rec_args(n, ntheta, ndist, nobj, niter)
    args.lam_prbfit = float(g["p_lam"])
    return Rec(args)


def test_prbfit_terms_match_reference(golden):
    """The probe-fit regulariser's gradient, Hessian form and objective, and the
    full gradient with it, against the reference's rec_mpi.py at lam_prbfit =
    2e-3 (rec_mpi.py:365-398, 305-325, 815-835)."""
    g = golden("prbfit")
    rec = _prbfit_rec(g)
    rec.ref[:] = cuda(g["p_ref"])
    rec.data[:] = cuda(g["p_data"])
    rec.eff_demagnifications[:] = (1 + rec.shrink_nd) / cuda(rec.norm_magnifications[None, :].astype("float32"))
    v = rec.vars
    v["obj"][:] = cuda(g["p_obj"])
    v["prb"][:] = cuda(g["p_prb"])
    v["pos"][:] = cuda(g["p_pos"])
    rec.fwd_tomo(v["obj"], out=v["proj"])
    gp = torch.zeros_like(v["prb"])
    rec.gradient_prbfit(gp, v["prb"])
    assert rel_l2(gp.cpu().numpy(), g["p_gprb_fit"]) < TOL
    h11, h12, _ = rec._prbfit_forms(v["prb"], cuda(g["p_d1"]), cuda(g["p_d2"]))
    assert abs(h12 / float(g["p_h12"]) - 1) < TOL
    assert abs(h11 / float(g["p_h11"]) - 1) < TOL
    assert abs(rec.min(v["prb"], v["obj"], v["pos"], v["proj"]) / float(g["p_F"]) - 1) < TOL
    rec.gradients(v, rec.grads)
    for k in ("prb", "obj", "pos"):
        assert rel_l2(rec.grads[k].cpu().numpy(), g[f"p_grad_{k}"]) < TOL, k


@pytest.mark.parametrize("mode", ["host", "graph"])
def test_bh_with_prbfit_matches_reference(golden, mode):
    """4 BH iterations with lam_prbfit = 2e-3 against the reference's run:
    state and step sizes, with host step sizes and graph-replayed (the
    probe-fit gradient and forms on the device, ht_prbfit_grad/forms)."""
    gr = golden("rec")
    g = golden("prbfit")
    from holotomocupy_b200.rec import Rec
    n, ntheta, ndist, nobj, niter = [int(v) for v in g["pbh_dims"]]
    args = rec_args(n, ntheta, ndist, nobj, niter)
    args.lam_prbfit = float(g["pbh_lam"])
    rec = Rec(args)
    rec.vars["obj"][:] = cuda(gr["bh_obj_true"])
    rec.vars["prb"][:] = cuda(gr["bh_prb_true"])
    rec.vars["pos"][:] = cuda(gr["bh_pos_true"])
    rec.gen_sqrt_data(rec.vars, rec.data)
    rec.gen_sqrt_ref(rec.vars["prb"], rec.ref)
    assert rel_l2(rec.ref.cpu().numpy(), g["pbh_ref"]) < TOL
    rec.vars["obj"][:] = 0
    rec.vars["prb"][:] = 1
    rec.vars["pos"][:] = cuda(gr["bh_pos_true"] + gr["bh_pos_err"])
    record = []
    rec.BH(record=record, mode=mode)
    tb = g["pbh_topbottom"]
    ref_alpha = [tb[0, 0] / tb[0, 1]] + [tb[2 * i, 0] / tb[2 * i, 1] for i in range(1, niter)]
    ref_beta = [0.0] + [tb[2 * i - 1, 0] / tb[2 * i - 1, 1] for i in range(1, niter)]
    for (i, a, b), ra, rb in zip(record, ref_alpha, ref_beta):
        assert abs(a / ra - 1) < 1e-4, (i, a, ra)
        if rb:
            assert abs(b / rb - 1) < 1e-4, (i, b, rb)
    for k in ("obj", "prb", "pos", "proj"):
        assert rel_l2(rec.vars[k].cpu().numpy(), g[f"pbh_{k}"]) < TOL, k


@pytest.fixture(scope="module")
def bh64_oracle():
    """32 BH iterations of the FP64 oracle at 64^3, 32 angles, 4 distances
    (3-6 mm, unit magnification), seeded ellipsoid phantom, random probe,
    positions +-2 px (0.5 px initial error), noise-free amplitudes."""
    from oracle import holo_oracle as O
    from holotomocupy_b200.synthetic import ellipsoid_phantom, random_positions, random_probe, workload_args
    n, ntheta, ndist, niter = 64, 32, 4, 32
    args = workload_args(n, ntheta, ndist, niter=niter)
    obj = ellipsoid_phantom(n, 20, 21, device="cpu").numpy()
    prb = random_probe(ndist, n, n, 22, device="cpu").numpy()
    pos = random_positions(ntheta, ndist, 2.0, 23, device="cpu").numpy()
    pos0 = pos + np.random.default_rng(24).uniform(-0.5, 0.5, pos.shape).astype("float32")
    orc = O.Rec(args, "complex128")
    orc.eff_demagnifications[:] = 1
    orc.vars["obj"][:] = obj
    orc.vars["prb"][:] = prb
    orc.vars["pos"][:] = pos
    orc.gen_sqrt_data(orc.vars, orc.data)
    orc.eff_demagnifications[:] = 0          # shrink_nd is the same array (rec_mpi.py:135-136)
    data = orc.data.astype("float32")
    orc.data[:] = data
    orc.vars["obj"][:] = 0
    orc.vars["prb"][:] = 1
    orc.vars["pos"][:] = pos0
    orc.BH()
    return args, data, pos0, {k: orc.vars[k].copy() for k in ("obj", "prb", "pos")}


@pytest.mark.parametrize("mode", ["host", "graph"])
def test_bh_32_iterations_64cubed_4dist_against_fp64_oracle(bh64_oracle, mode):
    """The 32-iteration bound at 64^3 x 32 angles x 4 distances: the FP32-bulk,
    FP64-reduction BH stays within rel L2 1e-4 of the FP64 oracle's BH."""
    from holotomocupy_b200.rec import Rec
    args, data, pos0, ref = bh64_oracle
    rec = Rec(args)
    rec.data[:] = cuda(data)
    rec.vars["prb"][:] = 1
    rec.vars["pos"][:] = cuda(pos0)
    rec.BH(mode=mode)
    for k in ("obj", "prb", "pos"):
        assert rel_l2(rec.vars[k].cpu().numpy(), ref[k]) < 1e-4, k


@pytest.mark.parametrize("mode", ["host", "graph"])
def test_chunked_bh_equals_unchunked(golden, mode):
    """Angle chunks of the fused cascade (each chunk's forward pass recomputed
    before its Hessian pass) and object slabs of the Radon transform give the
    BH iteration of the whole problem: 4 iterations, chunks of 5 of 12 angles
    and slabs of 12 of 32 slices, against the unchunked run and the
    reference's."""
    from holotomocupy_b200.rec import Rec
    g = golden("rec")
    n, ntheta, ndist, nobj, niter = [int(v) for v in g["bh_dims"]]
    out = []
    for chunk, slab in ((None, None), (5, 12)):
        args = rec_args(n, ntheta, ndist, nobj, niter)
        args.angle_chunk, args.slab_chunk = chunk, slab
        rec = Rec(args)
        rec.vars["obj"][:] = cuda(g["bh_obj_true"])
        rec.vars["prb"][:] = cuda(g["bh_prb_true"])
        rec.vars["pos"][:] = cuda(g["bh_pos_true"])
        rec.gen_sqrt_data(rec.vars, rec.data)
        rec.vars["obj"][:] = 0
        rec.vars["prb"][:] = 1
        rec.vars["pos"][:] = cuda(g["bh_pos_true"] + g["bh_pos_err"])
        rec.BH(mode=mode)
        out.append({k: rec.vars[k].cpu().numpy() for k in ("obj", "prb", "pos", "proj")})
    for k in out[0]:
        assert rel_l2(out[1][k], out[0][k]) < 1e-6, k
        assert rel_l2(out[1][k], g[f"bh_{k}"]) < TOL, k


def test_bh_checkpoints_hold_the_iteration_state(golden, tmp_path):
    """BH with a checkpoint writer (vis_step 2, rec_mpi.py's vis_debug) saves,
    at iteration 2, the state a 3-iteration run ends with; reading it back
    gives obj, prb and pos."""
    from holotomocupy_b200.checkpoint import Writer, read_checkpoint
    from holotomocupy_b200.rec import Rec
    g = golden("rec")
    n, ntheta, ndist, nobj, _ = [int(v) for v in g["bh_dims"]]
    states = []
    for niter, writer in ((4, Writer(str(tmp_path), fmt="npz")), (3, None)):
        args = rec_args(n, ntheta, ndist, nobj, niter)
        args.vis_step = 2
        rec = Rec(args)
        rec.vars["obj"][:] = cuda(g["bh_obj_true"])
        rec.vars["prb"][:] = cuda(g["bh_prb_true"])
        rec.vars["pos"][:] = cuda(g["bh_pos_true"])
        rec.gen_sqrt_data(rec.vars, rec.data)
        rec.vars["obj"][:] = 0
        rec.vars["prb"][:] = 1
        rec.vars["pos"][:] = cuda(g["bh_pos_true"] + g["bh_pos_err"])
        rec.BH(writer=writer)
        states.append({k: rec.vars[k].cpu().numpy() for k in ("obj", "prb", "pos")})
    ck = read_checkpoint(str(tmp_path / "checkpoint_0002.npz"), n, nobj)
    assert ck["iter"] == 2
    for k in ("obj", "prb", "pos"):
        assert rel_l2(ck[k].numpy(), states[1][k]) < 1e-6, k
