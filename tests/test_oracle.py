"""The CPU oracle against the golden vectors made by running the reference's
own operators (tests/golden/make_golden.py).  FP32 mode must reproduce the
reference to FP32 rounding; FP64 mode differs by the reference's own FP32
error (and, for the propagator, by the FP32 rounding of its Fresnel table).
Beside the fixtures, the properties the reference's own tests look at: the
adjoints of R and D, D's energy, and curlyS against scipy's cubic spline."""
import types

import numpy as np
import pytest

from conftest import rel_l2
from oracle import holo_oracle as O

TOL32 = 2e-6      # oracle in FP32 vs reference in FP32
TOL64 = 1e-5      # FP64 oracle vs FP32 reference (operators other than D/DT)
TOL64_D = 1e-4    # FP64 oracle (exact Fresnel table) vs FP32 reference table


@pytest.mark.parametrize("dt,tol", [("complex64", TOL32), ("complex128", TOL64)])
@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_tomo(golden, tag, dt, tol):
    g = golden("tomo")
    n, nz = int(g[f"{tag}_n"]), int(g[f"{tag}_nz"])
    t = O.Tomo(n, nz, g[f"{tag}_theta"], float(g[f"{tag}_mask_r"]), dt)
    assert t.m == int(g[f"{tag}_m"])
    assert rel_l2(t.phi, g[f"{tag}_phi"]) < tol
    for src, op, key in [("xc", t.R, "Rxc"), ("yc", t.RT, "RTyc"), ("xf", t.R, "Rxf"), ("yf", t.RT, "RTyf")]:
        out = op(g[f"{tag}_{src}"])
        assert out.shape == g[f"{tag}_{key}"].shape
        assert np.iscomplexobj(out) == np.iscomplexobj(g[f"{tag}_{key}"])
        assert rel_l2(out, g[f"{tag}_{key}"]) < tol


@pytest.mark.parametrize("dt,tol", [("complex64", TOL32), ("complex128", TOL64_D)])
@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_propagation(golden, tag, dt, tol):
    g = golden("prop")
    n, nz = int(g[f"{tag}_n"]), int(g[f"{tag}_nz"])
    p = O.Propagation(n, nz, 3, 3, float(g[f"{tag}_wavelength"]), float(g[f"{tag}_voxelsize"]),
                      g[f"{tag}_distance"], dt)
    for j in range(3):
        assert rel_l2(p.D(g[f"{tag}_a"], j), g[f"{tag}_D{j}"]) < tol
        assert rel_l2(p.DT(g[f"{tag}_b"], j), g[f"{tag}_DT{j}"]) < tol
    assert p.D(g[f"{tag}_a"][0], 1).shape == g[f"{tag}_D2d"].shape


def _crand(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def test_tomo_adjoint():
    """<R x, y> = <x, R^T y> in FP64 (the reference's tests/tomo/test_tomo.ipynb
    adjoint check, asserted)."""
    rng = np.random.default_rng(5)
    n, nz, ntheta = 32, 4, 24
    t = O.Tomo(n, nz, np.linspace(0, np.pi, ntheta, endpoint=False).astype("float32"), 1, "complex128")
    x, y = _crand(rng, (nz, n, n)), _crand(rng, (ntheta, nz, n))
    lhs, rhs = np.vdot(t.R(x), y), np.vdot(x, t.RT(y))
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_propagation_adjoint_and_energy():
    """<D x, y> = <x, D^T y> in FP64, and D keeps the energy of a smooth field
    away from the edges (the reference's
    tests/propagation/test_propagation.py:42-88, adjoint and energy sections)."""
    rng = np.random.default_rng(6)
    n, nz = 48, 40
    p = O.Propagation(n, nz, 2, 2, 7.3e-11, 20e-9, np.array([3e-3, 5e-3]), "complex128")
    x, y = _crand(rng, (2, nz, n)), _crand(rng, (2, nz, n))
    for j in range(2):
        lhs, rhs = np.vdot(p.D(x, j), y), np.vdot(x, p.DT(y, j))
        assert abs(lhs - rhs) / abs(lhs) < 1e-12
    yy, xx = np.meshgrid(np.arange(nz) - nz / 2, np.arange(n) - n / 2, indexing="ij")
    blob = np.exp(-(yy ** 2 + xx ** 2) / (2 * 4.0 ** 2))[None].astype("complex128")
    d = p.D(blob, 0)
    assert np.linalg.norm(d - blob) / np.linalg.norm(blob) > 0.5    # the field does change (measured 1.3)
    assert abs(np.linalg.norm(d) / np.linalg.norm(blob) - 1) < 1e-9  # measured 6e-16


def test_propagation_reference_table(golden):
    """table='ref32' rebuilds the reference's FP32 Fresnel table bit for bit."""
    g = golden("prop")
    for tag in "abc":
        n, nz = int(g[f"{tag}_n"]), int(g[f"{tag}_nz"])
        t = O.fresnel_kernel(n, nz, float(g[f"{tag}_wavelength"]), float(g[f"{tag}_voxelsize"]),
                             g[f"{tag}_distance"], "ref32")
        np.testing.assert_array_equal(t, g[f"{tag}_fker"])


@pytest.mark.parametrize("dt,tol", [("complex64", TOL32), ("complex128", TOL64)])
@pytest.mark.parametrize("key", ["complex64_a", "complex64_b", "float32_a", "float32_b"])
def test_shift(golden, key, dt, tol):
    g = golden("shift")
    G = lambda k: g[f"{key}_{k}"]
    n, npsi, nz, nzpsi, nt = [int(v) for v in G("dims")]
    s = O.Shift(n, npsi, nz, nzpsi, key.split("_")[0], dt)
    c = s.coeff(G("psi"))
    assert rel_l2(c, G("coeff")) < tol
    assert rel_l2(s.S(c, G("r"), G("m")), G("S")) < tol
    assert rel_l2(s.Sadj(G("g"), G("r"), G("m")), G("Sadj")) < tol
    assert rel_l2(s.curlyS(G("psi"), G("r"), G("m")), G("curlyS")) < tol
    assert rel_l2(s.dcurlySc(c, G("r"), G("m"), G("c1"), G("d1")), G("dS")) < tol
    assert rel_l2(s.d2curlySc(c, G("r"), G("m"), G("c1"), G("d1"), G("c2"), G("d2")), G("d2S")) < tol
    o1, o2 = s.dcurlySadjc(c, G("r"), G("m"), G("g"))
    assert rel_l2(o1, G("dSadj1")) < tol
    assert rel_l2(o2, G("dSadj2")) < tol


@pytest.mark.parametrize("ry,rx", [(0.0, 0.7), (1.3, -2.4), (-3.6, 0.25)])
def test_curlyS_is_scipys_cubic_spline_shift(ry, rx):
    """curlyS at unit magnification is a cubic B-spline interpolation: on an
    object that is zero within n/4 of its edges it equals
    scipy.ndimage.shift(order=3) (the comparison the reference's
    tests/shift/test_shift.ipynb plots, here asserted; measured 1.4-1.9e-10)."""
    import scipy.ndimage as nd
    n = 64
    s = O.Shift(n, n, n, n, "complex64", "complex128")
    rng = np.random.default_rng(3)
    pad = n // 4
    a = np.zeros((1, n, n), "complex128")
    a[0, pad:-pad, pad:-pad] = rng.standard_normal((n - 2 * pad,) * 2) + 1j * rng.standard_normal((n - 2 * pad,) * 2)
    got = s.curlyS(a, np.array([[ry, rx]]), np.ones(1))[0]
    ref = (nd.shift(a[0].real, [ry, rx], order=3, mode="constant", cval=0)
           + 1j * nd.shift(a[0].imag, [ry, rx], order=3, mode="constant", cval=0))
    assert rel_l2(got, ref) < 1e-8


@pytest.mark.parametrize("dt,tol", [("complex64", TOL32), ("complex128", TOL64)])
@pytest.mark.parametrize("tag", ["a", "b", "c", "d"])
def test_shift_back(golden, tag, dt, tol):
    """Sback, coeffback and curlySback (shift.py:84-96, 138-153) against the
    reference run under the shim."""
    g = golden("sback")
    G = lambda k: g[f"sb_{tag}_{k}"]
    n, npsi, nz, nzpsi, nt = [int(v) for v in G("dims")]
    s = O.Shift(n, npsi, nz, nzpsi, "complex64", dt)
    assert rel_l2(s.Sback(G("g"), G("r"), G("m")), G("Sback")) < tol
    if tag != "d":
        # the stretched spline's symbol dips to ~0.1 at m = 1.55, so its inverse
        # amplifies FP32 rounding about tenfold: 1e-5 for the back-filter
        tb = max(tol, 1e-5)
        assert rel_l2(s.coeffback(G("psi"), G("m")), G("coeffback")) < tb
        assert rel_l2(s.curlySback(G("g"), G("r"), G("m")), G("curlySback")) < tb


def _sback_loops(g, r, mag, n, npsi, nz, nzpsi):
    """The sback kernel (cuda_kernels.py:305-370, dir = 1) as plain loops over
    pixels and taps, in float64: a check on the vectorised restatement."""
    f = np.zeros((g.shape[0], nzpsi, npsi), complex)
    for tz in range(g.shape[0]):
        m0 = float(mag[tz])
        half = (m0 - 1.0) / 2.0
        span = 2.0 * m0
        for ty in range(nz):
            for tx in range(n):
                x = (m0 * (tx - n // 2) - r[tz, 1] + half) + npsi // 2
                y = (m0 * (ty - nz // 2) - r[tz, 0] + half) + nzpsi // 2
                ix, iy = int(np.floor(x)), int(np.floor(y))
                dx, dy = x - ix, y - iy
                for jy in range(int(np.ceil(dy - span)), int(dy + span)):
                    if not 0 <= iy + jy < nzpsi:
                        continue
                    pdym = O.K.bphi(np.float64((dy - jy) / m0))
                    for jx in range(int(np.ceil(dx - span)), int(dx + span)):
                        if not 0 <= ix + jx < npsi:
                            continue
                        f[tz, iy + jy, ix + jx] += O.K.bphi(np.float64((dx - jx) / m0)) * pdym * g[tz, ty, tx]
    return f


@pytest.mark.parametrize("mag", [[0.8], [1.0], [1.55], [0.8, 1.3]])
def test_sback_restatement_matches_kernel_loops(mag):
    rng = np.random.default_rng(11)
    n, npsi, nz, nzpsi = 8, 12, 6, 10
    nt = len(mag)
    g = rng.standard_normal((nt, nz, n)) + 1j * rng.standard_normal((nt, nz, n))
    r = rng.uniform(-2, 2, (nt, 2))
    mg = np.array(mag)
    s = O.Shift(n, npsi, nz, nzpsi, "complex64", "complex128")
    assert rel_l2(s.Sback(g, r, mg), _sback_loops(g, r, mg, n, npsi, nz, nzpsi)) < 1e-12


def rec_args(n, ntheta, ndist, nobj, niter=1):
    """The solver arguments make_golden.py used."""
    return types.SimpleNamespace(
        energy=17.1, detector_pixelsize=1.4760147601476e-6 * 2 * 2048 / n,
        focustodetectordistance=1.217,
        z1=(np.array([5.110, 5.464, 6.879, 9.817]) * 1e-3 + 3.135e-3)[:ndist],
        theta=np.linspace(0, np.pi, ntheta, endpoint=False).astype("float32"),
        ndist=ndist, ntheta=ntheta, nz=n, n=n, nzobj=nobj, nobj=nobj,
        obj_dtype="complex64", mask=0.9, lam_prbfit=0.0, rho=[1, 0.05, 0.02],
        niter=niter, nchunk=max(nobj, ntheta), vis_step=-1, err_step=-1, start_iter=0)


@pytest.mark.parametrize("dt,tol", [("complex64", TOL32), ("complex128", TOL64)])
def test_cascade(golden, dt, tol):
    g = golden("rec")
    n, ntheta, ndist, nobj = [int(v) for v in g["c_dims"]]
    rec = O.Rec(rec_args(n, ntheta, ndist, nobj), dt)
    rec.data[:] = g["c_data"]
    rec.eff_demagnifications[:] = (1 + rec.shrink_nd) / rec.norm_magnifications[None, :]
    v = {"prb": g["c_prb"].astype(rec.cdt), "proj": g["c_proj"].astype(rec.cdt), "pos": g["c_pos"]}
    gr = {k: g[f"c_g_{k}"] for k in ("prb", "proj", "pos")}
    et = {k: g[f"c_e_{k}"] for k in ("prb", "proj", "pos")}
    assert abs(rec.min(v["prb"], None, v["pos"], v["proj"]) / float(g["c_F"]) - 1) < tol
    assert abs(rec.hessian_cascade(v, gr, et) / float(g["c_h_ge"]) - 1) < tol
    assert abs(rec.hessian_cascade(v, et, et) / float(g["c_h_ee"]) - 1) < tol
    out = {k: np.zeros_like(v[k]) for k in v}
    rec.gradients_cascade(v, out)
    for k in ("prb", "proj", "pos"):
        assert rel_l2(out[k], g[f"c_grad_{k}"]) < 5 * tol


@pytest.mark.parametrize("dt,tol", [("complex64", 1e-5), ("complex128", 1e-5)])
def test_bh(golden, dt, tol):
    g = golden("rec")
    n, ntheta, ndist, nobj, niter = [int(v) for v in g["bh_dims"]]
    rec = O.Rec(rec_args(n, ntheta, ndist, nobj, niter), dt)
    rec.vars["obj"][:] = g["bh_obj_true"]
    rec.vars["prb"][:] = g["bh_prb_true"]
    rec.vars["pos"][:] = g["bh_pos_true"]
    rec.gen_sqrt_data(rec.vars, rec.data)
    assert rel_l2(rec.data, g["bh_data"]) < 1e-6
    rec.vars["obj"][:] = 0
    rec.vars["prb"][:] = 1
    rec.vars["pos"][:] = g["bh_pos_true"] + g["bh_pos_err"]
    rec.BH()
    for k in ("obj", "prb", "pos", "proj"):
        assert rel_l2(rec.vars[k], g[f"bh_{k}"]) < tol


@pytest.mark.parametrize("dt", ["complex64", "complex128"])
def test_bh_real_object(golden, dt):
    """BH with a real-valued object (obj_dtype float32) against the
    reference's run: its data, and the state after 4 iterations (measured rel
    L2: obj 0.9e-5 / 1.2e-5, proj 1.1e-5 / 1.4e-5 in FP32 / FP64 against the
    reference's FP32)."""
    g = golden("realbh")
    n, ntheta, ndist, nobj, niter = [int(v) for v in g["rbh_dims"]]
    args = rec_args(n, ntheta, ndist, nobj, niter)
    args.obj_dtype = "float32"
    rec = O.Rec(args, dt)
    assert not np.iscomplexobj(rec.vars["obj"])
    rec.vars["obj"][:] = g["rbh_obj_true"]
    rec.vars["prb"][:] = g["rbh_prb_true"]
    rec.vars["pos"][:] = g["rbh_pos_true"]
    rec.gen_sqrt_data(rec.vars, rec.data)
    assert rel_l2(rec.data, g["rbh_data"]) < 1e-6
    rec.vars["obj"][:] = 0
    rec.vars["prb"][:] = 1
    rec.vars["pos"][:] = g["rbh_pos_true"] + g["rbh_pos_err"]
    rec.BH()
    for k in ("obj", "prb", "pos", "proj"):
        assert rel_l2(rec.vars[k], g[f"rbh_{k}"]) < 3e-5, k


@pytest.mark.parametrize("dt,tol", [("complex64", TOL32), ("complex128", TOL64)])
def test_laplacian_terms(golden, dt, tol):
    """gradient_laplacian, hessian_laplacian and the energy (rec_mpi.py:402-496)."""
    g = golden("lap")
    n, ntheta, ndist, nobj = [int(v) for v in g["l_dims"]]
    args = rec_args(n, ntheta, ndist, nobj)
    args.lam_laplacian = float(g["l_lam"])
    rec = O.Rec(args, dt)
    rec.vars["obj"][:] = g["l_u"]
    rec.etas["obj"][:] = g["l_e"]
    gr = g["l_g0"].astype(rec.vars["obj"].dtype)
    rec.gradient_laplacian(gr)
    assert rel_l2(gr - g["l_g0"], g["l_g"] - g["l_g0"]) < 10 * tol
    assert abs(rec.hessian_laplacian(g["l_d1"]) / float(g["l_h"]) - 1) < 10 * tol
    assert abs(rec._lap_energy_local() / float(g["l_energy"]) - 1) < 10 * tol


@pytest.mark.parametrize("dt,tol", [("complex64", 1e-5), ("complex128", 1e-5)])
def test_bh_with_laplacian(golden, dt, tol):
    gr = golden("rec")
    g = golden("lap")
    n, ntheta, ndist, nobj, niter = [int(v) for v in g["lbh_dims"]]
    args = rec_args(n, ntheta, ndist, nobj, niter)
    args.lam_laplacian = float(g["lbh_lam"])
    rec = O.Rec(args, dt)
    rec.vars["obj"][:] = gr["bh_obj_true"]
    rec.vars["prb"][:] = gr["bh_prb_true"]
    rec.vars["pos"][:] = gr["bh_pos_true"]
    rec.gen_sqrt_data(rec.vars, rec.data)
    rec.vars["obj"][:] = 0
    rec.vars["prb"][:] = 1
    rec.vars["pos"][:] = gr["bh_pos_true"] + gr["bh_pos_err"]
    rec.BH()
    for k in ("obj", "prb", "pos", "proj"):
        assert rel_l2(rec.vars[k], g[f"lbh_{k}"]) < tol, k
