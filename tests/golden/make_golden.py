"""Generate golden vectors by running the reference's own Python operators.

Run in a container that has the reference source tree (read-only is fine):

    python tests/golden/make_golden.py /path/to/holotomocupy/src

The reference is CuPy code; ``oracle/refshim.py`` maps CuPy to NumPy and its
raw CUDA kernels to the NumPy restatements in ``oracle/kernels_np.py``, then
imports ``tomo.py``, ``shift.py``, ``propagation.py`` and ``rec_mpi.py``
unchanged.  Everything runs in the reference's FP32 arithmetic.  Outputs are
small ``.npz`` files next to this script; the GPU parity tests and the oracle
tests compare against them.
"""
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.refshim import load_reference  # noqa: E402


def crand(rng, shape, scale=1.0):
    return ((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * scale).astype("complex64")


def frand(rng, shape, scale=1.0):
    return (rng.standard_normal(shape) * scale).astype("float32")


def tomo_cases(ns):
    out = {}
    for (n, nz, ntheta, mask_r, tag) in [(32, 4, 24, 1, "a"), (18, 3, 10, 0, "b"), (48, 2, 40, 0.9, "c")]:
        rng = np.random.default_rng(100 + n)
        theta = np.linspace(0, np.pi, ntheta, endpoint=False).astype("float32")
        t = ns.tomo.Tomo(n, nz, theta, mask_r)
        xc = crand(rng, (nz, n, n))
        yc = crand(rng, (ntheta, nz, n))
        xf = frand(rng, (nz, n, n))
        yf = frand(rng, (ntheta, nz, n))
        out.update({
            f"{tag}_n": n, f"{tag}_nz": nz, f"{tag}_mask_r": mask_r, f"{tag}_theta": theta,
            f"{tag}_xc": xc, f"{tag}_yc": yc, f"{tag}_xf": xf, f"{tag}_yf": yf,
            f"{tag}_Rxc": t.R(ns.cp.array(xc)).get(), f"{tag}_RTyc": t.RT(ns.cp.array(yc)).get(),
            f"{tag}_Rxf": t.R(ns.cp.array(xf)).get(), f"{tag}_RTyf": t.RT(ns.cp.array(yf)).get(),
            f"{tag}_mask": np.asarray(t.mask, dtype="float32") * np.ones((n, n), "float32"),
            f"{tag}_m": t.pars[0], f"{tag}_phi": np.asarray(t.pars[2]),
        })
    np.savez_compressed(os.path.join(HERE, "tomo.npz"), **out)


def prop_cases(ns):
    out = {}
    wavelength = 1.24e-9 / 17.1
    for (n, nz, ntheta, tag) in [(32, 24, 3, "a"), (64, 64, 2, "b"), (48, 36, 2, "c")]:
        rng = np.random.default_rng(200 + n)
        distance = np.array([3e-3, 4.5e-3, 6e-3])
        p = ns.propagation.Propagation(n, nz, ntheta, len(distance), wavelength, 20e-9, distance)
        a = crand(rng, (ntheta, nz, n))
        b = crand(rng, (ntheta, nz, n))
        out.update({f"{tag}_n": n, f"{tag}_nz": nz, f"{tag}_a": a, f"{tag}_b": b,
                    f"{tag}_distance": distance, f"{tag}_wavelength": wavelength,
                    f"{tag}_voxelsize": 20e-9, f"{tag}_fker": np.asarray(p.fker)})
        for j in range(len(distance)):
            out[f"{tag}_D{j}"] = p.D(ns.cp.array(a), j).get()
            out[f"{tag}_DT{j}"] = p.DT(ns.cp.array(b), j).get()
        out[f"{tag}_D2d"] = p.D(ns.cp.array(a[0]), 1).get()
    np.savez_compressed(os.path.join(HERE, "prop.npz"), **out)


def shift_cases(ns):
    out = {}
    for dt in ("complex64", "float32"):
        for (n, npsi, nz, nzpsi, ntheta, tag) in [(24, 32, 20, 24, 3, "a"), (32, 32, 32, 32, 2, "b")]:
            key = f"{dt}_{tag}"
            rng = np.random.default_rng(300 + n + len(dt))
            s = ns.shift.Shift(n, npsi, nz, nzpsi, dt)
            mk = (lambda sh: crand(rng, sh)) if dt == "complex64" else (lambda sh: frand(rng, sh))
            psi = mk((ntheta, nzpsi, npsi))
            c1 = mk((ntheta, nzpsi, npsi))
            c2 = mk((ntheta, nzpsi, npsi))
            g = mk((ntheta, nz, n))
            r = (rng.uniform(-3, 3, (ntheta, 2))).astype("float32")
            d1 = frand(rng, (ntheta, 2))
            d2 = frand(rng, (ntheta, 2))
            m = np.ones(ntheta, "float32")
            if tag == "a":
                m = np.array([1.0, 0.93, 1.07], "float32")[:ntheta]
            C = lambda x: ns.cp.array(x)
            c = s.coeff(C(psi))
            o1, o2 = s.dcurlySadjc(c, C(r), C(m), C(g))
            out.update({
                f"{key}_dims": np.array([n, npsi, nz, nzpsi, ntheta]),
                f"{key}_psi": psi, f"{key}_c1": c1, f"{key}_c2": c2, f"{key}_g": g,
                f"{key}_r": r, f"{key}_d1": d1, f"{key}_d2": d2, f"{key}_m": m,
                f"{key}_coeff": c.get(),
                f"{key}_S": s.S(c, C(r), C(m)).get(),
                f"{key}_Sadj": s.Sadj(C(g), C(r), C(m)).get(),
                f"{key}_curlyS": s.curlyS(C(psi), C(r), C(m)).get(),
                f"{key}_dS": s.dcurlySc(c, C(r), C(m), C(c1), C(d1)).get(),
                f"{key}_d2S": s.d2curlySc(c, C(r), C(m), C(c1), C(d1), C(c2), C(d2)).get(),
                f"{key}_dSadj1": o1.get(), f"{key}_dSadj2": o2.get(),
            })
    np.savez_compressed(os.path.join(HERE, "shift.npz"), **out)


def sback_cases(ns):
    """Shift.Sback / coeffback / curlySback (shift.py:84-96, 138-153), the
    Paganin back-projection helpers: one image and a scalar magnification as
    the reference's callers use them (experimental/*/steps15.py), plus a
    three-image Sback with per-image magnifications."""
    out = {}
    cases = [(32, 48, 24, 36, 1, 0.8, "a"), (32, 32, 32, 32, 1, 1.0, "b"), (24, 32, 24, 32, 1, 1.55, "c"),
             (32, 36, 24, 48, 3, None, "d")]
    for (n, npsi, nz, nzpsi, nt, m, tag) in cases:
        rng = np.random.default_rng(700 + n + npsi + nz)
        s = ns.shift.Shift(n, npsi, nz, nzpsi, "complex64")
        g = crand(rng, (nt, nz, n))
        psi = crand(rng, (nt, nzpsi, npsi))
        r = rng.uniform(-3, 3, (nt, 2)).astype("float32")
        C = lambda x: ns.cp.array(x)
        key = f"sb_{tag}"
        out.update({f"{key}_dims": np.array([n, npsi, nz, nzpsi, nt]), f"{key}_g": g, f"{key}_psi": psi,
                    f"{key}_r": r})
        if m is None:
            mm = np.array([0.8, 1.0, 1.3], "float32")
            out[f"{key}_m"] = mm
            out[f"{key}_Sback"] = s.Sback(C(g), C(r), C(mm)).get()
        else:
            mm = np.array(m, "float32")        # a 0-d array, as the callers pass it
            out[f"{key}_m"] = mm
            out[f"{key}_Sback"] = s.Sback(C(g), C(r), C(mm)).get()
            out[f"{key}_coeffback"] = s.coeffback(C(psi), C(mm)).get()
            out[f"{key}_curlySback"] = s.curlySback(C(g), C(r), C(mm)).get()
    np.savez_compressed(os.path.join(HERE, "sback.npz"), **out)


def rec_args(n, ntheta, ndist, nobj, niter=1):
    return types.SimpleNamespace(
        energy=17.1, detector_pixelsize=1.4760147601476e-6 * 2 * 2048 / n,
        focustodetectordistance=1.217,
        z1=(np.array([5.110, 5.464, 6.879, 9.817]) * 1e-3 + 3.135e-3)[:ndist],
        theta=np.linspace(0, np.pi, ntheta, endpoint=False).astype("float32"),
        ndist=ndist, ntheta=ntheta, nz=n, n=n, nzobj=nobj, nobj=nobj,
        obj_dtype="complex64", mask=0.9, lam_prbfit=0.0, rho=[1, 0.05, 0.02],
        niter=niter, nchunk=max(nobj, ntheta), vis_step=-1, err_step=-1, start_iter=0,
        comm=sys.modules["mpi4py"].MPI.COMM_WORLD)


def phantom(n, rng, nell=6):
    """Small ellipsoid phantom: delta/beta inside random ellipsoids."""
    ax = np.arange(n) - n / 2
    z, y, x = np.meshgrid(ax, ax, ax, indexing="ij")
    obj = np.zeros((n, n, n), "complex64")
    for _ in range(nell):
        c = rng.uniform(-n / 5, n / 5, 3)
        s = rng.uniform(n / 12, n / 5, 3)
        delta = rng.uniform(1, 3)
        inside = ((z - c[0]) / s[0]) ** 2 + ((y - c[1]) / s[1]) ** 2 + ((x - c[2]) / s[2]) ** 2 <= 1
        obj[inside] += (-delta + 1j * delta / 50) * 0.05
    return obj


def rec_cases(ns):
    out = {}
    # ---- cascade building blocks at one point
    n, ntheta, ndist, nobj = 32, 6, 2, 32
    rng = np.random.default_rng(42)
    args = rec_args(n, ntheta, ndist, nobj)
    rec = ns.rec_mpi.Rec(args)
    prb = (1 + 0.2 * crand(rng, (ndist, n, n))).astype("complex64")
    proj = crand(rng, (ntheta, nobj, nobj), 0.1)
    pos = frand(rng, (ntheta, ndist, 2), 0.8)
    data = (np.abs(frand(rng, (ntheta, ndist, n, n))) + 0.5).astype("float32")
    dirs = {}
    for name in ("g", "e"):
        dirs[name] = {"prb": crand(rng, (ndist, n, n), 0.1), "proj": crand(rng, (ntheta, nobj, nobj), 0.05),
                      "pos": frand(rng, (ntheta, ndist, 2), 0.3)}
    rec.data[:] = data
    rec.eff_demagnifications[:] = (1 + rec.shrink_nd) / ns.cp.array(rec.norm_magnifications[None, :])
    vars_ = {"prb": ns.cp.array(prb), "proj": proj.copy(), "pos": ns.cp.array(pos)}
    grads = {k: (ns.cp.array(v) if k != "proj" else v.copy()) for k, v in dirs["g"].items()}
    etas = {k: (ns.cp.array(v) if k != "proj" else v.copy()) for k, v in dirs["e"].items()}
    Fval = float(ns.cp.asnumpy(rec.min(vars_["prb"], None, vars_["pos"], vars_["proj"])))
    h_ge = float(rec.hessian_cascade(vars_, grads, etas))
    h_ee = float(rec.hessian_cascade(vars_, etas, etas))
    g_out = {"prb": ns.cp.zeros((ndist, n, n), "complex64"), "proj": np.zeros((ntheta, nobj, nobj), "complex64"),
             "pos": ns.cp.zeros((ntheta, ndist, 2), "float32")}
    rec.gradients_cascade(vars_, g_out)
    out.update({
        "c_dims": np.array([n, ntheta, ndist, nobj]), "c_prb": prb, "c_proj": proj, "c_pos": pos, "c_data": data,
        "c_F": Fval, "c_h_ge": h_ge, "c_h_ee": h_ee,
        "c_grad_prb": np.asarray(g_out["prb"]), "c_grad_proj": np.asarray(g_out["proj"]),
        "c_grad_pos": np.asarray(g_out["pos"]),
        "c_fker": np.asarray(rec.cl_prop.fker),
    })
    for name in ("g", "e"):
        for k, v in dirs[name].items():
            out[f"c_{name}_{k}"] = v
    out["c_norm_mag"] = np.asarray(rec.norm_magnifications)
    # ---- a short BH run from a synthetic phantom
    n, ntheta, ndist, nobj, niter = 32, 12, 2, 32, 4
    rng = np.random.default_rng(7)
    args = rec_args(n, ntheta, ndist, nobj, niter)
    rec = ns.rec_mpi.Rec(args)
    obj = phantom(nobj, rng)
    prb = (1 + 0.1 * crand(rng, (ndist, n, n))).astype("complex64")
    pos = frand(rng, (ntheta, ndist, 2), 1.0)
    pos_err = frand(rng, (ntheta, ndist, 2), 0.2)
    rec.vars["obj"][:] = obj
    rec.vars["prb"][:] = ns.cp.array(prb)
    rec.vars["pos"][:] = ns.cp.array(pos)
    rec.gen_sqrt_data(rec.vars, rec.data)
    data = np.array(rec.data)
    rec.vars["obj"][:] = 0
    rec.vars["prb"][:] = ns.cp.array(1)
    rec.vars["pos"][:] = ns.cp.array(pos + pos_err)
    pairs = []
    orig = rec.allreduce2
    rec.allreduce2 = lambda a, b: (pairs.append((float(a), float(b))), orig(a, b))[1]
    rec.BH()
    out.update({
        "bh_dims": np.array([n, ntheta, ndist, nobj, niter]), "bh_obj_true": obj, "bh_prb_true": prb,
        "bh_pos_true": pos, "bh_pos_err": pos_err, "bh_data": data,
        "bh_obj": np.array(rec.vars["obj"]), "bh_prb": np.asarray(rec.vars["prb"]),
        "bh_pos": np.asarray(rec.vars["pos"]), "bh_proj": np.array(rec.vars["proj"]),
        "bh_topbottom": np.array(pairs, dtype="float64"),
    })
    np.savez_compressed(os.path.join(HERE, "rec.npz"), **out)


def realbh_cases(ns):
    """A short BH run with a real-valued object (obj_dtype float32): the
    reference's real-object path (rec_mpi.py:721, the real part of the
    back-propagated projections)."""
    n, ntheta, ndist, nobj, niter = 32, 12, 2, 32, 4
    rng = np.random.default_rng(17)
    args = rec_args(n, ntheta, ndist, nobj, niter)
    args.obj_dtype = "float32"
    rec = ns.rec_mpi.Rec(args)
    obj = np.ascontiguousarray(phantom(nobj, rng).real).astype("float32")
    prb = (1 + 0.1 * crand(rng, (ndist, n, n))).astype("complex64")
    pos = frand(rng, (ntheta, ndist, 2), 1.0)
    pos_err = frand(rng, (ntheta, ndist, 2), 0.2)
    rec.vars["obj"][:] = obj
    rec.vars["prb"][:] = ns.cp.array(prb)
    rec.vars["pos"][:] = ns.cp.array(pos)
    rec.gen_sqrt_data(rec.vars, rec.data)
    data = np.array(rec.data)
    rec.vars["obj"][:] = 0
    rec.vars["prb"][:] = ns.cp.array(1)
    rec.vars["pos"][:] = ns.cp.array(pos + pos_err)
    pairs = []
    orig = rec.allreduce2
    rec.allreduce2 = lambda a, b: (pairs.append((float(a), float(b))), orig(a, b))[1]
    rec.BH()
    out = {
        "rbh_dims": np.array([n, ntheta, ndist, nobj, niter]), "rbh_obj_true": obj, "rbh_prb_true": prb,
        "rbh_pos_true": pos, "rbh_pos_err": pos_err, "rbh_data": data,
        "rbh_obj": np.array(rec.vars["obj"]), "rbh_prb": np.asarray(rec.vars["prb"]),
        "rbh_pos": np.asarray(rec.vars["pos"]), "rbh_proj": np.array(rec.vars["proj"]),
        "rbh_topbottom": np.array(pairs, dtype="float64"),
    }
    np.savez_compressed(os.path.join(HERE, "realbh.npz"), **out)


def lap_cases(ns):
    """The 3-D Laplacian regulariser (rec_mpi.py:402-496): its gradient, Hessian
    form and energy at one point, and a 4-iteration BH run with lam_laplacian > 0."""
    out = {}
    n, ntheta, ndist, nobj = 32, 4, 1, 32
    rng = np.random.default_rng(3)
    args = rec_args(n, ntheta, ndist, nobj)
    args.lam_laplacian = 0.7
    rec = ns.rec_mpi.Rec(args)
    u = crand(rng, (nobj, nobj, nobj), 0.3)
    e = crand(rng, (nobj, nobj, nobj), 0.2)
    d1 = crand(rng, (nobj, nobj, nobj), 0.2)
    rec.vars["obj"][:] = u
    rec.etas["obj"][:] = e
    g = crand(rng, (nobj, nobj, nobj), 0.1)
    g0 = g.copy()
    rec.gradient_laplacian(g)
    out.update({"l_dims": np.array([n, ntheta, ndist, nobj]), "l_lam": np.array(args.lam_laplacian),
                "l_u": u, "l_e": e, "l_d1": d1, "l_g0": g0, "l_g": np.array(g),
                "l_h": np.array(float(rec.hessian_laplacian(d1))),
                "l_energy": np.array(float(rec._lap_energy_local()))})
    # BH with the regulariser
    n, ntheta, ndist, nobj, niter = 32, 12, 2, 32, 4
    rng = np.random.default_rng(7)
    args = rec_args(n, ntheta, ndist, nobj, niter)
    args.lam_laplacian = 2e-3
    rec = ns.rec_mpi.Rec(args)
    obj = phantom(nobj, rng)
    prb = (1 + 0.1 * crand(rng, (ndist, n, n))).astype("complex64")
    pos = frand(rng, (ntheta, ndist, 2), 1.0)
    pos_err = frand(rng, (ntheta, ndist, 2), 0.2)
    rec.vars["obj"][:] = obj
    rec.vars["prb"][:] = ns.cp.array(prb)
    rec.vars["pos"][:] = ns.cp.array(pos)
    rec.gen_sqrt_data(rec.vars, rec.data)
    rec.vars["obj"][:] = 0
    rec.vars["prb"][:] = ns.cp.array(1)
    rec.vars["pos"][:] = ns.cp.array(pos + pos_err)
    pairs = []
    orig = rec.allreduce2
    rec.allreduce2 = lambda a, b: (pairs.append((float(a), float(b))), orig(a, b))[1]
    rec.BH()
    out.update({
        "lbh_dims": np.array([n, ntheta, ndist, nobj, niter]), "lbh_lam": np.array(args.lam_laplacian),
        "lbh_obj": np.array(rec.vars["obj"]), "lbh_prb": np.asarray(rec.vars["prb"]),
        "lbh_pos": np.asarray(rec.vars["pos"]), "lbh_proj": np.array(rec.vars["proj"]),
        "lbh_topbottom": np.array(pairs, dtype="float64"),
    })
    np.savez_compressed(os.path.join(HERE, "lap.npz"), **out)


def _unit_mag_rec(ns, n, ntheta, ndist, nobj, distance, wavelength=7.3e-11, voxelsize=20e-9, niter=1):
    """The reference's Rec with the propagation geometry given directly and unit
    magnification: its constructor derives both from z1 and the focus distance
    (rec_mpi.py:55-60), so the propagator is replaced after construction."""
    args = rec_args(n, ntheta, ndist, nobj, niter)
    rec = ns.rec_mpi.Rec(args)
    rec.cl_prop = ns.propagation.Propagation(n, n, rec.nchunk, ndist, wavelength, voxelsize, distance)
    rec.norm_magnifications = np.ones(ndist)
    rec.eff_demagnifications[:] = 1
    return rec


def c1_data(ntheta, ndist, n):
    """Deterministic amplitudes for the adjoint chain of the small plain chain:
    0.8 + 0.1 k/17 with k = (7y + 13x + 5 angle + 3 distance) mod 17 (the
    residual against them is well away from zero, so the gradient carries no
    FP32 cancellation)."""
    a = np.arange(ntheta)[:, None, None, None]
    j = np.arange(ndist)[None, :, None, None]
    y = np.arange(n)[None, None, :, None]
    x = np.arange(n)[None, None, None, :]
    k = (7 * y + 13 * x + 5 * a + 3 * j) % 17
    return (0.8 + 0.1 * (k / 17)).astype("float32")


def c1_cases(ns):
    """The small plain chain at its full size: 128^3 ellipsoid phantom (20
    ellipsoids, k dx (-delta + i beta)), 180 angles, distances 3/4/5/6 mm at
    7.3e-11 m and 20 nm pixels, flat unit probe, positions uniform in +-2 px.
    Forward: proj = R(obj / norm_const) -> S(coeff(proj)) -> exp(i .) -> D(prb .)
    -> |.| (gen_sqrt_data, rec_mpi.py:882-897).  Adjoint: the full gradient
    (gF0..gF4, rec_mpi.py:305-353) at a perturbed state (object x 0.8, positions
    moved by up to 0.5 px) against the deterministic amplitudes of c1_data, so
    the test needs no stored data.  Full outputs are 20-50 MB each,
    so the fixture keeps an angle block (every 30th angle) of proj and the
    amplitudes, four slices of the object gradient, the probe and position
    gradients whole, and float64 checksums of every full array: its squared norm
    and its inner product with seeded unit normal weights over its float32 view
    (regenerated by the test from the seed 1000 + len(name))."""
    from holotomocupy_b200.synthetic import ellipsoid_phantom
    n, ntheta, ndist = 128, 180, 4
    distance = np.array([3e-3, 4e-3, 5e-3, 6e-3])
    obj = ellipsoid_phantom(n, 20, 11, device="cpu").numpy()
    rng = np.random.default_rng(12)
    pos = rng.uniform(-2, 2, (ntheta, ndist, 2)).astype("float32")
    pos_err = rng.uniform(-0.5, 0.5, (ntheta, ndist, 2)).astype("float32")
    prb = np.ones((ndist, n, n), "complex64")
    rec = _unit_mag_rec(ns, n, ntheta, ndist, n, distance)
    rec.vars["obj"][:] = obj
    rec.vars["prb"][:] = ns.cp.array(prb)
    rec.vars["pos"][:] = ns.cp.array(pos)
    amp = np.zeros((ntheta, ndist, n, n), "float32")
    rec.gen_sqrt_data(rec.vars, amp)
    proj = np.array(rec.vars["proj"])
    rec.data[:] = c1_data(ntheta, ndist, n)
    # the perturbed state, normalised as BH() has it (rec_mpi.py:149-158)
    rec.vars["obj"][:] = obj * np.float32(0.8) / rec.norm_const
    rec.vars["pos"][:] = ns.cp.array(pos + pos_err)
    rec.fwd_tomo(rec.vars["obj"], out=rec.proj_tmp)
    rec.vars["proj"][:] = rec.proj_tmp
    rec.gradients(rec.vars, rec.grads)
    # the position gradient is a per-image sum over nz * n pixels, which the
    # reference reduces in FP32 (3.9e-5 from FP64 here): keep the FP64 oracle's
    # value beside it
    from oracle import holo_oracle as O
    from holotomocupy_b200.synthetic import workload_args
    orc = O.Rec(workload_args(n, ntheta, ndist, niter=1, distances=tuple(distance)), "complex128")
    orc.eff_demagnifications[:] = 1
    orc.data[:] = c1_data(ntheta, ndist, n)
    v64 = {"obj": obj.astype("complex128") * np.float32(0.8) / np.sqrt(n / ntheta),
           "prb": np.ones((ndist, n, n), "complex128"), "pos": (pos + pos_err).astype("float64")}
    v64["proj"] = orc.fwd_tomo(v64["obj"])
    g64 = {k: np.zeros_like(x) for k, x in v64.items()}
    orc.gradients(v64, g64)
    blk = np.arange(0, ntheta, 30)
    sl = np.array([16, 63, 64, 100])
    out = {"dims": np.array([n, ntheta, ndist]), "distance": distance, "obj": obj, "pos": pos,
           "pos_err": pos_err, "blk": blk, "slices": sl, "proj_blk": proj[blk], "amp_blk": amp[blk],
           "grad_prb": np.asarray(rec.grads["prb"]), "grad_pos": np.asarray(rec.grads["pos"]),
           "grad_pos_fp64": g64["pos"],
           "grad_obj_sl": np.array(rec.grads["obj"])[sl], "grad_proj_blk": np.array(rec.grads["proj"])[blk]}
    full = {"proj": proj, "amp": amp, "grad_obj": np.array(rec.grads["obj"]),
            "grad_proj": np.array(rec.grads["proj"])}
    for k, v in full.items():
        vv = np.ascontiguousarray(v).view("float32").astype("float64")
        w = np.random.default_rng(1000 + len(k)).standard_normal(vv.shape)
        out[f"{k}_sq"] = np.array(np.sum(vv ** 2))
        out[f"{k}_wdot"] = np.array(np.sum(vv * w))
    np.savez_compressed(os.path.join(HERE, "c1.npz"), **out)


def prbfit_cases(ns):
    """The probe-fit regulariser lam_prbfit |||D prb| - ref||^2 (rec_mpi.py:365-398,
    815-835) at lam_prbfit = 2e-3: the full gradient, the Hessian form and the
    objective at one point, and a 4-iteration BH run, 32^3 x 12 angles x 2
    distances with ref = |D prb_true| (gen_sqrt_ref, rec_mpi.py:899-902)."""
    out = {}
    n, ntheta, ndist, nobj = 32, 6, 2, 32
    rng = np.random.default_rng(52)
    args = rec_args(n, ntheta, ndist, nobj)
    args.lam_prbfit = 2e-3
    rec = ns.rec_mpi.Rec(args)
    prb_true = (1 + 0.2 * crand(rng, (ndist, n, n))).astype("complex64")
    rec.gen_sqrt_ref(ns.cp.array(prb_true), rec.ref)
    prb = (prb_true + 0.1 * crand(rng, (ndist, n, n))).astype("complex64")
    obj = crand(rng, (nobj, nobj, nobj), 0.02)
    pos = frand(rng, (ntheta, ndist, 2), 0.8)
    data = (np.abs(frand(rng, (ntheta, ndist, n, n))) + 0.5).astype("float32")
    rec.data[:] = data
    rec.eff_demagnifications[:] = (1 + rec.shrink_nd) / ns.cp.array(rec.norm_magnifications[None, :])
    rec.vars["obj"][:] = obj
    rec.vars["prb"][:] = ns.cp.array(prb)
    rec.vars["pos"][:] = ns.cp.array(pos)
    rec.fwd_tomo(rec.vars["obj"], out=rec.proj_tmp)
    rec.vars["proj"][:] = rec.proj_tmp
    d1 = crand(rng, (ndist, n, n), 0.1)
    d2 = crand(rng, (ndist, n, n), 0.1)
    F = float(rec.min(rec.vars["prb"], rec.vars["obj"], rec.vars["pos"], rec.vars["proj"]))
    h12 = float(rec.hessian_prbfit(rec.vars["prb"], ns.cp.array(d1), ns.cp.array(d2)))
    h11 = float(rec.hessian_prbfit(rec.vars["prb"], ns.cp.array(d1), ns.cp.array(d1)))
    gp = ns.cp.zeros((ndist, n, n), "complex64")
    rec.gradient_prbfit(gp, rec.vars["prb"])
    rec.gradients(rec.vars, rec.grads)
    out.update({"p_dims": np.array([n, ntheta, ndist, nobj]), "p_lam": np.array(args.lam_prbfit),
                "p_prb_true": prb_true, "p_ref": np.asarray(rec.ref), "p_prb": prb, "p_obj": obj, "p_pos": pos,
                "p_data": data, "p_d1": d1, "p_d2": d2, "p_F": np.array(F), "p_h12": np.array(h12),
                "p_h11": np.array(h11), "p_gprb_fit": np.asarray(gp),
                "p_grad_prb": np.asarray(rec.grads["prb"]), "p_grad_obj": np.array(rec.grads["obj"]),
                "p_grad_pos": np.asarray(rec.grads["pos"])})
    # BH with the probe-fit term, from the golden BH problem of rec_cases
    n, ntheta, ndist, nobj, niter = 32, 12, 2, 32, 4
    rng = np.random.default_rng(7)
    args = rec_args(n, ntheta, ndist, nobj, niter)
    args.lam_prbfit = 2e-3
    rec = ns.rec_mpi.Rec(args)
    obj = phantom(nobj, rng)
    prb = (1 + 0.1 * crand(rng, (ndist, n, n))).astype("complex64")
    pos = frand(rng, (ntheta, ndist, 2), 1.0)
    pos_err = frand(rng, (ntheta, ndist, 2), 0.2)
    rec.vars["obj"][:] = obj
    rec.vars["prb"][:] = ns.cp.array(prb)
    rec.vars["pos"][:] = ns.cp.array(pos)
    rec.gen_sqrt_data(rec.vars, rec.data)
    rec.gen_sqrt_ref(ns.cp.array(prb), rec.ref)
    rec.vars["obj"][:] = 0
    rec.vars["prb"][:] = ns.cp.array(1)
    rec.vars["pos"][:] = ns.cp.array(pos + pos_err)
    pairs = []
    orig = rec.allreduce2
    rec.allreduce2 = lambda a, b: (pairs.append((float(a), float(b))), orig(a, b))[1]
    rec.BH()
    out.update({
        "pbh_dims": np.array([n, ntheta, ndist, nobj, niter]), "pbh_lam": np.array(args.lam_prbfit),
        "pbh_ref": np.asarray(rec.ref),
        "pbh_obj": np.array(rec.vars["obj"]), "pbh_prb": np.asarray(rec.vars["prb"]),
        "pbh_pos": np.asarray(rec.vars["pos"]), "pbh_proj": np.array(rec.vars["proj"]),
        "pbh_topbottom": np.array(pairs, dtype="float64"),
    })
    np.savez_compressed(os.path.join(HERE, "prbfit.npz"), **out)


def rectomo_cases(ns):
    """Tomo.rec_tomo (tomo.py:185-210), the conjugate-gradient initial guess,
    on a sinogram of the small ellipsoid phantom: 1 and 6 iterations, complex
    and real data."""
    out = {}
    for (n, nz, ntheta, niter, dt, tag) in [(32, 4, 40, 6, "complex64", "a"), (48, 3, 64, 6, "float32", "b")]:
        rng = np.random.default_rng(900 + n)
        theta = np.linspace(0, np.pi, ntheta, endpoint=False).astype("float32")
        t = ns.tomo.Tomo(n, nz, theta, 1)
        obj = phantom(n, rng)[n // 2 - nz // 2: n // 2 - nz // 2 + nz]
        obj = obj if dt == "complex64" else obj.real.astype("float32").copy()
        d = t.R(ns.cp.array(obj)).get()
        d = (d + 0.01 * np.abs(d).max() * (crand(rng, d.shape) if dt == "complex64" else frand(rng, d.shape))
             ).astype(dt)
        u = t.rec_tomo(ns.cp.array(d), niter).get()
        u1 = t.rec_tomo(ns.cp.array(d), 1).get()
        out.update({f"{tag}_dims": np.array([n, nz, ntheta, niter]), f"{tag}_theta": theta, f"{tag}_d": d,
                    f"{tag}_u": u, f"{tag}_u1": u1})
    np.savez_compressed(os.path.join(HERE, "rectomo.npz"), **out)


def nfp_args(n, nobj, ntheta, dt, niter=1):
    return types.SimpleNamespace(
        energy=17.1, detector_pixelsize=3e-6, focustodetectordistance=1.217, z1=8.245e-3,
        ntheta=ntheta, nz=n, n=n, nzobj=nobj, nobj=nobj, obj_dtype=dt, rho=[1, 0.5, 0.1],
        niter=niter, nchunk=ntheta, vis_step=-1, err_step=-1, start_iter=0,
        comm=sys.modules["mpi4py"].MPI.COMM_WORLD)


def nfp_cases(ns):
    """RecNFP (rec_nfp_mpi.py:20-469), near-field ptychography: one 2-D
    projection scanned at ntheta positions, one distance.  The gradient and the
    Hessian forms at one point, and a 4-iteration BH run from a flat probe, a
    zero projection and perturbed positions; complex and real projections."""
    out = {}
    for dt, tag in (("complex64", "c"), ("float32", "f")):
        n, nobj, ntheta, niter = 32, 48, 8, 4
        rng = np.random.default_rng(60 + len(dt))
        rec = ns.rec_nfp_mpi.RecNFP(nfp_args(n, nobj, ntheta, dt, niter))
        ph = phantom(nobj, rng)[nobj // 2]
        proj = (ph if dt == "complex64" else ph.real.astype("float32")).copy()
        prb = (1 + 0.2 * crand(rng, (n, n))).astype("complex64")
        pos = rng.uniform(-2, 2, (ntheta, 2)).astype("float32")
        pos_err = rng.uniform(-0.3, 0.3, (ntheta, 2)).astype("float32")
        C = lambda x: ns.cp.array(x)
        rec.vars["prb"][:] = C(prb)
        rec.vars["proj"][:] = C(proj)
        rec.vars["pos"][:] = C(pos)
        rec.gen_sqrt_data(rec.vars, rec.data)
        data = np.array(rec.data)
        # gradient and Hessian forms at a perturbed point
        mk = (lambda sh, sc: crand(rng, sh, sc)) if dt == "complex64" else (lambda sh, sc: frand(rng, sh, sc))
        v = {"prb": C(prb + 0.1 * crand(rng, (n, n))), "proj": C((proj * 0.7).astype(dt)),
             "pos": C((pos + pos_err).astype("float32"))}
        g = {"prb": C(0.1 * crand(rng, (n, n))), "proj": C(mk((nobj, nobj), 0.05)),
             "pos": C(frand(rng, (ntheta, 2), 0.3))}
        e = {"prb": C(0.1 * crand(rng, (n, n))), "proj": C(mk((nobj, nobj), 0.05)),
             "pos": C(frand(rng, (ntheta, 2), 0.3))}
        grads = {"prb": ns.cp.zeros((n, n), "complex64"), "proj": ns.cp.zeros((nobj, nobj), dt),
                 "pos": ns.cp.zeros((ntheta, 2), "float32")}
        rec.gradients(v, grads)
        F = float(rec.min(v["prb"], v["proj"], v["pos"]))
        h_ge = float(rec.hessian(v, g, e))
        h_ee = float(rec.hessian(v, e, e))
        out.update({f"{tag}_dims": np.array([n, nobj, ntheta, niter]), f"{tag}_data": data,
                    f"{tag}_prb_true": prb, f"{tag}_proj_true": proj, f"{tag}_pos_true": pos,
                    f"{tag}_pos_err": pos_err, f"{tag}_F": np.array(F), f"{tag}_h_ge": np.array(h_ge),
                    f"{tag}_h_ee": np.array(h_ee)})
        for name, d in (("v", v), ("g", g), ("e", e), ("grad", grads)):
            for k, x in d.items():
                out[f"{tag}_{name}_{k}"] = np.array(x)
        # BH from a flat probe and a zero projection
        rec.vars["prb"][:] = C(np.ones((n, n), "complex64"))
        rec.vars["proj"][:] = 0
        rec.vars["pos"][:] = C((pos + pos_err).astype("float32"))
        pairs = []
        orig = rec.allreduce2
        rec.allreduce2 = lambda a, b: (pairs.append((float(a), float(b))), orig(a, b))[1]
        rec.BH()
        out.update({f"{tag}_bh_{k}": np.array(rec.vars[k]) for k in ("prb", "proj", "pos")})
        out[f"{tag}_bh_topbottom"] = np.array(pairs, dtype="float64")
    np.savez_compressed(os.path.join(HERE, "nfp.npz"), **out)


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else None
    if src is None:
        raise SystemExit("usage: make_golden.py <reference src dir>")
    ns = load_reference(src)
    which = sys.argv[2:] or ["tomo", "prop", "shift", "rec", "realbh", "lap", "sback", "c1", "prbfit", "rectomo",
                             "nfp"]
    for w in which:
        {"tomo": tomo_cases, "prop": prop_cases, "shift": shift_cases, "rec": rec_cases, "realbh": realbh_cases,
         "lap": lap_cases,
         "sback": sback_cases, "c1": c1_cases, "prbfit": prbfit_cases, "rectomo": rectomo_cases,
         "nfp": nfp_cases}[w](ns)
        print("wrote", w)


if __name__ == "__main__":
    main()
