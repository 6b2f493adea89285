"""Near-field ptychography (RecNFP) on the GPU against the reference's own
rec_nfp_mpi.py (golden vectors, tests/golden/nfp.npz): synthetic amplitudes,
the objective, the gradient and the Hessian forms at one point, and a
4-iteration BH run (state and step sizes), complex and real projections.
Bound: rel 1e-5 (the BH step sizes 1e-4, as for Rec)."""
import types

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def nfp_args(n, nobj, ntheta, dt, niter=1):
    return types.SimpleNamespace(
        energy=17.1, detector_pixelsize=3e-6, focustodetectordistance=1.217, z1=8.245e-3,
        ntheta=ntheta, nz=n, n=n, nzobj=nobj, nobj=nobj, obj_dtype=dt, rho=[1, 0.5, 0.1],
        niter=niter, nchunk=ntheta, vis_step=-1, err_step=-1, start_iter=0)


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("tag,dt", [("c", "complex64"), ("f", "float32")])
def test_nfp_cascade_matches_reference(golden, tag, dt):
    from holotomocupy_b200 import RecNFP
    g = golden("nfp")
    n, nobj, ntheta, niter = [int(v) for v in g[f"{tag}_dims"]]
    rec = RecNFP(nfp_args(n, nobj, ntheta, dt))
    truth = {"prb": cuda(g[f"{tag}_prb_true"]), "proj": cuda(g[f"{tag}_proj_true"]), "pos": cuda(g[f"{tag}_pos_true"])}
    rec.gen_sqrt_data(truth, rec.data)
    assert rel_l2(rec.data.cpu().numpy(), g[f"{tag}_data"]) < TOL
    rec.data[:] = cuda(g[f"{tag}_data"])
    V = lambda name: {k: cuda(g[f"{tag}_{name}_{k}"]) for k in ("prb", "proj", "pos")}
    v, gr, et = V("v"), V("g"), V("e")
    assert abs(rec.min(v["prb"], v["proj"], v["pos"]) / float(g[f"{tag}_F"]) - 1) < TOL
    out = {k: torch.zeros_like(x) for k, x in v.items()}
    rec.gradients(v, out)
    for k in ("prb", "proj", "pos"):
        assert rel_l2(out[k].cpu().numpy(), g[f"{tag}_grad_{k}"]) < TOL, k
    assert abs(rec.hessian(v, gr, et) / float(g[f"{tag}_h_ge"]) - 1) < TOL
    assert abs(rec.hessian(v, et, et) / float(g[f"{tag}_h_ee"]) - 1) < TOL


@pytest.mark.parametrize("tag,dt", [("c", "complex64"), ("f", "float32")])
def test_nfp_bh_matches_reference(golden, tag, dt):
    from holotomocupy_b200 import RecNFP
    g = golden("nfp")
    n, nobj, ntheta, niter = [int(v) for v in g[f"{tag}_dims"]]
    rec = RecNFP(nfp_args(n, nobj, ntheta, dt, niter))
    rec.data[:] = cuda(g[f"{tag}_data"])
    rec.vars["prb"][:] = 1
    rec.vars["proj"][:] = 0
    rec.vars["pos"][:] = cuda(g[f"{tag}_pos_true"] + g[f"{tag}_pos_err"])
    record = []
    rec.BH(record=record)
    tb = g[f"{tag}_bh_topbottom"]
    ref_alpha = [tb[0, 0] / tb[0, 1]] + [tb[2 * i, 0] / tb[2 * i, 1] for i in range(1, niter)]
    ref_beta = [0.0] + [tb[2 * i - 1, 0] / tb[2 * i - 1, 1] for i in range(1, niter)]
    for (i, a, b), ra, rb in zip(record, ref_alpha, ref_beta):
        assert abs(a / ra - 1) < 1e-4, (i, a, ra)
        if rb:
            assert abs(b / rb - 1) < 1e-4, (i, b, rb)
    for k in ("prb", "proj", "pos"):
        assert rel_l2(rec.vars[k].cpu().numpy(), g[f"{tag}_bh_{k}"]) < TOL, k


def test_nfp_graph_iteration_matches_host(golden):
    """BH(mode="graph"): step sizes on the device (ht_bh_scalars, ht_axpby_dev)
    and the steady-state iteration replayed from a CUDA graph give the step
    sizes (rtol 1e-9) and the state (rel L2 1e-6) of the host-scalar BH."""
    from holotomocupy_b200 import RecNFP
    g = golden("nfp")
    tag, dt = "c", "complex64"
    n, nobj, ntheta, niter = [int(v) for v in g[f"{tag}_dims"]]
    out = []
    st = torch.cuda.Stream()
    for mode in ("host", "graph"):
        with torch.cuda.stream(st):
            rec = RecNFP(nfp_args(n, nobj, ntheta, dt, niter))
            rec.data[:] = cuda(g[f"{tag}_data"])
            rec.vars["prb"][:] = 1
            rec.vars["proj"][:] = 0
            rec.vars["pos"][:] = cuda(g[f"{tag}_pos_true"] + g[f"{tag}_pos_err"])
            record = []
            rec.BH(record=record, mode=mode)
            out.append((np.array([(a, b) for _, a, b in record]),
                        {k: rec.vars[k].cpu().numpy() for k in ("prb", "proj", "pos")}))
            rec.close()
    (h0, v0), (h1, v1) = out
    assert h1.shape == (niter, 2)
    np.testing.assert_allclose(h1, h0, rtol=1e-9)
    for k in v0:
        assert rel_l2(v1[k], v0[k]) < 1e-6, k
