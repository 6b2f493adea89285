"""Serving: reconstructions admitted into the persistent loop (own streams,
device-side step sizes, graph-replayed iterations, overlapping on the GPU)
give the same result as each run alone through the plain host-synchronised
Rec.BH iteration.  Bound: rel L2 <= 1e-5 (the same kernels on the same data;
only the order in which independent requests reach the GPU differs)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _requests(host=False):
    from holotomocupy_b200.serving import Request
    from holotomocupy_b200.synthetic import make_problem
    reqs = []
    for rid, (n, ntheta, seed) in enumerate([(64, 112, 11), (128, 224, 12), (64, 112, 13)]):
        args, data, prb0, pos0, _ = make_problem(n, ntheta, 4, seed, host=host)
        reqs.append(Request(rid=rid, args=args, data=data, prb0=prb0, pos0=pos0, niter=5, arrival=0.0))
    return reqs


@pytest.mark.parametrize("host", [False, True])
@pytest.mark.parametrize("workers", [True, False])
def test_served_results_equal_alone(host, workers):
    """Admissions and retirements on the host worker threads (workers=True)
    or inline in the launch loop give the same results."""
    from holotomocupy_b200.serving import Server, run_plain
    reqs = _requests(host)
    _, _, alone = run_plain(reqs)
    srv = Server(max_active=8, host_workers=workers)
    for r in reqs:
        srv.submit(r)
    done = {r.rid: r for r in srv.run(realtime=False)}
    assert srv.max_concurrent == 3
    for r, ref in zip(reqs, alone):
        got = done[r.rid].result
        for k in ("obj", "prb", "pos"):
            assert rel_l2(got[k].numpy(), ref[k].numpy()) < 1e-5, (r.rid, k)
        assert len(got["history"]) == r.niter
        assert len(done[r.rid].latencies_ms) == r.niter


def test_admission_respects_the_hbm_budget():
    """With a budget that holds one 128^3 request at a time, requests run one
    after another and still give the same results."""
    from holotomocupy_b200.serving import Server, estimate_bytes, run_plain
    reqs = _requests()
    _, _, alone = run_plain(reqs)
    big = max(estimate_bytes(r.args) for r in reqs)
    srv = Server(budget_bytes=big + 1, max_active=8)
    for r in reqs:
        srv.submit(r)
    done = {r.rid: r for r in srv.run(realtime=False)}
    assert srv.peak_bytes <= big + 1
    for r, ref in zip(reqs, alone):
        assert rel_l2(done[r.rid].result["obj"].numpy(), ref["obj"].numpy()) < 1e-5
    with pytest.raises(ValueError):
        Server(budget_bytes=1).submit(reqs[0])


def test_device_scalar_iteration_matches_host_iteration():
    """Rec.bh_iteration(sync=False) (alpha, beta on the device) and its graph
    replay equal the host-scalar iteration step for step."""
    from holotomocupy_b200.rec import Rec
    from holotomocupy_b200.synthetic import make_problem
    args, data, prb0, pos0, _ = make_problem(64, 112, 4, 21)
    out = []
    st = torch.cuda.Stream()
    for mode in ("host", "device", "graph"):
        with torch.cuda.stream(st):
            rec = Rec(args)
            rec.data.copy_(data)
            rec.vars["prb"].copy_(prb0)
            rec.vars["pos"].copy_(pos0)
            rec.bh_setup()
            hist = []
            for i in range(4):
                if mode == "host":
                    hist.append(rec.bh_iteration(i))
                elif mode == "device" or i == 0:
                    rec.bh_iteration(i, sync=False)
                else:
                    if rec._graph is None:
                        rec.capture_iteration()
                    rec.replay_iteration()
            if mode != "host":
                hist = [(a, b) for a, b in rec.bh_history()]
            rec.bh_finish()
            out.append((hist, {k: rec.vars[k].cpu().numpy() for k in ("obj", "prb", "pos")}))
            rec.release_graph()
    h0, v0 = out[0]
    for h, v in out[1:]:
        np.testing.assert_allclose(np.array(h), np.array(h0), rtol=1e-9)
        for k in v0:
            assert rel_l2(v[k], v0[k]) < 1e-6


def test_out_of_memory_admission_returns_the_released_bytes():
    """An admission that runs out of device memory while a retired request is
    still held releases it and takes its bytes off the ledger: after the run
    the ledger is back at zero and every request finished with the result it
    has alone.  Two slots for three requests: the small first request retires
    while the 128^3 one runs, and the third request's first admission attempt
    fails (injected), with the retired request unreleased."""
    from holotomocupy_b200.serving import Server, estimate_bytes, run_plain
    reqs = _requests()
    _, _, alone = run_plain(reqs)
    big = max(estimate_bytes(r.args) for r in reqs)
    srv = Server(budget_bytes=4 * big, max_active=2, reuse=False)
    admit = srv._admit
    state = {"injected": False}

    def flaky(slot):
        if not state["injected"] and srv._retired:
            state["injected"] = True
            raise torch.OutOfMemoryError("CUDA out of memory (injected)")
        return admit(slot)

    srv._admit = flaky
    for r in reqs:
        srv.submit(r)
    done = {r.rid: r for r in srv.run(realtime=False)}
    assert state["injected"]
    assert srv.used_bytes == 0
    for r, ref in zip(reqs, alone):
        assert rel_l2(done[r.rid].result["obj"].numpy(), ref["obj"].numpy()) < 1e-5


def test_reused_rec_gives_the_result_alone():
    """One slot: the third request (the first one's arguments) takes over the
    first request's retired Rec (Rec.reset) and still gives its result alone;
    the ledger ends at zero."""
    from holotomocupy_b200.serving import Server, run_plain
    reqs = _requests()
    _, _, alone = run_plain(reqs)
    srv = Server(max_active=1)
    for r in reqs:
        srv.submit(r)
    done = {r.rid: r for r in srv.run(realtime=False)}
    assert srv.reused == 1
    assert srv.used_bytes == 0
    for r, ref in zip(reqs, alone):
        got = done[r.rid].result
        for k in ("obj", "prb", "pos"):
            assert rel_l2(got[k].numpy(), ref[k].numpy()) < 1e-5, (r.rid, k)
        assert len(got["history"]) == r.niter


def test_real_object_iterations_are_launched_not_recorded():
    """A real-valued (float32) object's iteration allocates temporaries, so it
    is never recorded into a graph: capture_iteration() raises before any
    recording starts; the device-scalar iteration matches the host one step
    for step; BH(mode="graph") iterates as "host"; the server serves such a
    request beside a complex one with the results each has alone."""
    import copy
    from holotomocupy_b200.rec import Rec
    from holotomocupy_b200.serving import Request, Server, run_plain
    from holotomocupy_b200.synthetic import make_problem
    args, data, prb0, pos0, _ = make_problem(64, 112, 4, 31)
    args.obj_dtype = "float32"
    out = []
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        for mode in ("host", "device"):
            rec = Rec(args)
            assert not rec.graphable
            rec.data.copy_(data)
            rec.vars["prb"].copy_(prb0)
            rec.vars["pos"].copy_(pos0)
            rec.bh_setup()
            hist = [rec.bh_iteration(i, sync=mode == "host") for i in range(4)]
            if mode == "device":
                hist = list(rec.bh_history())
                with pytest.raises(ValueError):
                    rec.capture_iteration()
                assert rec._graph is None
            rec.bh_finish()
            out.append((hist, {k: rec.vars[k].cpu().numpy() for k in ("obj", "prb", "pos")}))
            rec.close()
    (h0, v0), (h1, v1) = out
    np.testing.assert_allclose(np.array(h1), np.array(h0), rtol=1e-9)
    for k in v0:
        assert rel_l2(v1[k], v0[k]) < 1e-6, k
    res = []
    for mode in ("host", "graph"):
        rec = Rec(args)
        rec.data.copy_(data)
        rec.vars["prb"].copy_(prb0)
        rec.vars["pos"].copy_(pos0)
        record = []
        rec.BH(niter=4, record=record, mode=mode)
        assert rec._graph is None and len(record) == 4
        res.append({k: rec.vars[k].cpu().numpy() for k in ("obj", "prb", "pos")})
        rec.close()
    for k in res[0]:
        assert rel_l2(res[1][k], res[0][k]) < 1e-6, k
    cargs, cdata, cprb0, cpos0, _ = make_problem(64, 112, 4, 32)
    reqs = [Request(rid=0, args=copy.copy(args), data=data, prb0=prb0, pos0=pos0, niter=5, arrival=0.0),
            Request(rid=1, args=cargs, data=cdata, prb0=cprb0, pos0=cpos0, niter=5, arrival=0.0)]
    _, _, alone = run_plain(reqs)
    srv = Server(max_active=4)
    for r in reqs:
        srv.submit(r)
    done = {r.rid: r for r in srv.run(realtime=False)}
    for r, ref in zip(reqs, alone):
        got = done[r.rid].result
        assert got["obj"].dtype == (torch.float32 if r.rid == 0 else torch.complex64)
        for k in ("obj", "prb", "pos"):
            assert rel_l2(got[k].numpy(), ref[k].numpy()) < 1e-5, (r.rid, k)
