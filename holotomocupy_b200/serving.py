"""Serving many BH reconstructions on one GPU with continuous batching.

The reference runs one reconstruction per job (``experimental/*/step6.py``
drives ``Rec.BH`` once).  Here a persistent loop keeps several
reconstructions resident at once:

* requests wait in arrival order and are admitted as soon as their estimated
  device memory fits the HBM budget and a slot is free;
* each admitted request owns a CUDA stream and a ``Rec`` whose object, probe,
  position and cascade state stay on the device;
* its first iteration runs eagerly; the steady-state iteration, whose step
  sizes stay on the device, is recorded once into a CUDA graph and then
  replayed with one launch per iteration, so iterations of different requests
  overlap on the GPU;
* the loop never blocks on one request: it polls each stream's last event,
  records the per-iteration latency, launches the next iteration or retires
  the request (results copied to the host);
* a retired request's device memory is released lazily -- when an admission
  needs it, or when the loop ends -- because releasing it synchronises the
  whole device and would drain the other requests' queued work.

Every request's arithmetic is the same as running it alone (the same kernels
in the same order on its own buffers).
"""
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .rec import Rec


def estimate_bytes(args):
    """Device bytes one reconstruction of these sizes holds: the arrays of
    Rec (vars/grads/etas, coefficients, data), the fused-cascade workspace,
    the Radon workspace and the propagator tables, plus 10 % and 64 MiB."""
    n, nz, nobj, nzobj, ntheta, ndist = args.n, args.nz, args.nobj, args.nzobj, args.ntheta, args.ndist
    c8 = 8
    obj = nzobj * nobj * nobj * c8
    proj = ntheta * nzobj * nobj * c8
    img = ntheta * ndist * nz * n
    total = 3 * obj + 7 * proj                                  # obj x3; proj, coefficients, gradient x7
    total += img * 4 + 4 * ndist * nz * n * c8                  # data, probe arrays
    total += 3 * img * c8 + max(img, ntheta * ndist * nz * nobj) * c8   # x0, P, two spectra / S^T rows
    zb = 8 if 2 * nobj <= 1024 else (4 if 2 * nobj == 2048 else 2)
    nzp = -(-nzobj // zb) * zb
    total += nzp * 6 * nobj * nobj * c8 + nzp * ntheta * nobj * c8   # Radon workspace
    total += ndist * 4 * nz * n * c8 + ndist * nz * n * c8          # Fresnel tables
    return int(total * 1.1) + (64 << 20)


@dataclass
class Request:
    """One reconstruction: ``args`` as for Rec, measured amplitudes, initial
    state (host or device tensors), number of BH iterations and an arrival
    time in seconds from the start of Server.run."""
    rid: int
    args: object
    data: torch.Tensor
    prb0: torch.Tensor
    pos0: torch.Tensor
    obj0: torch.Tensor = None
    niter: int = 16
    arrival: float = 0.0
    # filled by the server
    latencies_ms: list = field(default_factory=list)
    result: dict = None
    t_admit: float = None
    t_done: float = None


class _Slot:
    def __init__(self, req, stream):
        self.req = req
        self.stream = stream
        self.rec = None
        self.it = 0
        self.busy = False
        self.ev0 = torch.cuda.Event(enable_timing=True)
        self.ev1 = torch.cuda.Event(enable_timing=True)
        self.bytes = estimate_bytes(req.args)


class Server:
    """Persistent request loop (continuous batching of BH reconstructions)."""

    def __init__(self, budget_bytes=None, max_active=16, graphs=True, device=None):
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            budget_bytes = int(0.8 * free)
        self.budget = budget_bytes
        self.max_active = max_active
        self.graphs = graphs
        self.queue = []
        self.done = []
        self.peak_bytes = 0
        self.max_concurrent = 0
        self.used_bytes = 0       # estimated bytes of the active and not yet released requests
        # one stream per slot, reused by the requests that follow so that the
        # caching allocator hands their freed blocks to the next request
        self._streams = [torch.cuda.Stream(device=self.device) for _ in range(max_active)]

    def submit(self, req):
        if estimate_bytes(req.args) > self.budget:
            raise ValueError(f"request {req.rid} needs more than the HBM budget ({self.budget} bytes)")
        self.queue.append(req)

    # ----------------------------------------------------------- phases
    def _admit(self, slot):
        r = slot.req
        with torch.cuda.stream(slot.stream):
            rec = Rec(r.args)
            rec.data.copy_(r.data, non_blocking=True)
            if r.obj0 is not None:
                rec.vars["obj"].copy_(r.obj0, non_blocking=True)
            rec.vars["prb"].copy_(r.prb0, non_blocking=True)
            rec.vars["pos"].copy_(r.pos0, non_blocking=True)
            rec.bh_setup()
        slot.rec = rec

    def _launch(self, slot):
        rec = slot.rec
        with torch.cuda.stream(slot.stream):
            slot.ev0.record(slot.stream)
            if slot.it == 0 or not self.graphs:
                rec.bh_iteration(rec.start_iter + slot.it, sync=False)
            else:
                if rec._graph is None:
                    rec.capture_iteration()
                rec.replay_iteration()
            slot.ev1.record(slot.stream)
        slot.it += 1
        slot.busy = True

    def _retire(self, slot, t0):
        r, rec = slot.req, slot.rec
        with torch.cuda.stream(slot.stream):
            rec.bh_finish()
            out = {k: rec.vars[k].to("cpu", non_blocking=True) for k in ("obj", "prb", "pos")}
        slot.stream.synchronize()
        out["history"] = rec.bh_history()
        r.result = out
        r.t_done = time.perf_counter() - t0
        rec.release_graph()
        self._retired.append((rec, slot.bytes))   # freed lazily (see _release)
        slot.rec = None
        self.done.append(r)

    def _release(self):
        """Free the retired reconstructions' device memory (synchronises the
        device); returns the bytes released."""
        freed = sum(b for _, b in self._retired)
        torch.cuda.synchronize(self.device)
        for rec, _ in self._retired:
            rec.close()
        self._retired.clear()
        # the library allocates outside torch's caching allocator: hand the
        # cached blocks back so that its next allocations find them
        torch.cuda.empty_cache()
        return freed

    # ------------------------------------------------------------- loop
    def run(self, realtime=True):
        """Serve every submitted request; returns them with results and
        per-iteration latencies.  realtime=False admits requests regardless of
        their arrival times."""
        pending = sorted(self.queue, key=lambda q: q.arrival)
        self.queue = []
        active = []
        self.used_bytes = 0
        self._retired = []
        t0 = time.perf_counter()
        while pending or active:
            now = time.perf_counter() - t0
            while pending and len(active) < self.max_active and (not realtime or pending[0].arrival <= now):
                need = estimate_bytes(pending[0].args)
                if self.used_bytes + need > self.budget and self._retired:
                    self.used_bytes -= self._release()
                if active and self.used_bytes + need > self.budget:
                    break
                r = pending.pop(0)
                slot = _Slot(r, self._streams.pop())
                r.t_admit = time.perf_counter() - t0
                try:
                    self._admit(slot)
                except (torch.OutOfMemoryError, _lib.HoloError) as err:
                    # the estimate fitted but the device did not (fragmentation,
                    # other users of the GPU): free what is retired and retry
                    # once the active requests have made room
                    self._streams.append(slot.stream)
                    pending.insert(0, r)
                    self.used_bytes -= self._release()
                    if not active or "out of memory" not in str(err):
                        raise
                    break
                active.append(slot)
                self.used_bytes += slot.bytes
                self.peak_bytes = max(self.peak_bytes, self.used_bytes)
                self.max_concurrent = max(self.max_concurrent, len(active))
            progressed = False
            for slot in list(active):
                if slot.busy:
                    if not slot.ev1.query():
                        continue
                    slot.req.latencies_ms.append(slot.ev0.elapsed_time(slot.ev1))
                    slot.busy = False
                    progressed = True
                if slot.it >= slot.req.niter:
                    self._retire(slot, t0)
                    active.remove(slot)
                    self._streams.append(slot.stream)
                    progressed = True
                    continue
                self._launch(slot)
                progressed = True
            if not progressed:
                if not active and pending and realtime:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - (time.perf_counter() - t0))))
                else:
                    time.sleep(20e-6)
        self.wall = time.perf_counter() - t0
        self.used_bytes -= self._release()
        return self.done

    @staticmethod
    def completion_stats(reqs, realtime=True):
        """p50/p99 of the per-request completion latency: arrival (or the
        start of the run when arrivals are ignored) to the result on the host."""
        lat = np.array([r.t_done - (r.arrival if realtime else 0.0) for r in reqs if r.t_done is not None] or [0.0])
        return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99))}

    @staticmethod
    def latency_stats(reqs):
        """p50/p99 of the per-iteration latencies (first iterations excluded:
        they include the graph recording)."""
        lat = np.array([x for r in reqs for x in r.latencies_ms[1:]] or [0.0])
        return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "iterations": int(sum(len(r.latencies_ms) for r in reqs))}


def run_plain(reqs, realtime=False, done_times=None):
    """The same requests one at a time through Rec.BH's host-synchronised
    iteration (no graphs, no overlap), in arrival order; realtime=True waits
    for each arrival.  Returns (wall seconds, per-iteration latencies in ms,
    results); done_times (a list) receives each request's completion time in
    seconds from the start."""
    lat = []
    results = []
    t0 = time.perf_counter()
    for r in sorted(reqs, key=lambda q: q.arrival):
        if realtime:
            time.sleep(max(0.0, r.arrival - (time.perf_counter() - t0)))
        rec = Rec(r.args)
        rec.data.copy_(r.data)
        if r.obj0 is not None:
            rec.vars["obj"].copy_(r.obj0)
        rec.vars["prb"].copy_(r.prb0)
        rec.vars["pos"].copy_(r.pos0)
        rec.bh_setup()
        for i in range(r.niter):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            rec.bh_iteration(rec.start_iter + i)
            e1.record()
            e1.synchronize()
            lat.append(e0.elapsed_time(e1))
        rec.bh_finish()
        results.append({k: rec.vars[k].cpu() for k in ("obj", "prb", "pos")})
        if done_times is not None:
            done_times.append(time.perf_counter() - t0)
        rec.close()
        del rec
    torch.cuda.synchronize()
    return time.perf_counter() - t0, lat, results
