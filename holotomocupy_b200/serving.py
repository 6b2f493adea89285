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
* the loop never blocks on one request: it polls each stream's events,
  records the per-iteration latencies and keeps up to ``depth`` iterations of
  every request queued on its stream, so that its own pauses do not leave the
  GPU without work;
* the host work around the iterations -- building a request's Rec, uploading
  its data, the set-up pass; the final pass and copying the results to the
  host -- runs on two worker threads (admissions, retirements), overlapping
  the other requests' iterations: per request it is 0.1-0.9 s against
  0.04-2 s of iterations, a third of the plain form's time;
* a retired request's device memory is released lazily -- when an admission
  needs it, or when the loop ends -- because releasing it synchronises the
  whole device and would drain the other requests' queued work.

Every request's arithmetic is the same as running it alone (the same kernels
in the same order on its own buffers).
"""
import sys
import threading
import time
from collections import deque
from concurrent.futures import Future, ThreadPoolExecutor
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


def args_key(args):
    """Hashable identity of a request's Rec arguments: requests with equal
    keys can share one Rec, one after the other."""
    import hashlib
    items = []
    for k, v in sorted(vars(args).items()):
        if isinstance(v, torch.Tensor):
            v = v.detach().cpu().numpy()
        if isinstance(v, (np.ndarray, list, tuple)):
            a = np.asarray(v)
            items.append((k, a.dtype.str, a.shape, hashlib.sha1(np.ascontiguousarray(a).tobytes()).hexdigest()))
        else:
            items.append((k, repr(v)))
    return tuple(items)


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


class _Inline:
    """An executor that runs each job at once on the calling thread."""

    def submit(self, fn, *args):
        f = Future()
        try:
            f.set_result(fn(*args))
        except BaseException as e:  # noqa: BLE001 - handed to the caller through the future
            f.set_exception(e)
        return f


class _Slot:
    def __init__(self, req, stream, key, nbytes):
        self.req = req
        self.stream = stream
        self.rec = None
        self.it = 0              # iterations launched
        self.inflight = deque()  # (start, end) event pairs of the queued iterations, oldest first
        self.bytes = nbytes      # estimate_bytes(req.args)
        self.job = None          # the host worker's admission or retirement of this request
        self.key = key           # args_key(req.args)
        self.reused = None       # a retired request's (rec, bytes, key) this one takes over
        self.state = "admitting"  # -> "running" -> "retiring"


class Server:
    """Persistent request loop (continuous batching of BH reconstructions).

    graphs: replay a request's steady-state iteration from a CUDA graph
    (complex objects; a real-object request launches each iteration, with
    the same device-side step sizes, since its iteration allocates).
    depth: iterations a request may have queued on its stream.  host_workers:
    admissions (building the Rec, uploading, the set-up pass) and retirements
    (the final pass, copying the results to the host) run on two host worker
    threads, so that the launch loop keeps feeding the GPU meanwhile; False
    runs them inline in the loop.  reuse: a request takes over the Rec of a
    retired request with the same arguments (Rec.reset) instead of freeing
    it and allocating its own.  max_active: requests resident at once; more
    than a few make their working sets compete for L2 (a saturated stream of
    64 reconstructions of 128^3-512^3: 28.6 s with 4, 29-32 s with 8)."""

    def __init__(self, budget_bytes=None, max_active=4, graphs=True, device=None, depth=4, host_workers=True,
                 reuse=True):
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            budget_bytes = int(0.8 * free)
        self.budget = budget_bytes
        self.max_active = max_active
        self.graphs = graphs
        self.depth = max(1, int(depth))
        self.host_workers = host_workers
        self.reuse = reuse
        self.queue = []
        self.done = []
        self.peak_bytes = 0
        self.max_concurrent = 0
        self.used_bytes = 0       # estimated bytes of the active and not yet released requests
        # one stream per slot, reused by the requests that follow so that the
        # caching allocator hands their freed blocks to the next request
        self._streams = [torch.cuda.Stream(device=self.device) for _ in range(max_active)]
        # Device memory is allocated (admissions) and freed (releases, which
        # synchronise the device) only under this lock, and a graph is
        # recorded only while the loop holds it: a free inside a recording
        # would end the recording with an error.  The loop never waits for
        # it -- when a worker holds it, the iteration runs eagerly instead.
        self._dev_lock = threading.Lock()
        # (rec, bytes, key) of retired requests whose device memory is still
        # held: the next request with the same arguments takes the Rec over
        # (Rec.reset), the others are released when an admission needs room.
        # The retirement thread appends; only the loop takes entries out.
        self._retired = []
        self._ret_lock = threading.Lock()
        self.reused = 0           # admissions that took over a retired request's Rec

    def submit(self, req):
        if estimate_bytes(req.args) > self.budget:
            raise ValueError(f"request {req.rid} needs more than the HBM budget ({self.budget} bytes)")
        self.queue.append(req)

    # ----------------------------------------------------------- phases
    def _admit(self, slot):
        r = slot.req
        with torch.cuda.stream(slot.stream):
            if slot.reused is not None:
                rec = slot.reused[0]
                rec.reset()
            else:
                rec = Rec(r.args)
            rec.data.copy_(r.data, non_blocking=True)
            if r.obj0 is not None:
                rec.vars["obj"].copy_(r.obj0, non_blocking=True)
            rec.vars["prb"].copy_(r.prb0, non_blocking=True)
            rec.vars["pos"].copy_(r.pos0, non_blocking=True)
            rec.reserve_history(r.niter)
            rec.bh_setup()
        slot.rec = rec

    def _admit_job(self, slot, to_release):
        """Worker side of an admission: release the retired requests the loop
        handed over first; returns (bytes released, error or None)."""
        with torch.cuda.device(self.device), self._dev_lock:
            freed = self._release(to_release) if to_release else 0
            try:
                self._admit(slot)
            except (torch.OutOfMemoryError, _lib.HoloError) as err:
                return freed, err
        return freed, None

    def _launch(self, slot):
        rec = slot.rec
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(slot.stream):
            ev0.record(slot.stream)
            if slot.it == 0 or not self.graphs or not rec.graphable:   # real objects run eagerly
                rec.bh_iteration(rec.start_iter + slot.it, sync=False)
            elif rec._graph is None and not self._dev_lock.acquire(blocking=False):
                rec.bh_iteration(rec.start_iter + slot.it, sync=False)   # record on a later launch
            else:
                if rec._graph is None:
                    try:
                        rec.capture_iteration()
                    finally:
                        self._dev_lock.release()
                rec.replay_iteration()
            ev1.record(slot.stream)
        slot.inflight.append((ev0, ev1))
        slot.it += 1

    def _retire(self, slot, t0):
        r, rec = slot.req, slot.rec
        with torch.cuda.device(self.device), torch.cuda.stream(slot.stream):
            with self._dev_lock:   # the final pass may allocate
                rec.bh_finish()
            out = {k: rec.vars[k].to("cpu", non_blocking=True) for k in ("obj", "prb", "pos")}
        slot.stream.synchronize()
        out["history"] = rec.bh_history()
        r.result = out
        r.t_done = time.perf_counter() - t0
        with self._ret_lock:
            self._retired.append((rec, slot.bytes, slot.key))   # kept for reuse or freed lazily
        slot.rec = None

    def _take_retired(self, entries=None):
        """Remove entries (all when None) from the retired list; returns them."""
        with self._ret_lock:
            if entries is None:
                entries, self._retired = self._retired, []
            else:
                ids = {id(e) for e in entries}
                self._retired = [e for e in self._retired if id(e) not in ids]
        return entries

    def _release(self, retired):
        """Free these retired reconstructions' device memory (synchronises the
        device); returns the bytes released."""
        freed = sum(e[1] for e in retired)
        torch.cuda.synchronize(self.device)
        for e in retired:
            e[0].close()
        del retired
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
        # each request's argument key and memory estimate, formed once (the
        # admission test below runs on every pass of the loop)
        meta = {id(q): (args_key(q.args), estimate_bytes(q.args)) for q in pending}
        active = []
        self.used_bytes = 0
        self._retired = []
        force_release = False   # an admission ran out of memory: release before the next one
        wait_retire = False     # ... and nothing was retired then: wait for a retirement
        inline = _Inline() if not self.host_workers else None
        admit_pool = inline or ThreadPoolExecutor(1, thread_name_prefix="ht-admit")
        retire_pool = inline or ThreadPoolExecutor(1, thread_name_prefix="ht-retire")
        switch = sys.getswitchinterval()
        sys.setswitchinterval(5e-4)   # the loop gets the interpreter back quickly from the workers
        t0 = time.perf_counter()
        try:
            while pending or active:
                now = time.perf_counter() - t0
                while (pending and not wait_retire and len(active) < self.max_active
                       and (not realtime or pending[0].arrival <= now)):
                    slot = _Slot(pending[0], self._streams[-1], *meta[id(pending[0])])
                    with self._ret_lock:
                        snap = list(self._retired)
                    reuse = next((e for e in snap if e[2] == slot.key), None) if self.reuse else None
                    need = 0 if reuse is not None else slot.bytes   # a reused Rec's bytes are counted already
                    others = [e for e in snap if e is not reuse]
                    releasable = sum(e[1] for e in others)
                    release_first = releasable > 0 and (force_release or self.used_bytes + need > self.budget)
                    projected = self.used_bytes - (releasable if release_first else 0)
                    if active and projected + need > self.budget:
                        break
                    to_release = others if release_first else []
                    self._take_retired(([reuse] if reuse is not None else []) + to_release)
                    slot.reused = reuse
                    self.reused += reuse is not None
                    r = pending.pop(0)
                    self._streams.pop()
                    r.t_admit = time.perf_counter() - t0
                    # the ledger drops by what the release frees when the job reports it
                    slot.job = admit_pool.submit(self._admit_job, slot, to_release)
                    force_release = False
                    active.append(slot)
                    self.used_bytes += need
                    self.peak_bytes = max(self.peak_bytes, projected + need)
                    self.max_concurrent = max(self.max_concurrent, len(active))
                progressed = False
                for slot in list(active):
                    if slot.state == "admitting":
                        if not slot.job.done():
                            continue
                        freed, err = slot.job.result()
                        self.used_bytes -= freed
                        slot.job = None
                        progressed = True
                        if err is not None:
                            # the estimate fitted but the device did not (fragmentation,
                            # other users of the GPU): retry once the others have made room
                            active.remove(slot)
                            self._streams.append(slot.stream)
                            if slot.reused is not None:   # its Rec stays held: back to the retired list
                                with self._ret_lock:
                                    self._retired.append(slot.reused)
                            else:
                                self.used_bytes -= slot.bytes
                            pending.insert(0, slot.req)
                            if not active or "out of memory" not in str(err):
                                raise err
                            # retry after releasing the retired requests, or, with none
                            # retired, once an active request has retired
                            force_release = True
                            with self._ret_lock:
                                wait_retire = not self._retired
                            continue
                        slot.state = "running"
                    if slot.state == "retiring":
                        if slot.job.done():
                            slot.job.result()
                            wait_retire = False
                            self.done.append(slot.req)
                            active.remove(slot)
                            self._streams.append(slot.stream)
                            progressed = True
                        continue
                    while slot.inflight and slot.inflight[0][1].query():
                        ev0, ev1 = slot.inflight.popleft()
                        slot.req.latencies_ms.append(ev0.elapsed_time(ev1))
                        progressed = True
                    if slot.it >= slot.req.niter:
                        if not slot.inflight:
                            slot.state = "retiring"
                            slot.job = retire_pool.submit(self._retire, slot, t0)
                            progressed = True
                        continue
                    while slot.it < slot.req.niter and len(slot.inflight) < self.depth:
                        self._launch(slot)
                        progressed = True
                if not progressed:
                    if not active and pending and realtime:
                        time.sleep(max(0.0, min(0.01, pending[0].arrival - (time.perf_counter() - t0))))
                    else:
                        time.sleep(20e-6)
            self.wall = time.perf_counter() - t0
        finally:
            sys.setswitchinterval(switch)
            if inline is None:
                admit_pool.shutdown(wait=True)
                retire_pool.shutdown(wait=True)
        with self._dev_lock:
            self.used_bytes -= self._release(self._take_retired())
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
