#!/usr/bin/env python
"""Benchmark: Bilinear-Hessian iterations per second for a 512^3 complex
object, 900 angles, 4 propagation distances and a 512x512 detector (one BH
iteration = the data-term gradient, the Hessian forms for the step sizes,
one R and one R^T of the volume, and the variable updates).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One JSON line on stdout (rank 0).  Under torchrun (N > 1) every rank runs an
independent reconstruction (the solver does not shard across GPUs: replicas
only) and `value` is the sum over ranks; time is the max over ranks.

`value` is the served form of one reconstruction: device-side step sizes
and the iteration replayed from a CUDA graph.  `plain` is the same
reconstruction iterated the reference's way (step sizes on the host, one
round trip per iteration).  `served` runs a mixed stream of requests
(64 requests, grid n in {128, 256, 384, 512} with probabilities 0.4/0.3/0.2/0.1,
1.75 n angles, 4 distances, Poisson arrivals at 2/s, 16 iterations each)
through the continuous-batching server and, on the same requests, one at a
time through the plain path, with p50/p99 per-iteration latencies.

`--impl reference` times the reference algorithm's CPU implementation (the
NumPy port in oracle/, FP32, all host cores) on a bounded sample of the same
workload: each step runs the per-angle BH cascades (one gradient and three
Hessian cascades, as rec_mpi.py runs them) for a block of angles -- the steps
walk through distinct angles spread over [0, pi) -- and R + R^T for one slice,
scaled to 900 angles and 512 slices (`ms_per_step` is that extrapolation; the
measured seconds are reported beside it).  It also runs one whole BH
iteration of the small chain (128^3, 180 angles, 4 distances) end to end,
unscaled.

`--prop` compares the library's propagator with the padded-grid path on
torch's cuFFT (the reference's CuPy branch) at 1024^2 x 4 images (the
reference test script's size), 512^2 and 2048^2.
"""
import argparse
import gc
import json
import os
import subprocess
import sys
import tempfile
import time
import types

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BH iters/s at 512³×900 ang×4 dist (served vs plain); p50/p99 iter latency"
UNIT = "BH iterations/s"
DIST = np.array([3e-3, 4e-3, 5e-3, 6e-3])
WAVELENGTH = 7.3e-11
VOXEL = 20e-9


def bench_config(n, ntheta, ndist, world):
    """The workload description both arms print (the same dict)."""
    return {"workload": f"one BH iteration, {n}^3 object, {ntheta} angles, {ndist} distances, {n}^2 detector",
            "n": n, "ntheta": ntheta, "ndist": ndist, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (state ~60 GB)"}


def workload_args(n, ntheta, ndist, niter=10 ** 6):
    import types
    return types.SimpleNamespace(
        theta=np.linspace(0, np.pi, ntheta, endpoint=False).astype("float32"), ndist=ndist, ntheta=ntheta,
        nz=n, n=n, nzobj=n, nobj=n, obj_dtype="complex64", mask=0.9, lam_prbfit=0.0, rho=[1, 0.05, 0.02],
        niter=niter, nchunk=n, vis_step=-1, err_step=-1, start_iter=0, distance=DIST[:ndist],
        wavelength=WAVELENGTH, voxelsize=VOXEL, norm_magnifications=np.ones(ndist))


# ----------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------- CPU (oracle)
def _oracle(threads):
    os.environ["HOLO_ORACLE_WORKERS"] = str(threads)
    from oracle import holo_oracle as O
    O._WORKERS = threads
    return O


def cpu_sample(n, ntheta, ndist, threads, angles=None):
    """Seconds per BH iteration of the reference algorithm on the host: the
    per-angle cascades (1 gradient + 3 Hessian, as rec_mpi.py runs them) of the
    given angles (indices into the ntheta angles; default the first) and R, R^T
    of one slice, scaled linearly to ntheta angles and n slices.  Returns
    (seconds per iteration, measured seconds, description)."""
    O = _oracle(threads)
    rng = np.random.default_rng(0)
    th_all = workload_args(n, ntheta, ndist).theta
    idx = np.asarray([0] if angles is None else angles)
    na = len(idx)
    a = workload_args(n, na, ndist)
    a.theta = th_all[idx]
    rec = O.Rec(a, "complex64")
    rec.eff_demagnifications[:] = 1
    rec.data[:] = 1.0
    v = {"prb": np.ones((ndist, n, n), "complex64"),
         "proj": (0.01 * rng.standard_normal((na, n, n))).astype("complex64"),
         "pos": rng.uniform(-2, 2, (na, ndist, 2)).astype("float32")}
    g = {"prb": (0.01 * rng.standard_normal((ndist, n, n))).astype("complex64"),
         "proj": (0.01 * rng.standard_normal((na, n, n))).astype("complex64"),
         "pos": rng.uniform(-1, 1, (na, ndist, 2)).astype("float32")}
    e = {k: x.copy() for k, x in g.items()}
    tomo = O.Tomo(n, 1, th_all, 0, "complex64")
    x = (0.01 * rng.standard_normal((1, n, n))).astype("complex64")
    t0 = time.perf_counter()
    rec.gradients_cascade(v, g)
    rec.hessian_cascade(v, g, e)
    rec.hessian_cascade(v, e, e)
    rec.hessian_cascade(v, e, e)
    t1 = time.perf_counter()
    y = tomo.R(x)
    tomo.RT(y)
    t2 = time.perf_counter()
    per_iter = (t1 - t0) * ntheta / na + (t2 - t1) * n
    sample = (f"reference-structure BH cascades (1 gradient + 3 Hessian) for {na} of {ntheta} angles at "
              f"{n}x{n}x{ndist}, plus R and R^T of 1 of {n} slices, scaled linearly; FP32 NumPy/SciPy oracle")
    return per_iter, t2 - t0, sample


def cpu_small_chain_iteration(threads, n=128, ntheta=180, ndist=4):
    """Two whole BH iterations of the small chain (n^3, ntheta angles, ndist
    distances) on the host, unscaled: gradient with R^T, R of the gradient,
    the Hessian forms for the step sizes, the updates (the FP32 oracle's BH,
    rec_mpi.py:163-227).  Returns measured seconds."""
    O = _oracle(threads)
    from holotomocupy_b200.synthetic import ellipsoid_phantom
    args = workload_args(n, ntheta, ndist, niter=2)
    rec = O.Rec(args, "complex64")
    rng = np.random.default_rng(1)
    rec.eff_demagnifications[:] = 1
    rec.vars["obj"][:] = ellipsoid_phantom(n, 20, 11, device="cpu").numpy()
    rec.vars["prb"][:] = 1
    rec.vars["pos"][:] = rng.uniform(-2, 2, (ntheta, ndist, 2))
    rec.gen_sqrt_data(rec.vars, rec.data)
    rec.eff_demagnifications[:] = 0
    rec.vars["obj"][:] = 0
    t0 = time.perf_counter()
    rec.BH(niter=2)          # the first iteration (no beta) and one steady-state iteration
    t1 = time.perf_counter()
    return {"two_iterations_s": t1 - t0}


def run_reference(a, rank, budget_s=100.0):
    """The reference arm: rank 0 alone (other ranks exit without work)."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    n, ntheta, ndist = a.size, a.ntheta, 4
    # one angle first, to size the per-step angle block within the time budget
    t_cal = cpu_sample(n, ntheta, ndist, threads)[1]
    steps = a.warmup + a.steps
    per_angle = max(t_cal, 1e-3)
    na = int(max(1, min(90, budget_s / steps / per_angle)))
    # the steps walk through distinct angles spread over the 900
    order = np.random.default_rng(0).permutation(ntheta)
    blocks = [np.sort(order[(k * na) % ntheta: (k * na) % ntheta + na]) for k in range(steps)]
    per, measured = [], []
    for k in range(steps):
        p, w, sample = cpu_sample(n, ntheta, ndist, threads, blocks[k])
        if k >= a.warmup:
            per.append(p)
            measured.append(w)
    c1 = None if a.no_small_chain else cpu_small_chain_iteration(threads)
    ms = float(np.mean(per)) * 1e3
    value = 1e3 / ms
    distinct = len(np.unique(np.concatenate(blocks[a.warmup:])))
    sample = (f"per step: the BH cascades (1 gradient + 3 Hessian, rec_mpi.py's structure) of {na} of {ntheta} "
              f"angles and R + R^T of 1 of {n} slices at {n}^2 x {ndist} distances, scaled linearly to the whole "
              f"iteration; the {a.steps} timed steps cover {distinct} distinct angles; FP32 NumPy/SciPy oracle")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms, "ms_per_step_is": "extrapolated from the sampled angles and slice",
            "measured_s_per_step": float(np.mean(measured)), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64", "data": "synthetic", "impl": "reference",
            "config": bench_config(n, ntheta, ndist, a.gpus),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                             "angles_per_step": na, "distinct_angles_timed": distinct},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "small_chain_measured": None if c1 is None else {
                "workload": "two whole BH iterations at 128^3, 180 angles, 4 distances, unscaled (the first and "
                            "one steady-state iteration)", **c1, "iters_per_s": 2.0 / c1["two_iterations_s"]}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU
def max_over_ranks(values, device):
    """Element-wise max over the ranks of the process group (the times of
    independent replicas); identity without one."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def replica_value(ms_max, world):
    """Whole-job BH iterations/s of `world` replicas whose slowest rank took
    ms_max per iteration."""
    return world * 1e3 / ms_max


def build_problem(n, ntheta, ndist, seed, device):
    import torch
    from holotomocupy_b200 import synthetic
    from holotomocupy_b200.rec import Rec
    rec = Rec(workload_args(n, ntheta, ndist))
    nell = 80 if n >= 512 else 20
    obj = synthetic.ellipsoid_phantom(n, nell, seed, WAVELENGTH, VOXEL, device=device)
    prb = synthetic.random_probe(ndist, n, n, seed + 1, device=device)
    pos = synthetic.random_positions(ntheta, ndist, 2.0, seed + 2, device=device)
    data = rec.forward_amplitudes(obj, prb, pos)
    synthetic.noisy_amplitudes(data, 1e4, seed + 3)
    torch.cuda.synchronize()
    return rec, obj, prb, pos, data


def run_rows(a):
    """The rows beside the BH hot path, each timed on the device with CUDA
    events around `steps` calls after `warmup` (a checkpoint, host work, with
    the host clock), and -- where the oracle restates the reference's
    algorithm -- the oracle beside it on a bounded sample of the same workload
    on all host cores, scaled linearly as the main CPU baseline is:
      * a BH iteration at 512^3 x 900 x 4, graph-replayed, plain, with the
        probe-fit regulariser (lam_prbfit = 2e-3; rec_mpi.py:365-398) and with
        the Laplacian regulariser (lam_laplacian = 1e-3; rec_mpi.py:400-496);
      * Tomo.fbp and Tomo.rec_tomo (4 CG iterations) of a 900 x 512 x 512
        sinogram (tomo.py:163-210); oracle: one slice;
      * Shift.Sback of 3600 images of 512^2 (shift.py:138-148); oracle: 16 images;
      * RecNFP (rec_nfp_mpi.py:100-144), a 512^2 probe, a 768^2 projection and
        256 scan positions: BH iterations, host step sizes (as the reference) and
        graph-replayed with device step sizes;
      * a checkpoint of the 512^3 x 900 x 4 state written and read back
        (writer.py:57-110, reader.py:260-340; the .npz layout, h5py being
        absent on the box)."""
    import tempfile
    import types
    import torch
    from holotomocupy_b200 import RecNFP, Shift, Tomo
    from holotomocupy_b200.checkpoint import Writer, read_checkpoint
    from holotomocupy_b200.rec import Rec
    dev = torch.device("cuda", 0)
    threads = os.cpu_count() or 1
    n, ntheta, ndist = 512, 900, 4
    g = torch.Generator(device=dev).manual_seed(8)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    rng = np.random.default_rng(8)

    def timed(fn, steps=None, warmup=None):
        for _ in range(a.warmup if warmup is None else warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k = a.steps if steps is None else steps
        e0.record()
        for _ in range(k):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    out = {}
    # ---- BH iterations, plain and with each regulariser
    base, obj, prb, pos, data = build_problem(n, ntheta, ndist, 4321, dev)
    del obj
    prb0 = torch.ones_like(prb)

    def bh_ms(rec):
        st = torch.cuda.Stream(device=dev)
        with torch.cuda.stream(st):
            reset_state(rec, prb0, pos, data)
            rec.bh_setup()
            rec.bh_iteration(0, sync=False)
            rec.capture_iteration()
            ms = timed(rec.replay_iteration)
            rec.release_graph()
        return ms

    out["bh_plain_ms"] = bh_ms(base)
    base.close()
    del base
    torch.cuda.empty_cache()
    for key, lam in (("lam_prbfit", 2e-3), ("lam_laplacian", 1e-3)):
        args = workload_args(n, ntheta, ndist)
        setattr(args, key, lam)
        rec = Rec(args)
        rec.ref.copy_(prb.abs())   # the probe-fit's reference amplitude
        out[f"bh_{key}_ms"] = bh_ms(rec)
        rec.close()
        del rec
        torch.cuda.empty_cache()
    for key in ("lam_prbfit", "lam_laplacian"):
        out[f"bh_{key}_extra_pct"] = 100.0 * (out[f"bh_{key}_ms"] / out["bh_plain_ms"] - 1.0)
    del data, prb, pos, prb0
    torch.cuda.empty_cache()

    O = _oracle(threads)
    # ---- filtered back-projection and the CG initial guess
    theta = workload_args(n, ntheta, ndist).theta
    tomo = Tomo(n, n, theta, 0.9)
    d = torch.randn(ntheta, n, n, dtype=torch.complex64, device=dev, generator=g)
    out["fbp_ms"] = timed(lambda: tomo.fbp(d))
    # algorithmic bytes: the sinogram read once, the volume written once
    out["fbp_gbs"] = (ntheta + n) * n * n * 8 / (out["fbp_ms"] * 1e-3) / 1e9
    out["fbp_frac"] = out["fbp_gbs"] / peak
    out["rec_tomo_4it_ms"] = timed(lambda: tomo.rec_tomo(d, 4), steps=2, warmup=1)
    ot = O.Tomo(n, 1, theta, 0.9, "complex64")
    ds = (rng.standard_normal((ntheta, 1, n)) + 1j * rng.standard_normal((ntheta, 1, n))).astype("complex64")
    t0 = time.perf_counter()
    ot.fbp(ds)
    t1 = time.perf_counter()
    ot.rec_tomo(ds, 4)
    t2 = time.perf_counter()
    out["fbp_cpu_ms"] = (t1 - t0) * 1e3 * n
    out["rec_tomo_4it_cpu_ms"] = (t2 - t1) * 1e3 * n
    del tomo, d
    torch.cuda.empty_cache()
    # ---- back-projection shift
    nimg = ntheta * ndist
    sh = Shift(n, n, n, n, "complex64")
    sp = torch.randn(nimg, n, n, dtype=torch.complex64, device=dev, generator=g)
    rs = 4 * torch.rand(nimg, 2, device=dev, generator=g) - 2
    out["sback_ms"] = timed(lambda: sh.Sback(sp, rs, 1.0))
    # algorithmic bytes: the detector images read once, the coefficient grids written once
    out["sback_gbs"] = nimg * 2 * n * n * 8 / (out["sback_ms"] * 1e-3) / 1e9
    out["sback_frac"] = out["sback_gbs"] / peak
    osh = O.Shift(n, n, n, n, "complex64", dtype="complex64")
    t0 = time.perf_counter()
    osh.Sback(sp[:16].cpu().numpy(), rs[:16].cpu().numpy(), np.float32(1.0))
    out["sback_cpu_ms"] = (time.perf_counter() - t0) * 1e3 * nimg / 16
    del sh, sp, rs
    torch.cuda.empty_cache()
    # ---- near-field ptychography
    nargs = types.SimpleNamespace(distance=np.array([4e-3]), wavelength=WAVELENGTH, voxelsize=VOXEL, ntheta=256,
                                  nz=512, n=512, nzobj=768, nobj=768, obj_dtype="complex64", rho=[1, 0.5, 0.1],
                                  niter=10 ** 6, nchunk=256, vis_step=-1, err_step=-1, start_iter=0)
    rn = RecNFP(nargs)
    pos_t = 8 * torch.rand(256, 2, device=dev, generator=g) - 4
    rn.vars["prb"].copy_(1 + 0.2 * torch.randn(512, 512, dtype=torch.complex64, device=dev, generator=g))
    rn.vars["proj"].copy_(0.05 * torch.randn(768, 768, dtype=torch.complex64, device=dev, generator=g))
    rn.vars["pos"].copy_(pos_t)
    rn.gen_sqrt_data(rn.vars, rn.data)
    for dd in (rn.vars, rn.grads, rn.etas):
        for v in dd.values():
            v.zero_()
    rn.vars["prb"].fill_(1)
    rn.vars["pos"].copy_(pos_t + 0.3 * (2 * torch.rand(256, 2, device=dev, generator=g) - 1))
    for mode in ("host", "graph"):
        rn.BH(niter=2, mode=mode)   # warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rn.BH(niter=8, mode=mode)   # a solve of 8 iterations from the warm-up's state
        e1.record()
        torch.cuda.synchronize()
        out["nfp_bh_iteration_ms" if mode == "host" else "nfp_bh_iteration_graph_ms"] = e0.elapsed_time(e1) / 8
    rn.close()
    del rn
    torch.cuda.empty_cache()
    # ---- checkpoint of the 512^3 state
    st = {"obj": torch.randn(n, n, n, dtype=torch.complex64, device=dev, generator=g),
          "prb": torch.randn(ndist, n, n, dtype=torch.complex64, device=dev, generator=g),
          "pos": torch.rand(ntheta, ndist, 2, device=dev, generator=g)}
    nbytes = sum(v.numel() * v.element_size() for v in st.values())
    with tempfile.TemporaryDirectory() as tmp:
        w = Writer(tmp, fmt="npz")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        path = w.write_checkpoint(st, 1, 1.0)
        t1 = time.perf_counter()
        back = read_checkpoint(path, n, n, device=dev)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        out["checkpoint_write_s"], out["checkpoint_read_s"] = t1 - t0, t2 - t1
        out["checkpoint_write_gbs"], out["checkpoint_read_gbs"] = nbytes / (t1 - t0) / 1e9, nbytes / (t2 - t1) / 1e9
        out["checkpoint_obj_max_abs_diff"] = float((back["obj"] - st["obj"]).abs().max())
    line = {"metric": "rows beside the BH hot path: device time per call (ms), oracle on the host cores beside it",
            "unit": "ms", "value": out["bh_plain_ms"], "higher_is_better": False, "steps": a.steps,
            "warmup": a.warmup, "n_gpus": 1, "dtype": "c64", "data": "synthetic (seeded)", "cpu_cores": threads,
            "peak_gbs": peak, "peak_source": "measured" if peaks else "fallback",
            "config": {"workload": "512^3 object, 900 angles, 4 distances; RecNFP 512^2 probe, 768^2 projection, "
                                   "256 positions"},
            "rows": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in out.items()}}
    print(json.dumps(line), flush=True)


def reset_state(rec, prb0, pos0, data=None):
    import torch
    for d in (rec.vars, rec.grads, rec.etas):
        for v in d.values():
            v.zero_()
    for v in rec._c.values():
        v.zero_()
    rec.vars["prb"].copy_(prb0)
    rec.vars["pos"].copy_(pos0)
    if data is not None:
        rec.data.copy_(data)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=512, help="object/detector size n (the workload is n=512)")
    ap.add_argument("--ntheta", type=int, default=900)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--e2e-iters", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=64, help="requests in the mixed served stream (0: skip)")
    ap.add_argument("--serve-iters", type=int, default=16)
    ap.add_argument("--c5", action="store_true",
                    help="the 2048^3 x 1800 x 4 operator measurement (D, R, R^T on a 256-slice sub-volume) "
                         "instead of the BH line")
    ap.add_argument("--large", action="store_true",
                    help="8 BH iterations at 1024^3 x 900 angles x 4 distances with angle-chunked cascade and "
                         "slab-chunked Radon transform (the largest reconstruction whose state fits one B200) "
                         "instead of the BH line")
    ap.add_argument("--prop", action="store_true",
                    help="the propagator against the padded-grid path on torch's cuFFT (1024^2 x 4, 512^2, 2048^2) "
                         "instead of the BH line")
    ap.add_argument("--rows", action="store_true",
                    help="the rows beside the BH path (regularisers, fbp / rec_tomo, Sback, RecNFP, checkpoints) "
                         "instead of the BH line")
    ap.add_argument("--no-small-chain", action="store_true",
                    help="reference arm: skip the unscaled small-chain BH iterations")
    ap.add_argument("--profile", action="store_true",
                    help="time the device iterations only (no roofline, e2e or CPU legs): for ncu launch lists")
    a = ap.parse_args()
    if a.warmup < 3:
        a.warmup = 3

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if a.impl == "reference":
        run_reference(a, rank)
        return
    if a.c5:
        run_c5(a)
        return
    if a.prop:
        run_prop(a)
        return
    if a.large:
        run_large(a)
        return
    if a.rows:
        run_rows(a)
        return

    import torch
    import torch.distributed as dist
    from holotomocupy_b200 import _lib
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(minutes=10), device_id=device)

    n, ntheta, ndist = a.size, a.ntheta, 4
    rec, obj_true, prb_true, pos_true, data = build_problem(n, ntheta, ndist, 1234 + rank, device)
    prb0 = torch.ones_like(prb_true)
    gen = torch.Generator(device=device).manual_seed(99 + rank)
    pos0 = pos_true + 0.5 * (2 * torch.rand(pos_true.shape, generator=gen, device=device) - 1)

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- the plain path: host step sizes, one round trip per iteration
    reset_state(rec, prb0, pos0)
    rec.bh_setup()
    it = 0
    for _ in range(a.warmup):
        rec.bh_iteration(it)
        it += 1
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    lat_plain = []
    for k in KERNEL_BYTES:
        _lib.call("ht_ktimer_arm", k.encode(), 1)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(st)
    for _ in range(a.steps):
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(st)
        rec.bh_iteration(it)
        s1.record(st)
        lat_plain.append((s0, s1))
        it += 1
    p1.record(st)
    torch.cuda.synchronize()
    ktimes = kernel_times(rec)
    ms_plain = p0.elapsed_time(p1) / a.steps
    lat_plain = sorted(s.elapsed_time(e) for s, e in lat_plain)
    rec.bh_finish()

    # ---- the served form: device step sizes, graph-replayed iterations
    sst = torch.cuda.Stream(device=device)
    with torch.cuda.stream(sst):
        reset_state(rec, prb0, pos0)
        rec.bh_setup()
        rec.bh_iteration(0, sync=False)
        l0 = _lib.lib().ht_launch_count()
        rec.capture_iteration()
        launches = _lib.lib().ht_launch_count() - l0     # kernels recorded in one replayed iteration
        for _ in range(a.warmup - 1):
            rec.replay_iteration()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lat = []
    with torch.cuda.stream(sst):
        torch.cuda.nvtx.range_push("bh_timed")   # the timed iterations, for profilers' range filters
        e0.record(sst)
        for _ in range(a.steps):
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record(sst)
            rec.replay_iteration()
            s1.record(sst)
            lat.append((s0, s1))
        e1.record(sst)
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / a.steps
    per_lat = sorted(s.elapsed_time(e) for s, e in lat)
    ms, ms_plain = max_over_ranks([ms, ms_plain], device)
    with torch.cuda.stream(sst):
        rec.release_graph()
    rec.bh_finish()
    value = replica_value(ms, world)

    # ---- roofline of the dominant kernel family (the propagator passes)
    roof = None if a.profile else roofline(ktimes)

    # ---- end to end through the public API with pinned host buffers
    e2e = None if a.profile else end_to_end(a, rec, obj_true, prb0, pos0, data, device, barrier, world)

    # ---- mixed served stream vs the same requests one at a time (one GPU: the
    # stream's pinned requests and results take ~60 GB of host memory a process)
    served = None
    if a.serve_requests > 0 and not a.profile and world == 1:
        del rec, data, obj_true, prb_true, pos_true
        gc.collect()   # the reconstruction's device handles go with it (cudaMalloc'd outside torch's cache)
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        served = served_vs_plain(a.serve_requests, a.serve_iters, 4321 + rank)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT,
        "served_over_plain": {
            "single_512_job": ms_plain / ms,
            "poisson_stream": served["poisson_2_per_s"]["served_over_plain"] if served else None,
            "saturated_stream": served["saturated"]["served_over_plain"] if served else None},
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64",
        "data": "synthetic (seeded ellipsoid phantom, random probe and positions, Poisson noise at 1e4 photons)",
        "config": bench_config(n, ntheta, ndist, world),
        "form": "served: device step sizes, iteration replayed from a CUDA graph",
        "latency_ms_p50": float(np.percentile(per_lat, 50)), "latency_ms_p99": float(np.percentile(per_lat, 99)),
        "plain": {"value": replica_value(ms_plain, world), "unit": UNIT, "ms_per_step": ms_plain,
                  "latency_ms_p50": float(np.percentile(lat_plain, 50)),
                  "latency_ms_p99": float(np.percentile(lat_plain, 99)),
                  "form": "host step sizes (H and dots copied to the host each iteration), eager launches"},
        "served": served,
        "gpu_launches": launches * a.steps,      # the library's kernels in the timed region (all steps)
        "gpu_launches_per_step": launches,
        "roofline": roof,
        "e2e": e2e,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not (a.no_cpu_baseline or a.profile):
        per_iter, wall, sample = cpu_sample(n, ntheta, ndist, os.cpu_count() or 1)
        line["cpu_baseline"] = {"value": 1.0 / per_iter, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": sample, "sample_seconds": wall}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_c5(a, n=2048, ntheta=1800, ndist=4, nz_sub=256, nimg_chunk=256):
    """Operators at the 2048^3, 1800-angle, 4-distance size: the propagator D
    over image chunks and R, R^T of a 256-slice sub-volume (the full state,
    ~430 GB, exceeds one GPU; the BH iteration at this size is not run).
    Achieved = algorithmic bytes / CUDA-event time against the measured HBM
    copy bandwidth."""
    import torch
    from holotomocupy_b200 import Propagation, Tomo, _lib
    dev = torch.device("cuda", 0)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    g = torch.Generator(device=dev).manual_seed(5)

    def timed(fn, reps):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps * 1e-3

    out = {}
    prop = Propagation(n, n, nimg_chunk, ndist, WAVELENGTH, VOXEL, DIST[:ndist])
    x = torch.randn(nimg_chunk, n, n, dtype=torch.complex64, device=dev, generator=g)
    y = torch.empty_like(x)
    st = _lib.stream_ptr()
    t = timed(lambda: _lib.call("ht_prop_D", prop._h, _lib.ptr(x), _lib.ptr(y), nimg_chunk, 0, st), a.steps)
    alg = 16.0 * nimg_chunk * n * n + 32.0 * n * n
    out["D"] = {"images_per_launch": nimg_chunk, "launch_ms": t * 1e3, "achieved_gbs": alg / t / 1e9,
                "frac": alg / t / 1e9 / peak, "all_images_s": t * ntheta * ndist / nimg_chunk}
    del x, y, prop
    torch.cuda.empty_cache()
    theta = np.linspace(0, np.pi, ntheta, endpoint=False).astype("float32")
    tomo = Tomo(n, nz_sub, theta, 0.9)
    obj = torch.randn(nz_sub, n, n, dtype=torch.complex64, device=dev, generator=g)
    sino = torch.empty(ntheta, nz_sub, n, dtype=torch.complex64, device=dev)
    back = torch.empty_like(obj)
    t = timed(lambda: tomo.R(obj, out=sino), max(1, a.steps // 2))
    alg = 8.0 * nz_sub * n * n + 8.0 * ntheta * nz_sub * n
    out["R"] = {"slices": nz_sub, "launch_ms": t * 1e3, "achieved_gbs": alg / t / 1e9, "frac": alg / t / 1e9 / peak,
                "full_volume_s": t * n / nz_sub}
    t = timed(lambda: tomo.RT(sino, out=back), max(1, a.steps // 2))
    out["RT"] = {"slices": nz_sub, "launch_ms": t * 1e3, "achieved_gbs": alg / t / 1e9, "frac": alg / t / 1e9 / peak,
                 "full_volume_s": t * n / nz_sub}
    del obj, sino, back, tomo
    torch.cuda.empty_cache()
    out["D_host"] = host_streamed_D(a, n, ndist)
    line = {"metric": "operator HBM GB/s at 2048^3 x 1800 angles x 4 distances", "value": out["D"]["achieved_gbs"],
            "unit": "GB/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "higher_is_better": True,
            "dtype": "c64", "data": "synthetic (seeded normal complex64)", "peak_gbs": peak,
            "peak_source": "measured" if peaks else "fallback",
            "config": {"workload": "D over 256-image chunks of 2048^2; R, R^T of a 256-slice 2048^2 sub-volume at "
                                   "1800 angles", "n": n, "ntheta": ntheta, "ndist": ndist},
            "operators": out}
    print(json.dumps(line), flush=True)


def run_large(a, n=1024, ntheta=900, ndist=4, chunk=128, slab=128, niter=8):
    """BH at 1024^3 x 900 angles x 4 distances on one GPU: the state (object,
    projections and their B-spline coefficients for vars/grads/etas, data;
    ~100 GB) stays in HBM, the fused cascade runs in angle chunks of 128
    (each chunk's forward pass recomputed before its Hessian pass) and the
    Radon transform in slabs of 128 slices, so the workspaces stay ~25 GB.
    Timed: niter graph-replayed iterations after two eager ones.  Achieved =
    the algorithmic bytes of the timed kernels (KERNEL_BYTES) in the second,
    steady-state eager iteration / the replayed iteration time, against the
    measured HBM copy bandwidth."""
    import torch
    from holotomocupy_b200 import _lib, synthetic
    from holotomocupy_b200.rec import Rec
    dev = torch.device("cuda", 0)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    args = workload_args(n, ntheta, ndist)
    args.angle_chunk, args.slab_chunk = chunk, slab
    t0 = time.perf_counter()
    rec = Rec(args)
    obj = synthetic.ellipsoid_phantom(n, 80, 4321, WAVELENGTH, VOXEL, device=dev)
    prb = synthetic.random_probe(ndist, n, n, 4322, device=dev)
    pos = synthetic.random_positions(ntheta, ndist, 2.0, 4323, device=dev)
    rec.forward_amplitudes(obj, prb, pos, out=rec.data)
    synthetic.noisy_amplitudes(rec.data, 1e4, 4324)
    del obj
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0
    rec.vars["prb"].fill_(1)
    gen = torch.Generator(device=dev).manual_seed(4325)
    rec.vars["pos"].copy_(pos + 0.5 * (2 * torch.rand(pos.shape, generator=gen, device=dev) - 1))
    rec.bh_setup()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    st = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(st):
        rec.bh_iteration(0, sync=False)
    torch.cuda.synchronize()
    for k in KERNEL_BYTES:
        _lib.call("ht_ktimer_arm", k.encode(), 1)
    with torch.cuda.stream(st):
        e[0].record(st)
        rec.bh_iteration(1, sync=False)     # a steady-state iteration, eager, with the kernel timers
        e[1].record(st)
    torch.cuda.synchronize()
    kt = kernel_times(rec)
    alg = sum(v["alg_bytes"] * v["launches"] for v in kt.values())
    with torch.cuda.stream(st):
        rec.capture_iteration()
        e[2].record(st)
        for _ in range(niter):
            rec.replay_iteration()
        e[3].record(st)
    torch.cuda.synchronize()
    ms = e[2].elapsed_time(e[3]) / niter
    with torch.cuda.stream(st):
        rec.release_graph()
    hist = rec.bh_history()
    line = {"metric": "BH iterations/s at 1024^3 x 900 angles x 4 distances (angle- and slab-chunked, state in HBM)",
            "value": 1e3 / ms, "unit": "BH iterations/s", "ms_per_iteration": ms, "iterations": niter,
            "eager_iteration_ms": e[0].elapsed_time(e[1]), "n_gpus": 1, "dtype": "c64",
            "data": "synthetic (seeded ellipsoid phantom, random probe and positions, Poisson noise at 1e4 photons)",
            "config": {"workload": f"BH, {n}^3 object, {ntheta} angles, {ndist} distances, {n}^2 detector",
                       "angle_chunk": chunk, "slab_chunk": slab},
            "timed_kernel_alg_bytes_per_iteration": alg,
            "achieved_gbs_timed_kernels": alg / (ms * 1e-3) / 1e9,
            "frac_timed_kernels": alg / (ms * 1e-3) / 1e9 / peak, "peak_gbs": peak,
            "peak_source": "measured" if peaks else "fallback",
            "device_bytes_in_use": int(torch.cuda.mem_get_info(dev)[1] - torch.cuda.mem_get_info(dev)[0]),
            "setup_s": t_setup,
            "step_sizes_finite": bool(all(np.isfinite(a) and np.isfinite(b) for a, b in hist))}
    print(json.dumps(line), flush=True)


def run_prop(a):
    """The library's propagator (DCT form, ht_prop_D / ht_prop_DT) against the
    padded-grid path on torch's cuFFT -- the reference's CuPy branch
    (propagation.py:77-86, 98-110), the stand-in for its cuFFTDx path -- and the
    library's own padded-grid convolution (ht_conv2d_run, the surface of the
    cuFFTDx conv2d_run).  CUDA events around `steps` back-to-back calls after
    `warmup` calls; algorithmic bytes of D: 16 B n nz + 32 B n nz (table)."""
    import torch
    from holotomocupy_b200 import Propagation
    dev = torch.device("cuda", 0)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    g = torch.Generator(device=dev).manual_seed(6)

    def timed(fn):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / a.steps

    rows = []
    for n, batch in ((1024, 4), (512, 64), (1024, 32), (2048, 16)):
        cl = Propagation(n, n, batch, 4, WAVELENGTH, VOXEL, DIST)
        ref = Propagation(n, n, batch, 4, WAVELENGTH, VOXEL, DIST)
        ref._use_cufftdx = False
        x = torch.randn(batch, n, n, dtype=torch.complex64, device=dev, generator=g)
        err = float(torch.abs(cl.D(x, 0) - ref.D(x, 0)).max() / torch.abs(ref.D(x, 0)).max())
        pad = torch.empty(batch, 2 * n, 2 * n, dtype=torch.complex64, device=dev)
        cl._fwd_pad(x, pad)
        ybuf = torch.empty_like(pad)
        r = {"n": n, "images": batch,
             "D_ms": timed(lambda: cl.D(x, 0)), "DT_ms": timed(lambda: cl.DT(x, 0)),
             "cufft_D_ms": timed(lambda: ref.D(x, 0)), "cufft_DT_ms": timed(lambda: ref.DT(x, 0)),
             "conv2d_run_ms": timed(lambda: cl._conv2d.run(pad, cl.fker[0], ybuf)),
             "max_rel_diff_D": err}
        alg = 16.0 * batch * n * n + 32.0 * n * n
        r["D_achieved_gbs"] = alg / (r["D_ms"] * 1e-3) / 1e9
        r["D_frac"] = r["D_achieved_gbs"] / peak
        r["speedup_D"] = r["cufft_D_ms"] / r["D_ms"]
        r["speedup_DT"] = r["cufft_DT_ms"] / r["DT_ms"]
        rows.append(r)
        del cl, ref, x, pad, ybuf
        torch.cuda.empty_cache()
    line = {"metric": "Fresnel propagator D / D^T time: library vs padded-grid torch cuFFT", "unit": "ms",
            "value": rows[0]["D_ms"], "higher_is_better": False, "steps": a.steps, "warmup": a.warmup,
            "n_gpus": 1, "dtype": "c64", "data": "synthetic (seeded normal complex64)", "peak_gbs": peak,
            "peak_source": "measured" if peaks else "fallback",
            "config": {"workload": "D and D^T at distance 3 mm, 7.3e-11 m, 20 nm pixels"}, "rows": rows}
    print(json.dumps(line), flush=True)


def host_streamed_D(a, n, ndist, nimg=512, chunk=64):
    """D over a host-resident stack of nimg 2048^2 images through
    Chunking.gpu_batch (chunks of `chunk` images: host-to-device copy, D and
    device-to-host copy of consecutive chunks overlapped on three streams).
    The host arrays are page-locked once, before the timed calls.  Timed by
    the host clock around whole calls (each ends with its streams
    synchronised); PCIe-bound, so the figure of merit is host bytes moved per
    second."""
    import torch
    from holotomocupy_b200 import Propagation
    from holotomocupy_b200.chunking import Chunking, _HostPin
    prop = Propagation(n, n, chunk, ndist, WAVELENGTH, VOXEL, DIST[:ndist])
    x = np.empty((nimg, n, n), np.complex64)
    x.fill(1.0 + 0.5j)
    y = np.empty_like(x)
    pin = _HostPin([x, y])
    ch = Chunking(4 * chunk * n * n * 8 + (1 << 20), chunk)

    @ch.gpu_batch(axis_out=0, axis_inp=0, nout=1)
    def _d(cl, o, xc):
        o.copy_(prop.D(xc, 0))

    for _ in range(max(1, a.warmup - 2)):
        _d(ch, y, x)
    reps = max(1, a.steps // 2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        _d(ch, y, x)
    torch.cuda.synchronize()
    t = (time.perf_counter() - t0) / reps
    pin.close()
    host_bytes = 2.0 * x.nbytes
    return {"images": nimg, "chunk": chunk, "seconds": t, "host_gbs": host_bytes / t / 1e9,
            "h2d_bytes": x.nbytes, "d2h_bytes": y.nbytes,
            "timing": "host clock around whole calls (streams synchronised at the end of each)"}


def served_vs_plain(nreq, niter, seed):
    """The mixed request stream through the server and one at a time, twice:
    with the Poisson arrivals (2/s) and saturated (every request present at
    t = 0).  Reported per variant: aggregate BH iterations/s, p50/p99
    per-iteration latency and p50/p99 per-request completion latency (arrival
    to result on the host)."""
    import torch
    from holotomocupy_b200.serving import Request, Server, run_plain
    from holotomocupy_b200.synthetic import make_problem
    rng = np.random.default_rng(seed)
    sizes = rng.choice([128, 256, 384, 512], size=nreq, p=[0.4, 0.3, 0.2, 0.1])
    arrivals = np.cumsum(rng.exponential(0.5, nreq))
    arrivals -= arrivals[0]
    reqs = []
    for rid, (n, t) in enumerate(zip(sizes, arrivals)):
        args, data, prb0, pos0, _ = make_problem(int(n), int(round(1.75 * n)), 4, seed + 10 * rid, host=True)
        reqs.append(Request(rid=rid, args=args, data=data, prb0=prb0, pos0=pos0, niter=niter, arrival=float(t)))
        gc.collect()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    total = nreq * niter
    out = {"workload": f"{nreq} requests, n from {{128,256,384,512}} (p 0.4/0.3/0.2/0.1), 1.75 n angles, "
                       f"4 distances, {niter} BH iterations each", "sizes": [int(x) for x in sizes],
           "iterations": total}
    for variant, realtime in (("poisson_2_per_s", True), ("saturated", False)):
        done_plain = []
        wall_p, lat_p, _ = run_plain(reqs, realtime=realtime, done_times=done_plain)
        order = sorted(reqs, key=lambda q: q.arrival)
        comp_p = np.array([d - (q.arrival if realtime else 0.0) for d, q in zip(done_plain, order)])
        torch.cuda.empty_cache()
        for r in reqs:
            r.latencies_ms, r.result, r.t_admit, r.t_done = [], None, None, None
        srv = Server(max_active=4)
        for r in reqs:
            srv.submit(r)
        srv.run(realtime=realtime)
        st = Server.latency_stats(reqs)
        cs = Server.completion_stats(reqs, realtime)
        out[variant] = {
            "served_iters_per_s": total / srv.wall, "plain_iters_per_s": total / wall_p,
            "served_over_plain": wall_p / srv.wall, "served_wall_s": srv.wall, "plain_wall_s": wall_p,
            "served_p50_ms": st["p50_ms"], "served_p99_ms": st["p99_ms"],
            "plain_p50_ms": float(np.percentile(lat_p, 50)), "plain_p99_ms": float(np.percentile(lat_p, 99)),
            "served_completion_p50_s": cs["p50_s"], "served_completion_p99_s": cs["p99_s"],
            "plain_completion_p50_s": float(np.percentile(comp_p, 50)),
            "plain_completion_p99_s": float(np.percentile(comp_p, 99)),
            "max_concurrent": srv.max_concurrent, "peak_bytes_admitted": srv.peak_bytes}
        for r in reqs:
            r.latencies_ms, r.result, r.t_admit, r.t_done = [], None, None, None
        gc.collect()
        torch.cuda.empty_cache()
    return out


# Algorithmic HBM bytes per work unit of each timed kernel (inputs read once,
# outputs written once, at their stored types; a unit is one detector image
# for the cascade and column kernels -- one image and one direction for the
# two Hessian kernels -- and one object slice for the Radon kernels), and the
# DRAM bytes of one launch that ncu captured (below).
KERNEL_BYTES = {
    # c read (its share per image), u's DCT-II rows written
    "k_casc_fwd": lambda r: 8 * r.nz * r.n + 8 * r.nzobj * r.nobj / r.ndist,
    # spectrum and data read; x0 and the g0 spectrum written
    "k_casc_resid": lambda r: 28 * r.nz * r.n,
    # spectrum and c read; P and the horizontal S^T rows written
    "k_casc_adj": lambda r: 16 * r.nz * r.n + 8 * r.nz * r.nobj + 8 * r.nzobj * r.nobj / r.ndist,
    # two directions: c, c_y, c_z and P read, two spectra written
    "k_casc_hess_fwd": lambda r: 12 * r.nz * r.n + 12 * r.nzobj * r.nobj / r.ndist,
    # two directions: two spectra, x0 and data read
    "k_casc_hess_q": lambda r: 14 * r.nz * r.n,
    # one column pass of one image, in place
    "k_dct_cols": lambda r: 16 * r.nz * r.n,
    # the Fourier-grid disc the polar samples reach (radius n + m) read; sinogram rows written
    "k_tgather": lambda r: 8 * np.pi * (r.nobj + 4) ** 2 + 8 * r.ntheta * r.nobj,
    # sinogram spectra read; the 2n x 2n Fourier grid written
    "k_tcell": lambda r: 8 * r.ntheta * r.nobj + 32 * r.nobj ** 2,
}
# (dram__bytes_read.sum + dram__bytes_write.sum) of one captured launch, its
# work units and the case it ran on; traffic at other sizes is this ratio to
# the algorithmic bytes times the algorithmic bytes there.  The Radon kernels'
# capture keeps the benchmark's angle density (448 angles at 256, 900 at 512),
# since k_tcell's pair lists grow with it.
_CASE_512_96 = types.SimpleNamespace(n=512, nz=512, nobj=512, nzobj=512, ntheta=96, ndist=4)
_CASE_256_448 = types.SimpleNamespace(n=256, nz=256, nobj=256, nzobj=256, ntheta=448, ndist=4)
NCU_CAPTURE = {
    "k_casc_fwd": (0.967394e9, 384, _CASE_512_96),
    "k_casc_resid": (2.769351e9, 384, _CASE_512_96),
    "k_casc_adj": (2.659368e9, 384, _CASE_512_96),
    "k_casc_hess_fwd": (3.426991e9, 2 * 384, _CASE_512_96),
    "k_casc_hess_q": (2.828069e9, 2 * 384, _CASE_512_96),
    "k_dct_cols": (1.569036e9, 384, _CASE_512_96),
    "k_tgather": (0.651061e9, 256, _CASE_256_448),
    "k_tcell": (0.797557e9, 256, _CASE_256_448),   # the pair lists come from DRAM once (group-major block order)
}


def ncu_traffic_ratio(k):
    if k not in NCU_CAPTURE:
        return None
    b, units, case = NCU_CAPTURE[k]
    return b / (KERNEL_BYTES[k](case) * units)


def kernel_times(rec):
    """Per-kernel launches, mean CUDA-event duration and work units recorded
    by the library's timers during the plain timed iterations."""
    import ctypes
    from holotomocupy_b200 import _lib
    out = {}
    for k in KERNEL_BYTES:
        ms, n, u = ctypes.c_double(), ctypes.c_long(), ctypes.c_double()
        _lib.call("ht_ktimer_read", k.encode(), ctypes.byref(ms), ctypes.byref(n), ctypes.byref(u))
        _lib.call("ht_ktimer_arm", k.encode(), 0)
        if n.value:
            per_unit = float(KERNEL_BYTES[k](rec))
            out[k] = {"launches": n.value, "ms": ms.value / n.value, "units": u.value / n.value,
                      "alg_bytes": per_unit * u.value / n.value}
    return out


def roofline(kt):
    """The dominant kernel (largest summed time) against the measured HBM
    copy bandwidth, and the same figures for the other timed kernels."""
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    if not kt:
        return None
    rows = {}
    for k, v in kt.items():
        gbs = v["alg_bytes"] / (v["ms"] * 1e-3) / 1e9
        ratio = ncu_traffic_ratio(k)
        traffic = ratio * v["alg_bytes"] if ratio is not None else None   # per launch
        rows[k] = {"launch_ms": v["ms"], "launches": v["launches"], "alg_bytes": v["alg_bytes"], "achieved": gbs,
                   "frac": gbs / peak, "traffic": traffic, "total_ms": v["ms"] * v["launches"]}
    dom = max(rows, key=lambda k: rows[k]["total_ms"])
    d = rows[dom]
    return {"bound": "hbm", "kernel": dom, "achieved": d["achieved"], "peak": peak, "unit": "GB/s",
            "frac": d["frac"], "traffic": d["traffic"], "peak_source": "measured" if peaks else "fallback",
            "launch_ms": d["launch_ms"],
            "traffic_source": "ncu dram bytes / algorithmic bytes of one captured launch (512^3 x 96 angles; "
                              "256^3 x 448 angles for the Radon kernels), times the "
                              "algorithmic bytes of this launch",
            "kernels": rows}


def end_to_end(a, rec, obj_true, prb0, pos0, data, device, barrier, world):
    """Each step: upload data and the initial state from pinned host memory,
    run e2e-iters BH iterations through Rec.BH, download obj, prb and pos."""
    import torch
    h_data = data.cpu().pin_memory()
    h_prb = prb0.cpu().pin_memory()
    h_pos = pos0.cpu().pin_memory()
    h_obj = torch.zeros(rec.nzobj, rec.nobj, rec.nobj, dtype=torch.complex64).pin_memory()
    out_obj = torch.empty_like(h_obj).pin_memory()
    out_prb = torch.empty_like(h_prb).pin_memory()
    out_pos = torch.empty_like(h_pos).pin_memory()
    h2d = sum(t.numel() * t.element_size() for t in (h_data, h_prb, h_pos, h_obj))
    d2h = sum(t.numel() * t.element_size() for t in (out_obj, out_prb, out_pos))
    times = []
    for s in range(a.e2e_steps + 1):
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for d in (rec.grads, rec.etas):
            for v in d.values():
                v.zero_()
        rec.data.copy_(h_data, non_blocking=True)
        rec.vars["obj"].copy_(h_obj, non_blocking=True)
        rec.vars["prb"].copy_(h_prb, non_blocking=True)
        rec.vars["pos"].copy_(h_pos, non_blocking=True)
        rec.BH(niter=a.e2e_iters, mode="graph")
        out_obj.copy_(rec.vars["obj"], non_blocking=True)
        out_prb.copy_(rec.vars["prb"], non_blocking=True)
        out_pos.copy_(rec.vars["pos"], non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        if s > 0:
            times.append(e0.elapsed_time(e1))
    ms = max_over_ranks([float(np.mean(times))], device)[0]   # the slowest replica (every rank calls this)
    return {"value": world * a.e2e_iters * 1e3 / ms, "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "iterations_per_step": a.e2e_iters, "ms_per_step": ms,
            "step": "upload data + initial obj/prb/pos from pinned host memory, Rec.BH(mode='graph') with the "
                    "iterations, download obj/prb/pos"}


if __name__ == "__main__":
    main()
