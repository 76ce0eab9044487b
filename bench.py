#!/usr/bin/env python
"""Benchmark: converged helium resonance solves per second on B200, mixed
precision against plain FP64.

Workload (default ``solve-n6``): the reference's own logged configuration
(CSCALE-WORK/Outs/Out.S.D2d0.T0.2d0.N6.petsc: singlet, N=6 so NN=13 points
per axis and a 4,826,809-dimensional two-electron space, DELTA=2, THETA=0.2,
GPLMR with NEV=1, NS=5 and the BASIC inner solve of order 5, shift
-0.7131541429), solved to a residual of 1e-8 from a seeded complex-Gaussian
singlet start vector.  One step = one solve.  The headline is the mixed form
(``--precision mixed``: complex64 inner solve, FP64 outer iteration); the
plain FP64 form is timed beside it on the same start vector and the line
reports both rates and |dE| between them.

  value  solves/s with the start vector already in HBM (de_gplmr_eig_d)
  e2e    solves/s through the C ABI with host buffers (de_gplmr_eig: the
         start vector is copied host->device and the Ritz vector back)
  roofline  the dominant kernel (the FP32 matvec in the mixed form, the FP64
         matvec in the plain form; two passes per vector), timed with CUDA
         events recorded by the library on its stream over the timed region;
         the other matvec is reported beside it
  cpu_baseline  the oracle (the reference's loops restated: HAMMULT in C
         with OpenMP on all host cores, the inner solve and block operations
         in numpy/LAPACK) timed on a bounded sample, a few preconditioned
         blocks of one GPLMR iteration, and scaled by the blocks per
         iteration and the iterations the GPU solve took

Other workloads: ``matvec-n9`` / ``matvec-n8`` / ``matvec-n6`` (one step =
H applied to a block of vectors, FP64 and FP32 with the relative error per
call, CUDA-core and tensor-core kernels), ``serve`` (a seeded Poisson
stream of uneven solve requests through the server: solves/s, p50/p99) and
``batch`` (64 uneven requests queued at once).  Their roofline is the
stream's matvec flops over its wall time, a lower bound; their CPU
baseline charges each request oracle block times for its grid.

``--impl reference`` runs that CPU path alone (rank 0) and prints its line.
Multi-GPU: independent replicas (one solve stream per rank, no collective
on the data path); value = solves of all ranks / max rank time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: grid/solver settings; iters_ref = GPLMR iterations to converge
    # from this seeded start (deterministic; the CPU oracle and the GPU solver
    # agree), used only by the CPU arm to convert matvec time to solve time.
    "solve-n6": dict(n=6, delta=2.0, theta=0.2, nev=1, ns=5, order=5, sigma=-0.7131541429, tol=1e-8,
                     seed=0, spin="singlet", maxit=200, iters_ref=50),
    "solve-n5": dict(n=5, delta=2.0, theta=0.2, nev=1, ns=5, order=5, sigma=-0.7131541429, tol=1e-9,
                     seed=0, spin="singlet", maxit=200, iters_ref=52),
    # the full resonance-solve configuration restated on this grid: N=8,
    # theta=0.35, eight resonances nearest each shift (run with --start guess)
    "solve-n8-nev8": dict(n=8, delta=2.0, theta=0.35, nev=8, ns=5, order=5, sigma=-0.78, tol=1e-8,
                          seed=2, spin="singlet", maxit=200, iters_ref=None),
    "solve-n8-nev8-s060": dict(n=8, delta=2.0, theta=0.35, nev=8, ns=5, order=5, sigma=-0.60, tol=1e-8,
                               seed=2, spin="singlet", maxit=200, iters_ref=None),
}

# Block-matvec throughput (one step = H applied to a block of vectors): the
# FP64 plain matvec and the mixed form's complex64 matvec on the same block,
# with the mixed result's relative error against the FP64 one per call.
MATVEC = {
    "matvec-n9": dict(n=9, theta=0.35, nvec=16, seed=1),
    "matvec-n8": dict(n=8, theta=0.35, nvec=16, seed=1),
    "matvec-n6": dict(n=6, theta=0.35, nvec=2, seed=1),  # small case for kernel captures
}


# Served stream: Poisson arrivals of uneven solve requests (seeded); sizes
# are the batched configuration's mix scaled to grids a few-minute run can
# finish (N 3-6 instead of 4-8) and to one resonance per request (with the
# shift near the 2s^2 resonance, the second-nearest eigenvalue of a seeded
# two-column start is a rotated-continuum state on which GPLMR stalls, or
# whose inner-solve Gram matrix fails the reference's 1e-10 self-check).
SERVE = dict(requests=40, rate=40.0, seed=4, ns=[3, 4, 5, 6], n_weights=[0.2, 0.3, 0.3, 0.2],
             thetas=[0.20, 0.25, 0.30, 0.35, 0.40, 0.45, 0.50], nevs=[1], spins=["singlet", "triplet"],
             sigma=-0.7131541429, tol=1e-9, maxit=200, workers=4)


def serve_requests(cfg):
    import numpy as np

    rng = np.random.Generator(np.random.PCG64(cfg["seed"]))
    t = 0.0
    out = []
    for k in range(cfg["requests"]):
        t += rng.exponential(1.0 / cfg["rate"]) if cfg["rate"] else 0.0
        out.append(dict(t=t, n=int(rng.choice(cfg["ns"], p=cfg["n_weights"])), theta=float(rng.choice(cfg["thetas"])),
                        nev=int(rng.choice(cfg["nevs"])), spin=str(rng.choice(cfg["spins"])), seed=1000 + k))
    return out


def run_served(de, seeded_start, cfg, precision, workers=None):
    """Replay the arrival schedule against a Server; latencies from the
    server clock (submission to completion)."""
    import numpy as np

    reqs = serve_requests(cfg)
    srv = de.Server(workers=workers or cfg["workers"])
    built = []
    guesses = {}
    for r in reqs:
        m = (2 * r["n"] + 1) ** 3
        if cfg.get("start") == "guess":  # the reference's initial guess, formed before the stream
            key = (r["n"], r["theta"], r["spin"], r["nev"])
            if key not in guesses:
                with de.Problem(n=r["n"], delta=2.0, theta=r["theta"]) as h:
                    guesses[key] = h.subspace_guess(14, r["spin"] == "singlet", False, cfg["sigma"], r["nev"])[1]
            x0 = guesses[key]
        else:
            x0 = seeded_start(m, r["nev"], r["seed"], r["spin"])
        built.append(srv.request(r["n"], x0, cfg["sigma"], theta=r["theta"], precision=precision, ns=5,
                                 maxit=cfg["maxit"], tol=cfg["tol"]))
    done = {}
    t0 = srv.now()
    k = 0
    while len(done) < len(reqs):
        now = srv.now() - t0
        while k < len(reqs) and reqs[k]["t"] <= now:
            srv.submit(built[k], tag=k)
            k += 1
        nxt = (reqs[k]["t"] - now) if k < len(reqs) else 1.0
        res = srv.wait_any(max(1e-4, min(nxt, 1.0)))
        if res is not None:
            done[res.tag] = res
    t_end = max(r.t_end_s for r in done.values()) - t0
    srv.close()
    lat = np.array([done[i].latency_s for i in range(len(reqs))])
    ok = [done[i].status == 0 for i in range(len(reqs))]
    conv = [done[i].converged for i in range(len(reqs))]
    return {"solves_per_s": len(reqs) / t_end, "wall_s": t_end, "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()), "ok": int(sum(ok)),
            "converged": int(sum(conv)), "e": {i: done[i].e.copy() for i in range(len(reqs))},
            "conv": {i: bool(done[i].converged and done[i].status == 0) for i in range(len(reqs))},
            "iters": {i: int(done[i].iterations) for i in range(len(reqs))},
            "matvecs": {i: int(done[i].matvecs) for i in range(len(reqs))},
            "not_converged": [dict(reqs[i], status=int(done[i].status)) for i in range(len(reqs))
                              if not (done[i].converged and done[i].status == 0)]}


def hammults_per_solve(w, iters):
    """The reference's HAMMULT count (ICALLED) for a solve of `iters`
    iterations: NEV for the start, then per iteration (1+NS) MATBLOCKs of NEV
    and (1+NS) PRECBLOCK_BASIC calls of (2*order+1) products of NEV."""
    nev, ns, order = w["nev"], w["ns"], w["order"]
    return nev + iters * (1 + ns) * (nev + nev * (2 * order + 1))


def alg_flops(nn):
    """Algorithmic FP64 flops of one vector-matvec: 6 axes x NN MACs x 2
    flops x 2 (re, im) per element, plus the complex potential multiply-add."""
    return 24 * nn ** 7 + 8 * nn ** 6


def alg_bytes(nn):
    """Read x and write y once, complex128."""
    return 32 * nn ** 6


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum, pass A + pass B)
# per vector-matvec of the kernels the library picks, keyed by (NN,
# storage): one ncu capture of the block-of-2 matvec at N=6 (`--workload
# matvec-n6`), both passes' bytes over 2 vectors: ev_kernel<float, 13> and
# ev_kernel<double, 13>.  Kernels without a capture report null.
NCU_TRAFFIC_PER_VECTOR = {(13, "f32"): 149.3e6, (13, "f64"): 342.6e6}

# The timed solves keep the library's matvec events on for the roofline
# figures, on every 8th MATBLOCK call of each storage: all calls of one
# solve are the same kernels on the same sizes, and the events' own cost
# (a few microseconds a call) stays out of the timed work.
PROFILE_EVERY = 8


def solve_config(a, w):
    """The workload's config dict, printed identically by both arms."""
    nn = 2 * w["n"] + 1
    return {"workload": a.workload, "start": a.start, "N": w["n"], "NN": nn, "dim": nn ** 6, "nev": w["nev"],
            "ns": w["ns"], "order": w["order"], "theta": w["theta"], "delta": w["delta"], "sigma": w["sigma"],
            "tol": w["tol"], "spin": w["spin"], "seed": w["seed"],
            "l2": "inputs larger than L2 (GPLMR workspace "
                  f"{(17 + 2 * w['order']) * w['nev'] * nn ** 6 * 16 / 1e9:.1f} GB per solve)"}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def fp64_peak_tflops(torch):
    """Measured FP64 dense peak on this GPU: cuBLAS DGEMM 8192^3 (FP64 tensor
    cores), best of 5 -- the compute denominator of the matvec roofline."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2 * n ** 3 / best / 1e12


def fp32_peak_tflops(torch):
    """Measured FP32 CUDA-core peak: cuBLAS SGEMM 8192^3 with TF32 off, best
    of 5 -- the compute denominator of the FP32 matvec roofline."""
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = 8192
        a = torch.randn(n, n, dtype=torch.float32, device="cuda")
        b = torch.randn(n, n, dtype=torch.float32, device="cuda")
        for _ in range(2):
            torch.matmul(a, b)
        best = 1e30
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        del a, b
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old
    return 2 * n ** 3 / best / 1e12


def cpu_matvec_seconds(w, reps):
    """Seconds per oracle HAMMULT (C, OpenMP over columns, all host cores)."""
    from oracle import oracle as O  # CPU baseline only

    p = O.Params(n=w["n"], delta=w["delta"], theta=w["theta"])
    h = O.init_hamiltonian(p, nelec=2)
    x = O.seeded_start(p, 1, w["seed"], w["spin"])[:, 0]
    h.matvec(x)  # warm
    t0 = time.perf_counter()
    for _ in range(reps):
        h.matvec(x)
    return (time.perf_counter() - t0) / reps, os.cpu_count()


def max_over_ranks(x, dist, device):
    """The slowest rank's time: every rank contributes its own and all get
    the maximum (replica timing; no data-path collective)."""
    import torch

    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, world, seconds):
    """Whole-job throughput of N independent replicas timed as the max over
    ranks: all ranks' units over the slowest rank's time."""
    return units_per_rank * world / seconds


def dist_setup():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def matvec_kernel_name(nn, fp32):
    """The kernels the library picks for a grid (de_set_matvec_kernel's
    default): even/odd-split kernels for complex64 at NN 9..17 and
    complex128 at NN 9..13, streaming kernels at NN 15..19, cube kernels
    elsewhere."""
    r = "float" if fp32 else "double"
    if 9 <= nn <= (17 if fp32 else 13):
        return f"hammult ev_kernel<{r}, {nn}> pass A + pass B"
    if 13 <= nn <= 19:
        return f"hammult stream_kernel<{r}, {nn}> pass A + pass B"
    return f"hammult cube_kernel<{r}, {nn}> pass A + pass B"


class OracleBlockStep:
    """One sixth of a GPLMR iteration of the oracle (the reference's loops
    restated: C HAMMULT with OpenMP over all host cores, the BASIC inner
    solve and block operations in numpy/LAPACK).  An iteration
    preconditions and multiplies 1 + NS blocks the same way
    (gplmr.F90:92-190); this is one of them: PRECBLOCK_BASIC on the residual
    block, projection against X, cholQR and MATBLOCK."""

    def __init__(self, w):
        import numpy as np

        from oracle import oracle as O  # the reference arm's CPU restatement

        self.O = O
        p = O.Params(n=w["n"], delta=w["delta"], theta=w["theta"])
        self.h = O.init_hamiltonian(p, nelec=2)
        x = O.seeded_start(p, w["nev"], w["seed"], w["spin"])
        self.x = x / O.colnorms(x)[None, :]
        ax = self.h.matblock(self.x)
        e = np.einsum("ij,ij->j", self.x.conj(), ax)
        self.r = ax - self.x * e[None, :]
        self.w = w

    def seconds(self):
        O, w = self.O, self.w
        t0 = time.perf_counter()
        b = O.basicblocklansolve(self.r, w["order"], self.h.params.m ** 2, complex(w["sigma"], 0.0),
                                 self.h.matblock)
        b = b - self.x @ O.hdot(self.x, b)
        O.cholqr(b)
        self.h.matblock(b)
        return time.perf_counter() - t0


def serve_roofline(reqs, matvecs, wall_s, peak_tflops):
    """The served or batched stream's matvec work rate: the algorithmic
    flops of every vector-matvec of every request (alg_flops at its grid)
    over the stream's wall time.  The wall time also holds everything that
    is not a matvec, so this is a lower bound on the matvec kernels' own
    rate; the denominator is the measured FP32 peak, as for the mixed
    form's matvec."""
    flops = sum(matvecs[i] * alg_flops(2 * r["n"] + 1) for i, r in enumerate(reqs))
    achieved = flops / wall_s / 1e12
    return {"bound": "fp32-fma", "achieved": achieved, "peak": peak_tflops, "unit": "TFLOP/s",
            "frac": achieved / peak_tflops, "traffic": None,
            "kernel": "all vector-matvecs of the stream (both precisions) over its wall time: a lower bound",
            "matvecs": int(sum(matvecs.values())), "alg_flops": float(flops), "wall_s": wall_s}


def serve_cpu_baseline(cfg, reqs, iters, ns=5):
    """The oracle on a served or batched mix, one solve at a time on all
    host cores (the reference runs one solve per job).  One preconditioned
    block with one column (OracleBlockStep) is timed per grid size N of the
    mix; each request is charged that time x its NEV (the block's matvecs,
    inner solve and projections grow with the columns) x (1 + NS) blocks
    per iteration (gplmr.F90:92-190) x the iterations its GPU solve took."""
    t_blk = {}
    for n in sorted({r["n"] for r in reqs}):
        w = dict(n=n, delta=2.0, theta=cfg["thetas"][0], nev=1, seed=0, spin="singlet", order=5,
                 sigma=cfg["sigma"], ns=ns)
        t_blk[n] = OracleBlockStep(w).seconds()
    cpu_s = sum(t_blk[r["n"]] * r["nev"] * (1 + ns) * max(1, iters[i]) for i, r in enumerate(reqs))
    cores = os.cpu_count()
    blocks = ", ".join(f"N={n} {t:.3f} s" for n, t in t_blk.items())
    return {"value": len(reqs) / cpu_s, "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": f"one preconditioned one-column block of the oracle per grid size ({blocks}: "
                      f"PRECBLOCK_BASIC, projection, cholQR, MATBLOCK; C HAMMULT with OpenMP on {cores} "
                      f"threads, block operations in numpy/LAPACK) x NEV x {1 + ns} blocks per iteration "
                      f"x each request's GPU iteration count, summed over the {len(reqs)} requests "
                      f"(one solve at a time)"}


def run_reference(a, w):
    """--impl reference: the reference's CPU path (the oracle restatement: the
    Fortran/MPI/PETSc program cannot be built on this image) on the same
    workload.  One step = one of the 1 + NS preconditioned blocks of a GPLMR
    iteration (OracleBlockStep), block operations included; ms_per_step is
    that measured time.  solves/s = 1 / (median step time x (1 + NS) x the
    workload's iterations to convergence)."""
    rank, world, local = dist_setup()
    if rank != 0:
        return 0
    iters = w["iters_ref"]
    if iters is None:
        print(json.dumps({"impl": "reference", "unavailable": "no converged iteration count recorded for this "
                                                              "workload (a complete CPU solve takes hours)"}))
        return 0
    step = OracleBlockStep(w)
    for _ in range(a.warmup):
        step.seconds()
    times = [step.seconds() for _ in range(a.steps)]
    cores = os.cpu_count()
    t_blk = statistics.median(times)
    v = 1.0 / (t_blk * (1 + w["ns"]) * iters)
    line = {
        "impl": "reference", "metric": "resonance solves/s", "value": v, "unit": "solves/s", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": t_blk * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": solve_config(a, w),
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": f"one step = one of the {1 + w['ns']} preconditioned blocks of a GPLMR iteration "
                                   f"of the oracle at N={w['n']} (PRECBLOCK_BASIC, projection, cholQR, MATBLOCK; C "
                                   f"HAMMULT with OpenMP on {cores} threads, block operations in numpy/LAPACK); "
                                   f"solves/s = 1 / (median {t_blk:.2f} s x {1 + w['ns']} blocks x {iters} "
                                   f"iterations to converge)"},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def matvec_main(a):
    """--workload matvec-*: block MATBLOCK throughput, FP64 and mixed (FP32)
    on the CUDA-core kernels (the default), the FP64 tensor-core kernels
    beside; value = FP64 vector-matvecs/s on the device."""
    import ctypes

    import numpy as np
    import torch

    import doublyexcited_b200 as de
    from doublyexcited_b200._lib import check, lib

    rank, world, local = dist_setup()
    w = MATVEC[a.workload]
    if a.impl == "reference":
        if rank != 0:
            return 0
        t = []
        for _ in range(a.steps):
            tm, cores = cpu_matvec_seconds(dict(n=w["n"], delta=2.0, theta=w["theta"], seed=w["seed"],
                                                spin="singlet"), 1)
            t.append(tm)
        v = 1.0 / statistics.median(t)
        print(json.dumps({"impl": "reference", "metric": "vector-matvecs/s", "value": v, "unit": "matvecs/s",
                          "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 / v,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic", "config": {"workload": a.workload, **w},
                          "cpu_baseline": {"value": v, "unit": "matvecs/s", "cores": cores, "kind": "port",
                                           "sample": f"{a.steps} oracle HAMMULTs (C, OpenMP, all cores)"},
                          "e2e": {"value": v, "unit": "matvecs/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return 0
    torch.cuda.set_device(local)
    nn = 2 * w["n"] + 1
    nv = w["nvec"]
    st = torch.cuda.current_stream()
    gen = torch.Generator(device="cuda").manual_seed(w["seed"])
    out = {}
    clocks = None
    launches = 0
    with de.Problem(n=w["n"], delta=2.0, theta=w["theta"], device=local) as g64, \
            de.Problem(n=w["n"], delta=2.0, theta=w["theta"], device=local, precision="mixed") as g32:
        dim = g64.dim
        x = torch.randn(nv, dim, dtype=torch.complex128, device="cuda", generator=gen)
        y = torch.empty_like(x)
        x32 = x.to(torch.complex64)
        y32 = torch.empty_like(x32)
        for g in (g64, g32):
            g.set_stream(st.cuda_stream)

        def timed(fn, steps):
            for _ in range(a.warmup):
                fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(steps):
                fn()
            e1.record(st)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / 1e3 / steps

        f64 = lambda: g64.matblock_d(x.data_ptr(), y.data_ptr(), nv)  # noqa: E731
        f32 = lambda: g32.matblock32_d(x32.data_ptr(), y32.data_ptr(), nv)  # noqa: E731
        sampler = ClockSampler(local)
        sampler.start()
        l0 = lib().de_kernel_launches()
        t64 = timed(f64, a.steps)
        launches = (lib().de_kernel_launches() - l0) * a.steps // (a.steps + a.warmup)
        clocks = sampler.stop()
        t32 = timed(f32, a.steps)
        rel = []
        for j in range(nv):
            rel.append((torch.linalg.norm(y32[j].to(torch.complex128) - y[j]) / torch.linalg.norm(y[j])).item())
        g64.set_matvec_kernel("tensor")
        g32.set_matvec_kernel("tensor")
        t64tc = timed(f64, a.steps)
        t32tc = timed(f32, a.steps)
        g64.set_matvec_kernel("fma")
        # end to end: host buffers through de_matblock (H2D + D2H per step)
        xh = x.cpu().numpy().T.copy(order="F")
        yh = np.empty_like(xh)
        t0 = time.perf_counter()
        e2e_steps = max(1, min(a.steps, 2))
        for _ in range(e2e_steps):
            check(lib().de_matblock(g64.handle, ctypes.c_void_p(xh.ctypes.data), ctypes.c_void_p(yh.ctypes.data),
                                    g64.m, dim // g64.m, nv), "de_matblock")
        torch.cuda.synchronize()
        t_e2e = (time.perf_counter() - t0) / e2e_steps
    peak64, peak32 = fp64_peak_tflops(torch), fp32_peak_tflops(torch)
    fl = alg_flops(nn) * nv

    def roof(t, pk, ebytes, kernel):
        ach = fl / t / 1e12
        return {"bound": "tensor" if ebytes == 32 else "fp32-fma", "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                "frac": ach / pk, "traffic": NCU_TRAFFIC_PER_VECTOR.get((nn, "f64" if ebytes == 32 else "f32")),
                "kernel": kernel, "ms_per_vector": t / nv * 1e3,
                "achieved_gbs_alg": ebytes * nn ** 6 * nv / t / 1e9}

    cpu = None
    if not a.no_cpu_baseline:
        tm, cores = cpu_matvec_seconds(dict(n=w["n"], delta=2.0, theta=w["theta"], seed=w["seed"], spin="singlet"), 1)
        cpu = {"value": 1.0 / tm, "unit": "matvecs/s", "cores": cores, "kind": "port",
               "sample": f"1 oracle HAMMULT at N={w['n']} (C, OpenMP over columns, {cores} threads)"}
    line = {"metric": "vector-matvecs/s", "value": nv / t64, "unit": "matvecs/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": t64 * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded complex-Gaussian block)",
            "config": {"workload": a.workload, **w, "NN": nn, "dim": nn ** 6,
                       "l2": f"block of {nv} x {16 * nn ** 6 / 1e6:.0f} MB"},
            "e2e": {"value": nv / t_e2e, "unit": "matvecs/s", "h2d_bytes_per_step": int(xh.nbytes),
                    "d2h_bytes_per_step": int(yh.nbytes)},
            "roofline": roof(t64, peak64, 32, matvec_kernel_name(nn, False)),
            "mixed": {"value": nv / t32, "unit": "matvecs/s", "speedup_vs_fp64": t64 / t32,
                      "rel_err_vs_fp64_max": max(rel),
                      "roofline": roof(t32, peak32, 16, matvec_kernel_name(nn, True))},
            "tensor_cores": {"fp64_value": nv / t64tc, "mixed_value": nv / t32tc,
                             "fp64_roofline": roof(t64tc, peak64, 32, "hammult tc kernels <double> (DMMA)")},
            "cpu_baseline": cpu, "gpu_launches": int(launches), "clocks": clocks}
    print(json.dumps(line))
    return 0


def serve_main(a):
    """--workload serve: the served stream, mixed and FP64 back to back on one
    GPU, one JSON line.  value = mixed solves/s over the stream."""
    import numpy as np
    import torch

    import doublyexcited_b200 as de
    from doublyexcited_b200.starts import seeded_start

    rank, world, local = dist_setup()
    if a.impl == "reference" or rank != 0:
        if a.impl == "reference" and rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving layer "
                              "(one GPLMR_EIG per MPI job)"}))
        return 0
    torch.cuda.set_device(local)
    cfg = dict(SERVE)
    if a.workload == "batch":
        # the batched configuration restated: 64 uneven problems all queued
        # at once, from the reference's initial guess, 1, 2 or 4 resonances
        cfg.update(requests=64, rate=0.0, seed=3, start="guess", nevs=[1, 2, 4])
    if a.workers:
        cfg["workers"] = a.workers
    if a.start == "guess":  # starts from the initial guess: several resonances per request
        cfg["start"], cfg["nevs"] = "guess", [1, 2, 4]
    # warm-up (untimed): the operator tables of every grid size (the TINV
    # solve is cached per process) and the kernels of both precisions
    for n in cfg["ns"]:
        m = (2 * n + 1) ** 3
        for prec in ("mixed", "fp64"):
            with de.Problem(n=n, delta=2.0, theta=cfg["thetas"][0], precision=prec) as h:
                h.gplmr_eig(seeded_start(m, 1, 0, "singlet"), cfg["sigma"], ns=5, maxit=2, tol=cfg["tol"])
    sampler = ClockSampler(local)
    l0 = de.lib().de_kernel_launches()
    sampler.start()
    mixed = run_served(de, seeded_start, cfg, "mixed")
    clocks = sampler.stop()
    launches = de.lib().de_kernel_launches() - l0
    fp64 = run_served(de, seeded_start, cfg, "fp64")
    # the plain FP64 solver: one solve at a time, in arrival order
    plain = run_served(de, seeded_start, cfg, "fp64", workers=1)
    # the mixed solver one solve at a time (what concurrency adds)
    mixed1 = run_served(de, seeded_start, cfg, "mixed", workers=1) if a.workload == "batch" else None
    reqs = serve_requests(cfg)
    roofline = serve_roofline(reqs, mixed["matvecs"], mixed["wall_s"], fp32_peak_tflops(torch))
    cpu = None if a.no_cpu_baseline else serve_cpu_baseline(cfg, reqs, mixed["iters"])
    both = [i for i in mixed["e"] if mixed["conv"][i] and fp64["conv"][i]]
    de_max = max((float(np.max(np.abs(np.sort_complex(mixed["e"][i]) - np.sort_complex(fp64["e"][i]))))
                  for i in both), default=None)
    strip = lambda d: {k: v for k, v in d.items() if k not in ("e", "conv", "iters", "matvecs")}  # noqa: E731
    name = "batched uneven solves" if a.workload == "batch" else "served stream"
    line = {"metric": f"resonance solves/s ({name})", "value": mixed["solves_per_s"], "unit": "solves/s",
            "n_gpus": 1, "steps": cfg["requests"], "warmup": 2 * len(cfg["ns"]), "ms_per_step": mixed["wall_s"] / cfg["requests"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 inner solve / f64 outer iteration", "data": ("synthetic (64 problems queued at once, " if a.workload == "batch" else
                                                                   "synthetic (seeded Poisson arrivals, ")
                    + ("starts from the reference's initial guess)" if cfg.get("start") == "guess" else "seeded starts)"),
            "config": {"workload": a.workload, **{k: v for k, v in cfg.items()}},
            "p50_s": mixed["p50_s"], "p99_s": mixed["p99_s"], "mixed": strip(mixed), "fp64": strip(fp64),
            "fp64_one_at_a_time": strip(plain),
            "mixed_one_at_a_time": strip(mixed1) if mixed1 else None,
            "speedup_vs_fp64": mixed["solves_per_s"] / fp64["solves_per_s"],
            "speedup_vs_plain_fp64_solver": mixed["solves_per_s"] / plain["solves_per_s"],
            "dE_mixed_vs_fp64_max": de_max,
            "dE_compared": len(both),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "gpu_launches": int(launches), "clocks": clocks}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="solve-n6",
                    choices=sorted(WORKLOADS) + sorted(MATVEC) + ["serve", "batch"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="mixed: FP32 inner solve, FP64 outer iteration (the product form); fp64: plain")
    ap.add_argument("--no-fp64-compare", action="store_true",
                    help="skip the plain-FP64 solves timed beside the mixed ones")
    ap.add_argument("--workers", type=int, default=None, help="serve: concurrent solves (CUDA streams)")
    ap.add_argument("--start", default="seeded", choices=["seeded", "guess"],
                    help="seeded complex-Gaussian start blocks, or the reference's initial guess "
                         "(de_subspace_guess: 14 He+ orbitals, etarget = sigma), formed before timing; "
                         "with serve, guess starts also let requests ask for 1, 2 or 4 resonances")
    ap.add_argument("--maxit", type=int, default=None,
                    help="cap the GPLMR iterations (short runs for kernel profiling; not a bench value)")
    a = ap.parse_args()
    if a.workload in ("serve", "batch"):
        return serve_main(a)
    if a.workload in MATVEC:
        return matvec_main(a)
    w = dict(WORKLOADS[a.workload])
    if a.maxit is not None:
        w["maxit"] = a.maxit
    if a.impl == "reference":
        return run_reference(a, w)

    import numpy as np
    import torch

    import doublyexcited_b200 as de
    from doublyexcited_b200.starts import seeded_start

    rank, world, local = dist_setup()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist

    def barrier():
        if pg:
            pg.barrier()

    nn = 2 * w["n"] + 1
    import ctypes

    from doublyexcited_b200._lib import check, de_complex, de_gmres, de_stats, lib

    L = lib()
    gm = de_gmres(w["order"], 1, 1e-3, 0)
    sig = de_complex(w["sigma"], 0.0)
    stream = torch.cuda.current_stream()

    def measure(precision, sample_clocks):
        """W untimed + K timed solves at one precision, device-timed."""
        prob = de.Problem(n=w["n"], delta=w["delta"], theta=w["theta"], device=local, precision=precision)
        prob.set_stream(stream.cuda_stream)
        if a.start == "guess":
            _, x0 = prob.subspace_guess(14, w["spin"] == "singlet", False, w["sigma"], w["nev"])
        else:
            x0 = seeded_start(prob.m, w["nev"], w["seed"], w["spin"])
        dim = prob.dim
        x0_dev = torch.from_numpy(np.ascontiguousarray(x0.T)).to("cuda")  # (nev, dim): columns contiguous
        x_dev = torch.empty_like(x0_dev)
        e_host = np.empty(w["nev"], np.complex128)

        def solve_dev():
            x_dev.copy_(x0_dev)
            st = de_stats()
            check(L.de_gplmr_eig_d(prob.handle, ctypes.c_void_p(x_dev.data_ptr()),
                                   ctypes.c_void_p(e_host.ctypes.data), prob.m, dim // prob.m, sig, w["nev"],
                                   w["ns"], w["maxit"], w["tol"], ctypes.byref(gm), 0, ctypes.byref(st)),
                  "de_gplmr_eig_d")
            return st

        for _ in range(a.warmup):
            solve_dev()
        torch.cuda.synchronize()
        barrier()
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.start()
        prob.set_profiling(True, every=PROFILE_EVERY)
        prob.profile_read()
        prob.profile_read32()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        marks = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
        launches0 = L.de_kernel_launches()
        e0.record(stream)
        stats = []
        for i in range(a.steps):
            marks[i].record(stream)
            stats.append(solve_dev())
        marks[a.steps].record(stream)
        e1.record(stream)
        launches = L.de_kernel_launches() - launches0
        torch.cuda.synchronize()
        elapsed = e0.elapsed_time(e1) / 1e3
        per_solve = [marks[i].elapsed_time(marks[i + 1]) / 1e3 for i in range(a.steps)]
        barrier()
        clocks = sampler.stop() if sampler else None
        prof = prob.profile_read()
        prof32 = prob.profile_read32()
        prob.set_profiling(False)
        if pg:
            elapsed = max_over_ranks(elapsed, pg, "cuda")
        out = {"prob": prob, "x0": x0, "dim": dim, "elapsed": elapsed, "stats": stats, "st": stats[-1],
               "e": complex(e_host[0]), "e_all": e_host.copy(), "prof": prof, "prof32": prof32,
               "launches": launches, "per_solve": per_solve,
               "clocks": clocks, "value": replica_rate(a.steps, world, elapsed)}
        del x_dev, x0_dev
        return out

    head = measure(a.precision, True)
    other, other_err = None, None
    if a.precision != "fp64" and not a.no_fp64_compare:
        try:
            other = measure("fp64", False)
        except de.DeError as exc:  # e.g. the reference's 1e-10 self-check STOP at NEV > 1
            other_err = str(exc)
    prob, x0, dim = head["prob"], head["x0"], head["dim"]
    elapsed, st, e_final, prof, launches, clocks = (head["elapsed"], head["st"], head["e"], head["prof"],
                                                     head["launches"], head["clocks"])
    value = head["value"]
    lat = np.array(head["per_solve"])
    latency = {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
               "solves": len(lat), "note": "device time per solve, one solve at a time"}
    e_host = np.empty(w["nev"], np.complex128)

    # end to end through the host-pointer C ABI (pinned host buffers)
    x_pin = torch.from_numpy(np.asfortranarray(x0).reshape(-1, order="F").view(np.float64)).pin_memory()
    x_host = x_pin.numpy().view(np.complex128).reshape(x0.shape, order="F")
    x_work = torch.empty_like(x_pin).pin_memory()
    xw = x_work.numpy().view(np.complex128).reshape(x0.shape, order="F")
    prob.set_stream(0)
    # the same K steps and the same profiling state as the device-timed value
    prob.set_profiling(True, every=PROFILE_EVERY)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    e2e_steps = a.steps
    for _ in range(e2e_steps):
        np.copyto(xw, x_host)
        st2 = de_stats()
        check(L.de_gplmr_eig(prob.handle, ctypes.c_void_p(xw.ctypes.data), ctypes.c_void_p(e_host.ctypes.data),
                             prob.m, dim // prob.m, sig, w["nev"], w["ns"], w["maxit"], w["tol"], ctypes.byref(gm), 0,
                             ctypes.byref(st2)), "de_gplmr_eig")
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t0
    prob.profile_read()
    prob.profile_read32()
    prob.set_profiling(False)
    if pg:
        t_e2e = max_over_ranks(t_e2e, pg, "cuda")
    e2e = replica_rate(e2e_steps, world, t_e2e)

    peak = fp64_peak_tflops(torch)
    peak32 = fp32_peak_tflops(torch)

    def roof(pr, fp32, pk, src):
        ms = pr["pass_a_ms"] + pr["pass_b_ms"]
        vecs = max(1, pr["vectors"])
        ach = alg_flops(nn) * vecs / (ms / 1e3) / 1e12 if ms > 0 else 0.0
        ebytes = 16 if fp32 else 32
        return {"bound": "tensor" if not fp32 else "fp32-fma", "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                "frac": ach / pk if pk else None,
                "traffic": NCU_TRAFFIC_PER_VECTOR.get((nn, "f32" if fp32 else "f64")),
                "kernel": matvec_kernel_name(nn, fp32) + ", per vector-matvec",
                "alg_flops_per_vector": alg_flops(nn), "alg_bytes_per_vector": ebytes * nn ** 6,
                "achieved_gbs_alg": ebytes * nn ** 6 * vecs / (ms / 1e3) / 1e9 if ms > 0 else None,
                "matvec_ms_per_vector": ms / vecs, "pass_a_ms": pr["pass_a_ms"] / vecs,
                "pass_b_ms": pr["pass_b_ms"] / vecs, "vectors": pr["vectors"], "device_ms_total": ms,
                "peak_source": src}

    src64 = "FP64 dense peak measured in this run: cuBLAS DGEMM 8192^3 (no FP64 entry in MEASURED_PEAKS.json)"
    src32 = "FP32 CUDA-core peak measured in this run: cuBLAS SGEMM 8192^3 with TF32 off"
    roof64 = roof(prof, False, peak, src64)
    roof32 = roof(head["prof32"], True, peak32, src32) if head["prof32"]["vectors"] else None
    # the dominant kernel of the run heads the line
    if roof32 and roof32["device_ms_total"] > roof64["device_ms_total"]:
        roofline, roofline_other = roof32, roof64
    else:
        roofline, roofline_other = roof64, roof32

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline and w["n"] <= 6:
        step = OracleBlockStep(w)
        t_blk = statistics.median([step.seconds() for _ in range(3)])
        cores = os.cpu_count()
        cpu = {"value": 1.0 / (t_blk * (1 + w["ns"]) * st.iterations), "unit": "solves/s", "cores": cores,
               "kind": "port",
               "sample": f"3 x one preconditioned block of a GPLMR iteration of the oracle at N={w['n']} (median "
                         f"{t_blk:.2f} s: PRECBLOCK_BASIC, projection, cholQR, MATBLOCK; C HAMMULT with OpenMP on "
                         f"{cores} threads, block operations in numpy/LAPACK) x {1 + w['ns']} blocks per "
                         f"iteration x the {st.iterations} iterations this solve took"}

    compare = {"fp64_error": other_err} if other_err else None
    if other is not None:
        de_max = float(np.max(np.abs(np.sort_complex(head["e_all"]) - np.sort_complex(other["e_all"]))))
        olat = np.array(other["per_solve"])
        compare = {"fp64_value": other["value"], "fp64_ms_per_step": other["elapsed"] / a.steps * 1e3,
                   "fp64_p50_s": float(np.percentile(olat, 50)), "fp64_p99_s": float(np.percentile(olat, 99)),
                   "fp64_iterations": other["st"].iterations, "fp64_E": [other["e"].real, other["e"].imag],
                   "speedup_vs_fp64": value / other["value"], "dE_vs_fp64": de_max}
        other["prob"].close()

    if rank == 0:
        line = {
            "metric": "resonance solves/s", "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": elapsed / a.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if a.precision == "fp64" else "f32 inner solve / f64 outer iteration",
            "data": ("synthetic (seeded complex-Gaussian singlet start vector; operator from the reference's physics)"
                     if a.start == "seeded" else
                     "synthetic operator from the reference's physics; start block from the reference's initial guess"),
            "config": solve_config(a, w),
            "precision": a.precision, "parallelism": f"replicas x{world}",
            "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": int(x0.nbytes),
                    "d2h_bytes_per_step": int(x0.nbytes + e_host.nbytes)},
            "roofline": roofline,
            "roofline_other_matvec": roofline_other,
            "cpu_baseline": cpu,
            "latency": latency,
            "mixed_vs_fp64": compare,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "solve": {"iterations": st.iterations, "converged": bool(st.converged), "E": [e_final.real, e_final.imag],
                      "max_residual": st.max_residual, "matvecs": st.matvecs,
                      "matvecs_reference": st.matvecs_reference, "t_prec_s": st.t_prec_s,
                      "t_dense_s": st.t_dense_s},
        }
        print(json.dumps(line))
    prob.close()
    if pg:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
