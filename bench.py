#!/usr/bin/env python
"""Benchmark of the Krylov-solve path on one node.

Workload (one "step" = one complete solve from x0 = 0 to a 1e-8 relative
residual): W2-W3 Helmholtz-type operator A = M2 + 0.1 D^T D on an extruded
C96 cubed sphere with 30 levels (1 658 880 cells, 5 031 936 W2 dofs; seeded
perturbed geometry, b ~ N(0,1)), GMRES(10) preconditioned by a column
tridiagonal on the vertical faces and Jacobi on the horizontal faces.

  value     solves/s of the mixed-precision solve (FP32 LMA apply and FP32
            Krylov vectors inside FP64 iterative refinement; residual,
            correction update and convergence test in FP64), inputs resident
  fp64      the same solve in plain FP64 (bit-identical to the CPU oracle)
  e2e       the mixed-precision solve through the C ABI with the right-hand
            side copied in from pinned host memory and the solution copied
            out every step
  roofline  the FP32 LMA apply (dominant kernel) against the measured HBM peak,
            its time from CUDA events around every apply of a second timed
            pass of the same solves (the events slow a solve, so the
            headline pass runs without them)
  cpu_baseline  the oracle (CPU restatement of the reference) on this host
  workloads the other configurations: plain FP64 CG on C24x20 W0 against the
            oracle; 64 right-hand sides of C48x30 W0 with tensor-core (TF32 /
            BF16) applies in FP64 refinement; 256 batched uneven W0 solves;
            a Poisson stream of W2 requests served by continuous batching

--impl reference times the oracle port on the host cores instead (the
reference itself is Fortran + PSyclone and cannot be built here).
Multi-GPU runs are replicas: every rank solves its own copy of the system.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "solves/sec and p50/p99 latency at 1e-8 rel. residual vs plain FP64, 1 B200"
N_EDGE, NLAYERS, GCRK, RTOL, SEED = 96, 30, 10, 1e-8, 2
WORKLOAD = ("C96x30 W2-W3 Helmholtz A=M2+0.1*D^T*D, GMRES(10) + column-tridiagonal(W2V)"
            " / Jacobi(W2H) preconditioner, solve to 1e-8 rel. residual")
INNER_RTOL = 1e-4
# a solution at 1e-8 relative residual lies within cond(A) * 2e-8 of another;
# cond(A) of the C96x30 Helmholtz system is below 50 (mass-dominated, tau 0.1)
E2E_TOL = 1e-6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=3, help="oracle solves timed on the host")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--quick", action="store_true", help="skip the batched and serving legs")
    ap.add_argument("--apply", default="",
                    help="pin the LMA apply configuration kernel:stages[:warps] for FP32,FP64, e.g. 5:0,5:0 "
                         "(default: the autotuner's choice; a profiler's replays can move that "
                         "choice, so profiled runs pin the one an unprofiled run tunes to)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock / throttle samples while a timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self._first = threading.Event()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            # nvidia-smi takes a moment to start sampling: the timed region
            # begins once the first sample is in (or after 5 s without one)
            self._first.wait(timeout=5.0)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())
            self._first.set()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self._t.join(timeout=2)

    def summary(self):
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


def measured_hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per FP32 apply (all its launches) from the committed ncu
    summary, if any."""
    p = ROOT / "profiles" / "lma_apply_fp32_c96x30.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get("dram_bytes_per_launch")
        except ValueError:
            return None
    return None


def solve_bytes(n, ncell_2d, nrow, a32, a64, gcrk, steps, inner_iters, fp64_cycles):
    """Algorithmic HBM bytes of the operations one headline solve executes.

    a32 / a64: bytes of one FP32 / FP64 apply as the tuned kernel reads them
    (local matrices + x + y + map rows); a residual-form apply also reads b.
    The column preconditioner reads its factors (3 per row) and the diagonal
    and x, and writes y. Each vector pass counts every vector it reads or
    writes once. Mixed: `steps` refinement steps of one FP32 GMRES cycle each
    (`inner_iters` iterations in all, split evenly), classical Gram-Schmidt
    (iteration j: dots over j basis vectors + w, update reading j + 1 and
    writing 1), no closing residual; FP64 residual, norm and solution update
    per step. `inner_iters` counts the iterations that did work (a cycle that
    reaches its tolerance early skips the rest); they are split over the
    cycles as evenly as they go. FP64: `fp64_cycles` full GMRES(gcrk) cycles
    with the reference's modified Gram-Schmidt (a pass per basis vector) and
    a residual per cycle."""
    v4, v8 = 4 * n, 8 * n
    p32 = 3 * v4 + 3 * nrow * ncell_2d * 4
    p64 = 3 * v8 + 3 * nrow * ncell_2d * 8
    a64r = a64 + v8
    initial = 4 * v8  # zero check of x, b copied to r, ||r||
    steps = max(int(steps), 1)
    inner_iters = int(inner_iters)
    mixed = initial
    for k in range(steps):
        m = inner_iters // steps + (1 if k < inner_iters % steps else 0)
        per_iter = sum(a32 + p32 + (j + 1) * v4 + (j + 2) * v4 for j in range(1, m + 1))
        mixed += ((v8 + 2 * v4) + 2 * v4 + (p32 + v4) + per_iter + (m + 2) * v4
                  + (2 * v8 + v4) + a64r + v8)
    k = gcrk
    mgs = sum(2 * v8 + (j - 1) * 4 * v8 + 3 * v8 + (2 * v8 if j < k else 0) for j in range(1, k + 1))
    cycle = (p64 + v8 + 2 * v8) + k * (a64 + p64) + mgs + (k + 2) * v8 + a64r + v8
    fp64 = initial + fp64_cycles * cycle
    return int(mixed), int(fp64)


def leg_batched(ctx, lfx, mg, wl, torch, stream):
    """256 independent W0 solves of uneven size (C12-C48 x 10-70 levels,
    tolerances 1e-10..1e-6) in one batch (FP32 PCG with FP64 reliable
    updates, one CUDA graph per 8 super-iterations), against the same solves
    run one after another with the plain FP64 device-resident CG."""
    specs = wl.config3_specs()
    t0 = time.perf_counter()
    systems = [wl.batch_system(ctx, n, l, sd, mg.W0) for n, l, _, sd in specs]
    setup_s = time.perf_counter() - t0
    tot = sum(s.undf for s in systems)
    B = lfx.Batch(ctx, 8, len(systems), reserve_bytes=2 << 30, iters=16)
    xs = [lfx.FieldVector(ctx, [s.undf]) for s in systems]

    def batched(tune=False):
        slots = []
        for s, x, (_, _, tol, _) in zip(systems, xs, specs):
            x.set_scalar(0.0)
            slots.append(B.admit(s.ops[lfx.R64], s.ops[lfx.R32], s.prec32, s.b, x, tol, 20000))
        if tune:
            B.autotune(iters=4)
        steps = 0
        while B.step() < len(systems):
            steps += 1
        infos = [B.slot(sl)[2].as_dict() for sl in slots]
        for sl in slots:
            B.retire(sl)
        return infos, steps

    batched(tune=True)  # warm-up with the launch-shape autotuner (pages the pool in)
    r0 = B.tuning()["replays"]
    ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    ctx.synchronize()
    ev[0].record(stream)
    w0 = time.perf_counter()
    infos, steps = batched()
    ev[1].record(stream)
    ctx.synchronize()
    t_batch = ev[0].elapsed_time(ev[1]) / 1e3
    wall_batch = time.perf_counter() - w0
    ok = all(i["status"] == 0 and i["final_rel"] <= tol * 1.0001
             for i, (_, _, tol, _) in zip(infos, specs))
    x_batch = [x.export_field() for x in xs]
    # plain FP64 serial solves of the same systems (graphs warmed first)
    cgs = [s.cg64(tol) for s, (_, _, tol, _) in zip(systems, specs)]
    for c, s, x in zip(cgs, systems, xs):
        x.set_scalar(0.0)
        c.apply(x, s.b)
    ctx.synchronize()
    ev[0].record(stream)
    it64 = []
    for c, s, x in zip(cgs, systems, xs):
        x.set_scalar(0.0)
        it64.append(c.apply(x, s.b).iterations)
    ev[1].record(stream)
    ctx.synchronize()
    t_serial = ev[0].elapsed_time(ev[1]) / 1e3
    cells = sum(6 * n * n * l for n, l, _, _ in specs)
    tune = B.tuning()
    err = []
    for xb, x in zip(x_batch, xs):
        x64 = x.export_field()
        err.append(float(np.linalg.norm(xb - x64) / np.linalg.norm(x64)))
    # two systems against the oracle's own FP64 CG on the host (the smallest
    # and a mid-size one; the parity tests pin the device CG to it bit for bit)
    from oracle import oracle as orc
    sample = {}
    for i in sorted(range(len(specs)), key=lambda i: 6 * specs[i][0] ** 2 * specs[i][1])[:2]:
        n, l, tol, sd = specs[i]
        p = mg.w0_problem(n, l, seed=sd)
        npc, cic = p.mesh.colour_lookup()
        o = orc.LmaOperator(p.ncell_2d, l, 8, 8, p.map, p.map, p.undf, p.undf, p.lma, npc, cic)
        xo, _ = orc.solve("cg", o, orc.Preconditioner.diagonal(o.diagonal()),
                          systems[i].b.export_field(), r_tol=tol, a_tol=0.0, max_iter=20000)
        sample[f"C{n}x{l}"] = float(np.linalg.norm(x_batch[i] - xo) / np.linalg.norm(xo))
    return {
        "workload": "256 uneven W0 mass+diffusion solves, C12-C48 x 10-70 levels, tol 1e-10..1e-6 "
                    "(seeded), FP32 PCG + FP64 reliable updates, one batch",
        "cells_total": cells, "dofs_total": tot,
        "batched_solves_per_s": round(len(specs) / t_batch, 2),
        "batched_s": round(t_batch, 4), "batched_wall_s": round(wall_batch, 4),
        "graph_replays": tune["replays"] - r0, "kernel_launches_per_replay": 1,
        "launch_shape": {k: tune[k] for k in ("cells_per_item", "blocks_per_sm", "grid",
                                              "group_bytes", "cooperative")},
        "tuned_us_per_iteration": round(tune["us_per_iteration"], 2),
        "iterations_max": max(i["iterations"] for i in infos),
        "all_converged_on_fp64_residual": ok,
        "error_vs_fp64_max": max(err), "error_vs_fp64_median": float(np.median(err)),
        "error_reference": "each system's serial FP64 device CG solution at the same tolerance "
                           "(that solve equals the oracle's bit for bit in the parity tests)",
        "error_vs_fp64_oracle_sample": sample,
        "serial_fp64_solves_per_s": round(len(specs) / t_serial, 2), "serial_fp64_s": round(t_serial, 4),
        "serial_fp64_iterations_max": max(it64),
        "speedup_vs_serial_fp64": round(t_serial / t_batch, 3), "setup_s": round(setup_s, 1),
    }


def leg_plain_cg(ctx, lfx, mg, wl, torch, stream, nsolves=50, ncpu=5):
    """Plain FP64 Jacobi CG on the C24x20 W0 mass+diffusion system
    (b ~ U[-1,1], x0 = 0, r_tol 1e-8, a_tol 1e-16): device-resident solves
    against the oracle's CG on the host cores, and the solution compared bit
    for bit with the oracle's."""
    from oracle import oracle as orc
    p = mg.w0_problem(24, 20, seed=1)
    s = wl.device_w0(ctx, p)
    cg = lfx.ConjugateGradient(s.op, s.prec, RTOL, 1e-16, 1000)
    B = lfx.FieldVector.from_array(ctx, p.rhs)
    X = lfx.FieldVector(ctx, [p.undf])
    for _ in range(3):
        X.set_scalar(0.0)
        cg.apply(X, B)
    ctx.synchronize()
    ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    ev[0].record(stream)
    for _ in range(nsolves):
        X.set_scalar(0.0)
        info = cg.apply(X, B)
    ev[1].record(stream)
    ctx.synchronize()
    t = ev[0].elapsed_time(ev[1]) / 1e3
    x_gpu = X.export_field()
    npc, cic = p.mesh.colour_lookup()
    o = orc.LmaOperator(p.ncell_2d, p.nlayers, 8, 8, p.map, p.map, p.undf, p.undf, p.lma, npc, cic)
    od = orc.Preconditioner.diagonal(o.diagonal())
    times = []
    for _ in range(ncpu):
        t0 = time.perf_counter()
        x_cpu, oi = orc.solve("cg", o, od, p.rhs, r_tol=RTOL, a_tol=1e-16, max_iter=1000)
        times.append(time.perf_counter() - t0)
    return {"workload": "C24x20 W0 mass+diffusion, Jacobi CG, FP64, b ~ U[-1,1], 1e-8",
            "undf": p.undf, "iterations": info.iterations, "oracle_iterations": oi.iterations,
            "gpu_solves_per_s": round(nsolves / t, 2), "gpu_ms_per_solve": round(1e3 * t / nsolves, 4),
            "cpu_oracle_solves_per_s": round(ncpu / sum(times), 2), "cpu_threads": os.cpu_count(),
            "solution_bitwise_equal_to_oracle": bool(np.array_equal(x_gpu.view(np.int64),
                                                                     x_cpu.view(np.int64)))}


def leg_multi_rhs(ctx, lfx, mg, wl, torch, stream, n=48, nl=30, nrhs=64):
    """64 seeded N(0,1) right-hand sides of the C48x30 W0 mass+diffusion
    operator solved together: FP64 refinement around an FP32 Jacobi CG whose
    per-cell products run as (64 x 8).(8 x 8) tensor-core GEMMs in TF32 and in
    BF16, against 64 serial plain FP64 device CG solves; per-RHS error of the
    solution against the FP64 solve."""
    p = mg.w0_problem(n, nl, seed=1, rhs="normal")
    s = wl.device_w0(ctx, p)
    Bh = np.stack([mg.normal(1000 + r, p.undf) for r in range(nrhs)])
    b = torch.from_numpy(Bh).cuda()
    x = torch.zeros_like(b)
    torch.cuda.synchronize()
    ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    # plain FP64: one device-resident CG per right-hand side
    cg = lfx.ConjugateGradient(s.op, s.prec, RTOL, 0.0, 20000)
    X = lfx.FieldVector(ctx, [p.undf])
    Bv = [lfx.FieldVector.from_array(ctx, Bh[r]) for r in range(nrhs)]
    X.set_scalar(0.0)
    cg.apply(X, Bv[0])  # warm-up
    ctx.synchronize()
    x64, it64 = [], []
    ev[0].record(stream)
    for r in range(nrhs):
        X.set_scalar(0.0)
        it64.append(cg.apply(X, Bv[r]).iterations)
        x64.append(X.export_field())
    ev[1].record(stream)
    ctx.synchronize()
    t64 = ev[0].elapsed_time(ev[1]) / 1e3
    out = {"workload": f"C{n}x{nl} W0 mass+diffusion, {nrhs} N(0,1) right-hand sides, 1e-8 rel. "
                       "residual, Jacobi; FP32 CG with tensor-core apply inside FP64 refinement",
           "undf": p.undf, "ncell_3d": p.mesh.ncell_3d,
           "serial_fp64_solves_per_s": round(nrhs / t64, 2), "serial_fp64_s": round(t64, 4),
           "serial_fp64_iterations_max": max(it64)}
    peak, _ = measured_hbm_peak()
    xr = torch.randn(p.undf, nrhs, device="cuda", dtype=torch.float32)
    yr = torch.empty_like(xr)
    from oracle import oracle as orc
    npc, cic = p.mesh.colour_lookup()
    o = orc.LmaOperator(p.ncell_2d, nl, 8, 8, p.map, p.map, p.undf, p.undf, p.lma, npc, cic)
    x_or, _ = orc.solve("cg", o, orc.Preconditioner.diagonal(o.diagonal()), Bh[0], r_tol=RTOL,
                        a_tol=0.0, max_iter=20000)
    runs = [(lfx.MRHS_TF32, "tf32", lfx.MRHS_PER_RHS_CG, False),
            (lfx.MRHS_BF16, "bf16", lfx.MRHS_PER_RHS_CG, False),
            (lfx.MRHS_TF32, "tf32_block_cg", lfx.MRHS_BLOCK_CG, False),
            (lfx.MRHS_BF16, "bf16_block_cg", lfx.MRHS_BLOCK_CG, False),
            (lfx.MRHS_BF16, "bf16_block_cg_tcgen05_gram", lfx.MRHS_BLOCK_CG, True)]
    for kind, name, method, tc_gram in runs:
        M = lfx.MultiRhsOperator(s.op, kind, nrhs)
        M.set_gram(tc_gram)
        inf = M.info()
        tune = M.autotune(10)
        torch.cuda.synchronize()
        us = M.time_apply(xr.data_ptr(), yr.data_ptr(), 20)
        algo = inf["matrix_bytes"] + 2 * p.undf * nrhs * 4
        x.zero_()
        torch.cuda.synchronize()
        M.solve(s.op, s.diag, b.data_ptr(), x.data_ptr(), p.undf, r_tol=RTOL, method=method)  # warm-up
        x.zero_()
        torch.cuda.synchronize()
        l0 = ctx.launch_count()
        ev[0].record(stream)
        info = M.solve(s.op, s.diag, b.data_ptr(), x.data_ptr(), p.undf, r_tol=RTOL, method=method)
        ev[1].record(stream)
        ctx.synchronize()
        t = ev[0].elapsed_time(ev[1]) / 1e3
        X2 = x.cpu().numpy()
        err = [float(np.linalg.norm(X2[r] - x64[r]) / np.linalg.norm(x64[r])) for r in range(nrhs)]
        out[name] = {
            "method": ("block CG (one search space for the 64 right-hand sides)"
                       + (", Gram products on tcgen05 (3xTF32)" if tc_gram else ""))
                      if method == lfx.MRHS_BLOCK_CG else "CG per right-hand side",
            "error_vs_fp64_oracle_rhs0": float(np.linalg.norm(X2[0] - x_or) / np.linalg.norm(x_or)),
            "solves_per_s": round(nrhs / t, 2), "s": round(t, 4),
            "speedup_vs_serial_fp64": round(t64 / t, 3),
            "all_converged": all(i.converged for i in info),
            "final_rel_residual_max": max(i.final_rel for i in info),
            "outer_iterations_max": max(i.outer_iterations for i in info),
            "inner_iterations_max": max(i.inner_iterations for i in info),
            "error_vs_fp64_max": max(err), "error_vs_fp64_median": float(np.median(err)),
            "gpu_launches": ctx.launch_count() - l0,
            "apply_us": round(us, 2), "apply_algorithmic_bytes": algo,
            "apply_hbm_gbs": round(algo / (us * 1e-6) / 1e9, 1),
            "apply_hbm_frac": round(algo / (us * 1e-6) / 1e9 / peak, 4),
            "patches": inf["patches"], "levels_per_block": tune["levels_per_block"],
            "cell_levels_computed_per_cell": round(inf["cell_levels"] / p.mesh.ncell_3d, 3)}
        del M
    return out


def leg_serving(ctx, lfx, mg, wl, torch, nreq=200, npool=48):
    """Poisson stream (2000 requests/s, seeded) of W2 Helmholtz solves, each
    request with its own operator and right-hand side: the operators are 48
    distinct seeded geometries C12-C96 x 20-70 levels (assembled on the device
    before the stream starts, as the client model hands them over), the
    right-hand side of every request is its own N(0,1) vector in pinned host
    memory, copied to the device at admission, and the solution is copied
    back at completion; tolerances 1e-10..1e-6. Continuous batching: a request
    is admitted as soon as it has arrived, a slot is free and the device keeps
    its memory reserve; its Krylov state lives on the device until it is
    retired. Against serial plain FP64 device CG solves of the same request
    list (same copies)."""
    shapes, reqs = wl.config4_stream(nreq=nreq, pool=npool)
    t0 = time.perf_counter()
    systems = [wl.batch_system(ctx, n, l, 500 + i, mg.W2) for i, (n, l) in enumerate(shapes)]
    setup_s = time.perf_counter() - t0
    # every request's right-hand side, in pinned host memory (its own seed)
    tot = sum(systems[w].undf for _, w, _ in reqs)
    pin = torch.empty(2 * tot, dtype=torch.float64, pin_memory=True).numpy()
    off, bh, xh = 0, [], []
    for r, (_, w, _) in enumerate(reqs):
        n = systems[w].undf
        pin[off:off + n] = mg.normal(7000 + r, n)
        bh.append(pin[off:off + n])
        xh.append(pin[tot + off:tot + off + n])
        off += n
    free = {}  # device (b, x) pairs by operator, reused; a new pair when none is free

    def pair(w):
        lst = free.setdefault(w, [])
        if lst:
            return lst.pop()
        n = systems[w].undf
        return lfx.FieldVector(ctx, [n]), lfx.FieldVector(ctx, [n])

    # serial plain FP64: one device-resident CG per request (graphs warmed)
    cgs = {}
    for w, sy in enumerate(systems):
        cgs[w] = sy.cg64(1e-10)
        bv, xv = pair(w)
        xv.set_scalar(0.0)
        cgs[w].apply(xv, sy.b)
        free[w].append((bv, xv))
    service, x64 = [], []
    for r, (_, w, tol) in enumerate(reqs):
        bv, xv = pair(w)
        ctx.synchronize()
        t = time.perf_counter()
        bv.import_field_async(bh[r])
        xv.set_scalar(0.0)
        cgs[w].set_tolerance(tol)
        cgs[w].apply(xv, bv)
        xv.export_field(out=xh[r])
        service.append(time.perf_counter() - t)
        x64.append(xh[r].copy())
        free[w].append((bv, xv))
    fin, lat_serial = 0.0, []
    for (arr, _, _), sv in zip(reqs, service):
        fin = max(fin, arr) + sv
        lat_serial.append(fin - arr)
    serial_makespan = fin - reqs[0][0]

    B = lfx.Batch(ctx, 6, 64, reserve_bytes=4 << 30, iters=4)
    # launch shape for this request mix, chosen offline from measured serving
    # runs (eight cell columns an apply item, three blocks an SM: 1.25x the
    # serial solves against 0.92-0.99x with the W0 batch's shape); the
    # engine's autotuner times single replays on the slots it holds, which a
    # stream that admits and retires as it goes does not keep still
    B.set_tuning(8, 3, 1 << 40)
    launch_shape = B.tuning()

    def serve():
        pending, inflight, lat, lat_adm, done = list(range(nreq)), {}, [0.0] * nreq, [0.0] * nreq, 0
        occupancy, refused = [], 0
        ctx.synchronize()
        t0 = time.perf_counter()
        while done < nreq:
            now = time.perf_counter() - t0
            while pending and reqs[pending[0]][0] <= now:
                r = pending[0]
                _, w, tol = reqs[r]
                sy = systems[w]
                bv, xv = pair(w)
                bv.import_field_async(bh[r])
                xv.set_scalar(0.0)
                slot = B.admit(sy.ops[lfx.R64], sy.ops[lfx.R32], sy.prec32, bv, xv, tol, 20000, r)
                if slot is None:  # no slot or no memory: wait for a retirement
                    free[w].append((bv, xv))
                    refused += 1
                    break
                inflight[slot] = (r, w, bv, xv, time.perf_counter() - t0)
                pending.pop(0)
            if not inflight:
                if pending:
                    time.sleep(max(0.0, reqs[pending[0]][0] - (time.perf_counter() - t0)))
                continue
            occupancy.append(len(inflight))
            B.step()
            for slot in B.done_slots():
                r, w, bv, xv, t_adm = inflight.pop(slot)
                ph, tag, info = B.slot(slot)
                assert info.status == 0, info.as_dict()
                xv.export_field(out=xh[r])
                now = time.perf_counter() - t0
                lat[r] = now - reqs[r][0]
                lat_adm[r] = now - t_adm
                B.retire(slot)
                free[w].append((bv, xv))
                done += 1
        return time.perf_counter() - t0 - reqs[0][0], lat, lat_adm, occupancy, refused

    serve()  # warm-up: the device vectors of the busiest moment exist afterwards
    makespan, lat, lat_adm, occupancy, refused = serve()
    err = [float(np.linalg.norm(xh[r] - x64[r]) / np.linalg.norm(x64[r])) for r in range(nreq)]
    pct = lambda v, q: round(1e3 * float(np.percentile(v, q)), 3)
    return {
        "workload": f"{nreq} W2 Helmholtz requests, Poisson 2000/s, each with its own operator "
                    f"({npool} distinct seeded geometries C12-C96 x 20-70 levels) and right-hand "
                    "side (copied in at admission, solution copied out at completion), tol "
                    "1e-10..1e-6, continuous batching (FP32 PCG + FP64 reliable updates, column "
                    "preconditioner), admission by free device memory (4 GiB reserve)",
        "solves_per_s": round(nreq / makespan, 2),
        "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
        "admission_to_completion_p50_ms": pct(lat_adm, 50),
        "admission_to_completion_p99_ms": pct(lat_adm, 99),
        "mean_inflight": round(float(np.mean(occupancy)), 2) if occupancy else 0,
        "max_inflight": int(max(occupancy)) if occupancy else 0,
        "admissions_deferred": refused,
        "serial_fp64_solves_per_s": round(nreq / serial_makespan, 2),
        "serial_fp64_p50_ms": pct(lat_serial, 50), "serial_fp64_p99_ms": pct(lat_serial, 99),
        "serial_fp64_mean_service_ms": round(1e3 * float(np.mean(service)), 3),
        "speedup_vs_serial_fp64": round(serial_makespan / makespan, 3),
        "error_vs_fp64_max": max(err), "error_vs_fp64_median": float(np.median(err)),
        "error_reference": "each request's serial FP64 device CG solution (that solve equals "
                           "the oracle's bit for bit in the parity tests)",
        "launch_shape": launch_shape,
        "setup_s": round(setup_s, 1),
    }


def cpu_baseline(problem, nsolves):
    """The oracle (CPU FP64 restatement of the reference path) on all host
    threads: full GMRES solves of the same system."""
    from oracle import oracle as orc
    from lfric_core_b200 import meshgen as mg
    p = problem
    npc, cic = p.mesh.colour_lookup()
    op = orc.LmaOperator(p.ncell_2d, p.nlayers, 6, 6, p.map, p.map, p.undf, p.undf, p.lma, npc, cic)
    prm = mg.w2v_cma_params(p.nlayers)
    band = orc.assemble_cma(mg.lma_block(p.lma, p.mesh.ncell_3d, 6, mg.W2V_DFS), p.ncell_2d,
                            p.nlayers, prm)
    P = orc.Preconditioner.cma(p.ncell_2d, prm["nrow"], 3, p.map[:, 4], prm["indirection"], band,
                               op.diagonal(), p.undf)
    times, info, x_oracle = [], None, None
    for _ in range(nsolves):
        t0 = time.perf_counter()
        x_oracle, info = orc.solve("gmres", op, P, p.rhs, r_tol=RTOL, max_iter=200, gcrk=GCRK)
        times.append(time.perf_counter() - t0)
    cores = os.cpu_count()
    # and one solve on a single thread
    orc.lib().or_set_threads(1)
    t0 = time.perf_counter()
    orc.solve("gmres", op, P, p.rhs, r_tol=RTOL, max_iter=200, gcrk=GCRK)
    t1 = time.perf_counter() - t0
    orc.lib().or_set_threads(cores)
    return {"value": nsolves / sum(times), "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": f"{nsolves} full FP64 GMRES(10) solves of the same C96x30 system "
                      f"({info.iterations} cycles each), OpenMP on {cores} threads; one more "
                      "on 1 thread",
            "p50_ms": 1e3 * statistics.median(times),
            "one_thread": {"value": 1.0 / t1, "unit": "solves/s", "cores": 1},
            "cpu_model": cpu_model(), "_x": x_oracle}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def max_over_ranks(v, dist=None, device="cuda"):
    """The largest v over the ranks of the process group (v itself when there
    is no group): timings are the slowest rank's."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, steps, ms):
    """Whole-job solves/s of `world` replicas that each ran `steps` solves in
    `ms` milliseconds (the slowest rank's time)."""
    return world * steps / (ms / 1e3)


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from lfric_core_b200 import meshgen as mg
    p = mg.w2_problem(N_EDGE, NLAYERS, seed=SEED)
    steps, warm = max(args.steps, 1), max(args.warmup, 0)
    # each step is one full oracle solve; bounded so the whole run stays short
    steps = min(steps, 20)
    cb = cpu_baseline(p, warm) if warm else None
    cb = cpu_baseline(p, steps)
    cb.pop("_x", None)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "solves/s",
            "n_gpus": args.gpus, "steps": steps, "warmup": warm,
            "ms_per_step": 1e3 / cb["value"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "implementation": "CPU restatement of the reference "
                       "(Fortran reference not buildable here: no Fortran compiler / PSyclone)"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank, world, local = dist_env()
    import torch
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA GPU")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    from lfric_core_b200 import lfx, meshgen as mg, workloads as wl

    p = mg.w2_problem(N_EDGE, NLAYERS, seed=SEED)
    ctx = lfx.Context(local)
    s64 = wl.device_w2(ctx, p, lfx.R64)
    s32 = wl.device_w2(ctx, p, lfx.R32, op64=s64.op64, cma=s64.cma, diag64=s64.diag)
    # apply autotuner (set-up, untimed): fastest launch configuration per operator
    if args.apply:
        tuning = {}
        for name, sys_, spec in zip(("fp32", "fp64"), (s32, s64), args.apply.split(",")):
            k, st, w = ([int(v) for v in spec.split(":")] + [0])[:3]
            sys_.op.set_apply(k, st, w)
            tuning[name] = {"kernel": lfx.APPLY_KERNEL_NAMES[k], "stages": st, "warps": w,
                            "us": round(sys_.op.time_apply(k, st, w, 10), 2), "pinned": True}
    else:
        tuning = {"fp32": s32.op.autotune(reps=10), "fp64": s64.op.autotune(reps=10)}
    fp64 = lfx.GMRES(s64.op, s64.prec, GCRK, RTOL, 1e-16, 200)
    mixed = wl.refined_gmres(s32, gcrk=GCRK, inner_rtol=INNER_RTOL, r_tol=RTOL)
    B = lfx.FieldVector.from_array(ctx, p.rhs)
    X = lfx.FieldVector(ctx, [p.undf])
    R = lfx.FieldVector(ctx, [p.undf])
    stream = torch.cuda.ExternalStream(ctx.stream)
    bnorm = B.norm()

    def true_rel():
        s64.op.apply(X, R)
        R.aypx(-1.0, B)
        return R.norm() / bnorm

    def barrier():
        if dist:
            dist.barrier()

    def timed_e2e(solver, steps, host):
        """Solves through the C ABI from pinned host memory, every step with
        its own host->device copy of b and device->host copy of x, queued on
        a copy stream and double-buffered so that step k+1's b arrives and
        step k-1's x leaves while step k solves."""
        cs = torch.cuda.Stream()
        Xs = [X, lfx.FieldVector(ctx, [p.undf])]
        Bs = [B, lfx.FieldVector(ctx, [p.undf])]
        outs = [host["x"], host["x2"]]
        for i in range(2):  # both buffer pairs warmed (untimed)
            Bs[i].import_field(host["rhs"])
            Xs[i].set_scalar(0.0)
            solver.apply(Xs[i], Bs[i])
        ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
        ev_in, ev_done, ev_out = [ev(), ev()], [ev(), ev()], [ev(), ev()]
        st, en = [ev() for _ in range(steps)], [ev() for _ in range(steps)]
        t0, t1 = ev(), ev()
        infos = []
        barrier()
        torch.cuda.synchronize()
        ctx.synchronize()
        t0.record(cs)
        st[0].record(cs)
        Bs[0].import_field_async(host["rhs"], cs.cuda_stream)
        ev_in[0].record(cs)
        for k in range(steps):
            i, j = k % 2, 1 - k % 2
            if k + 1 < steps:
                if k >= 1:
                    cs.wait_event(ev_done[j])        # solve k-1 has finished with B[j]
                st[k + 1].record(cs)
                Bs[j].import_field_async(host["rhs"], cs.cuda_stream)   # pinned host -> device
                ev_in[j].record(cs)
            stream.wait_event(ev_in[i])
            if k >= 2:
                stream.wait_event(ev_out[i])         # step k-2's x has left X[i]
            Xs[i].set_scalar(0.0)
            infos.append(solver.apply(Xs[i], Bs[i]).as_dict())
            ev_done[i].record(stream)
            cs.wait_event(ev_done[i])
            Xs[i].export_field_async(outs[i], cs.cuda_stream)           # device -> pinned host
            ev_out[i].record(cs)
            en[k].record(cs)
        cs.wait_stream(stream)
        t1.record(cs)
        torch.cuda.synchronize()
        ctx.synchronize()
        barrier()
        return {"ms": t0.elapsed_time(t1), "lat": [a.elapsed_time(b) for a, b in zip(st, en)],
                "infos": infos}

    def timed(solver, steps):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        t_all = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        infos = []
        barrier()
        torch.cuda.synchronize()
        ctx.synchronize()
        l0 = ctx.launch_count()
        w0 = time.perf_counter()
        t_all[0].record(stream)
        for k in range(steps):
            ev[k][0].record(stream)
            X.set_scalar(0.0)
            infos.append(solver.apply(X, B).as_dict())
            ev[k][1].record(stream)
        t_all[1].record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        wall = time.perf_counter() - w0
        barrier()
        lat = [a.elapsed_time(b) for a, b in ev]
        return {"ms": t_all[0].elapsed_time(t_all[1]), "wall_ms": 1e3 * wall, "lat": lat,
                "infos": infos, "launches": ctx.launch_count() - l0}

    # warm-up (also checks both paths reach the tolerance)
    for _ in range(max(args.warmup, 3)):
        X.set_scalar(0.0)
        i64 = fp64.apply(X, B)
        X.set_scalar(0.0)
        imx = mixed.apply(X, B)
    assert i64.converged and imx.converged, (i64.as_dict(), imx.as_dict())

    K = args.steps
    # mixed precision: the headline, uninstrumented
    # (an NVTX range "timed" lets a profiler keep to these solves:
    # ncu --nvtx --nvtx-include "timed/")
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("timed")
        mx = timed(mixed, K)
        torch.cuda.nvtx.range_pop()
    rel_mixed = true_rel()
    # the same K solves again with CUDA events around every apply inside the
    # solver graphs (the roofline's kernel times; the event nodes themselves
    # slow the solve, so this pass is reported beside the headline, not as it)
    ctx.enable_apply_timing(True)
    ctx.apply_timing(0, reset=True)
    mx_ev = timed(mixed, K)
    n32, ms32 = ctx.apply_timing(32, reset=False)
    n64m, ms64m = ctx.apply_timing(64, reset=True)
    ctx.enable_apply_timing(False)
    # plain FP64 solve
    f = timed(fp64, K)
    rel_fp64 = true_rel()
    # end to end through the C ABI with pinned host buffers
    pin = torch.empty(3 * p.undf, dtype=torch.float64, pin_memory=True).numpy()
    host = {"rhs": pin[:p.undf], "x": pin[p.undf:2 * p.undf], "x2": pin[2 * p.undf:]}
    host["rhs"][:] = p.rhs
    e = timed_e2e(mixed, K, host)

    t_mx = max_over_ranks(mx["ms"], dist)
    t_64 = max_over_ranks(f["ms"], dist)
    t_e2e = max_over_ranks(e["ms"], dist)
    value = replica_throughput(world, K, t_mx)
    fp64_value = replica_throughput(world, K, t_64)
    e2e_value = replica_throughput(world, K, t_e2e)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    # roofline of the FP32 LMA apply (dominant kernel of the mixed solve).
    # Algorithmic bytes: the local matrices as the tuned kernel reads them
    # (the packed upper triangle for the cell scatter of this symmetric
    # operator), x read once, y written once, the map rows. The time is the
    # event-timed pass's total over its FP32 applies (events around each apply
    # in the solver graphs) per apply that did work.
    nc3 = p.mesh.ncell_3d

    def apply_bytes(op, esz, kernel):
        st = op.storage()
        mat = (st["packed_bytes"] if kernel.startswith("cell-scatter") and st["packed_bytes"]
               else st["full_bytes"])
        return mat + 2 * p.undf * esz + p.ncell_2d * 6 * 4
    bytes32 = apply_bytes(s32.op, 4, tuning["fp32"]["kernel"])
    # FP32 applies that did work: the refined solve counts its initial
    # residual (idle at x = 0), each inner iteration and one FP64 residual per
    # step; a cycle that reaches its tolerance early leaves its remaining
    # launches idle (they read a device flag and return). The idle applies'
    # short event times stay in the total, so this average errs high.
    inf_last = mx["infos"][-1]
    exec32 = max(inf_last["applies"] - 1 - inf_last["outer_iterations"], 1)
    avg32 = ms32 / max(K * exec32, 1)
    achieved = bytes32 / (avg32 / 1e3) / 1e9
    peak, peak_kind = measured_hbm_peak()
    traffic = profiled_traffic()
    roof = {"kernel": f"{tuning['fp32']['kernel']} (FP32 LMA apply)", "bound": "hbm",
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
            "traffic": traffic,
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one apply, from "
                               "the committed capture profiles/lma_apply_fp32_c96x30.json (not "
                               "measured in this run)") if traffic else None,
            "algorithmic_bytes_per_launch": bytes32,
            "launch": {"cell-scatter": "one apply (the cell scatter: one kernel per colour)",
                       "cell-scatter-persistent": "one apply (the cell scatter: one persistent "
                                                  "launch over the colours)"}.get(
                           tuning["fp32"]["kernel"], "one apply (one launch)"),
            "launches_timed": n32, "applies_executed": K * exec32,
            "avg_launch_us": round(1e3 * avg32, 2),
            "timed_pass": "a second pass of the same solves with events around each apply "
                          f"({round(mx_ev['ms'] / K, 4)} ms per solve instrumented, "
                          f"{round(mx['ms'] / K, 4)} uninstrumented)",
            "standalone_us": tuning["fp32"]["us"],
            "standalone_frac": round(bytes32 / (tuning["fp32"]["us"] / 1e6) / 1e9 / peak, 4)}
    # the whole solves against the same peak: algorithmic bytes of every
    # operation they execute over their measured time per solve
    steps_mx = mx["infos"][-1]["outer_iterations"]
    sb_mixed, sb_fp64 = solve_bytes(
        p.undf, p.ncell_2d, p.nlayers + 1, bytes32, apply_bytes(s64.op, 8, tuning["fp64"]["kernel"]),
        GCRK, steps_mx, exec32, f["infos"][-1]["iterations"])
    solve_roof = {"unit": "GB/s", "peak": peak,
                  "mixed": {"bytes": sb_mixed, "achieved": round(sb_mixed / (t_mx / K / 1e3) / 1e9, 1),
                            "frac": round(sb_mixed / (t_mx / K / 1e3) / 1e9 / peak, 4),
                            "refinement_steps": steps_mx,
                            "inner_iterations": exec32},
                  "fp64": {"bytes": sb_fp64, "achieved": round(sb_fp64 / (t_64 / K / 1e3) / 1e9, 1),
                           "frac": round(sb_fp64 / (t_64 / K / 1e3) / 1e9 / peak, 4),
                           "cycles": f["infos"][-1]["iterations"]}}
    if n64m:
        bytes64 = apply_bytes(s64.op, 8, tuning["fp64"]["kernel"])
        avg64 = ms64m / n64m
        roof["fp64_apply"] = {"achieved": round(bytes64 / (avg64 / 1e3) / 1e9, 1),
                              "avg_launch_us": round(1e3 * avg64, 2), "launches_timed": n64m,
                              "algorithmic_bytes": bytes64}

    cb, x_oracle = None, None
    if world == 1 and not args.no_cpu:
        cb = cpu_baseline(p, args.cpu_sample)
        x_oracle = cb.pop("_x")
    # the headline's solutions against the oracle's FP64 GMRES solution of the
    # same system (the mixed one within its 1e-8 residual; the plain FP64 one
    # bit for bit)
    oracle_check = None
    if x_oracle is not None:
        X.set_scalar(0.0)
        mixed.apply(X, B)
        xm = X.export_field()
        X.set_scalar(0.0)
        fp64.apply(X, B)
        xf = X.export_field()
        on = np.linalg.norm(x_oracle)
        oracle_check = {
            "mixed_error_vs_fp64_oracle": float(np.linalg.norm(xm - x_oracle) / on),
            "fp64_bitwise_equal_to_oracle": bool(np.array_equal(xf.view(np.int64),
                                                                x_oracle.view(np.int64))),
            "e2e_error_vs_fp64_oracle": float(np.linalg.norm(host["x"] - x_oracle) / on),
            "e2e_tolerance": E2E_TOL}
    extra = {}
    if not args.quick:
        extra["plain_cg_w0"] = leg_plain_cg(ctx, lfx, mg, wl, torch, stream)
        extra["multi_rhs_w0"] = leg_multi_rhs(ctx, lfx, mg, wl, torch, stream)
        extra["batched_uneven_w0"] = leg_batched(ctx, lfx, mg, wl, torch, stream)
        extra["serving_w2"] = leg_serving(ctx, lfx, mg, wl, torch)

    def pct(v, q):
        return float(np.percentile(np.array(v), q))

    inf_mx = mx["infos"][-1]
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "solves/s", "n_gpus": world,
        "steps": K, "warmup": args.warmup, "ms_per_step": round(t_mx / K, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 apply + f64 refinement", "data": "synthetic (seeded perturbed geometry, b~N(0,1))",
        "config": {"workload": WORKLOAD, "ncell_3d": nc3, "undf_w2": p.undf,
                   "precision": "FP32 LMA/CMA apply and Krylov vectors, FP64 dots, residual, "
                                "refinement and column factorisation",
                   "inner": f"GMRES({GCRK}) FP32 to {INNER_RTOL:g}",
                   "l2": "inputs larger than L2 (FP32 LMA 239 MB, FP64 LMA 478 MB)",
                   "parallelism": f"replicas x{world}", "apply_tuning": tuning},
        "latency_ms": {"p50": round(pct(mx["lat"], 50), 4), "p99": round(pct(mx["lat"], 99), 4)},
        "final_rel_residual": rel_mixed,
        "mixed": {"outer_iterations": inf_mx["outer_iterations"],
                  "inner_cycles": inf_mx["inner_iterations"], "applies": inf_mx["applies"]},
        "fp64": {"solves_per_s": round(fp64_value, 3), "p50_ms": round(pct(f["lat"], 50), 4),
                 "p99_ms": round(pct(f["lat"], 99), 4), "cycles": f["infos"][-1]["iterations"],
                 "final_rel_residual": rel_fp64},
        "speedup_vs_fp64": round(value / fp64_value, 3),
        "roofline": roof,
        "solve_roofline": solve_roof,
        "cpu_baseline": cb,
        "e2e": {"value": round(e2e_value, 3), "unit": "solves/s",
                "h2d_bytes_per_step": p.undf * 8, "d2h_bytes_per_step": p.undf * 8,
                "p50_ms": round(pct(e["lat"], 50), 4),
                "copies": "async on a copy stream, double-buffered (overlap the neighbouring solves)",
                "solution_checked": (None if oracle_check is None else
                                     oracle_check["e2e_error_vs_fp64_oracle"] <= E2E_TOL),
                "solution_reference": "the oracle's FP64 GMRES solution of the same system"},
        "error_vs_fp64_oracle": oracle_check,
        "gpu_launches": mx["launches"],
        "clocks": clk.summary(),
        "workloads": extra,
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
