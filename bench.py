#!/usr/bin/env python
"""MLFMA matvec throughput on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload: the PEC sphere of radius 2 wavelengths meshed as a level-5
subdivided icosahedron (20,480 triangles, 30,720 RWG unknowns), 7-point
triangle quadrature, root box 4 wavelengths, boxes split while they hold more
than 54 RWGs (every 0.25-wavelength box is a leaf), 3-digit angular sampling,
6-point interpolation, plain complex FP64.  One step is one MLFMA
matrix-vector product y = A x on one right-hand side.

`value` is device-resident throughput (x and y already in HBM), timed with
CUDA events on the launching stream; `e2e` is the same product through the
C-ABI host-buffer call mlfma_matvec_mapped (called through ctypes, pointers
prepared once) on pinned host buffers: its first kernel reads x and its last
kernel writes y across the bus inside the timed region, and the call
synchronises before it returns.  `e2e.copy_path` times mlfma_matvec on the
same buffers (cudaMemcpyAsync in, product, cudaMemcpyAsync out).  The operator
reads 0.41 GB per matvec, more than the 126 MB L2, so no flush runs between
steps.  With N > 1 every rank runs an independent replica of the product
(there is no data exchange on this path); rank 0 reports N * K / max time,
and the secondary blocks (many right-hand sides, many problems, adjoint,
8-wavelength sphere) run only when N = 1.

`dense_check` (and `dense_rel_err` / `dense_residual` in the mixed and solve
blocks) states the relative error of the product, and the residual of each
solution, on 64 seeded rows against the dense FP64 operator (every
interaction evaluated directly on the GPU, mlfma_dense_rows).

`--impl reference` times the reference's own CPU code (oracle/_ref, built from
its sources, single-threaded by construction) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

METRIC = "MLFMA matvecs/s, GMRES solve s @1e-4 resid: mixed/batched vs FP64 on 1 B200"
UNIT = "matvecs/s"
WORKLOAD = dict(name="rwg_sphere_r2lambda_ico5", kind="rwg", level=5, radius=2.0, root_leng=4.0,
                max_node_srcs=54, quad_prec=2, digits=3, interp_order=3, over_interp=2.0)
HERE = os.path.dirname(os.path.abspath(__file__))
SOLVE = dict(restart=50, tol=1e-4, max_iter=3000)
# The large benchmark: PEC sphere of radius 8 wavelengths, level-7 icosphere
# (327,680 triangles, 491,520 RWGs), root box 16, leaves 0.25 wavelength.
LARGE = dict(name="rwg_sphere_r8lambda_ico7", level=7, radius=8.0, root_leng=16.0, max_node_srcs=54, quad_prec=2,
             digits=3, interp_order=3, over_interp=2.0)
LARGE_SOLVE = dict(restart=50, tol=1e-4, max_iter=6000)
LARGE_FLEX = dict(restart=30, inner_iters=50)  # flexible GMRES: outer steps per cycle, inner iterations
LARGE_NRHS = 16
LARGE_FLEX_NRHS = 64  # plane waves of the batched flexible solve (the many-rhs kernels' tile width)
LARGE_INNER_DIGITS = 2  # angular sampling digits of the flexible solve's inner operator
NRHS = 64
NPROB = 32
DENSE_ROWS = 64


def make_problem():
    sys.path.insert(0, HERE)
    from mlfma_b200 import inputs
    mesh = inputs.make_icosphere(WORKLOAD["level"], radius=WORKLOAD["radius"])
    pw = inputs.PlaneWave(amplitude=1.0, pol=(1.0, 0.0, 0.0), khat=(0.0, 0.0, -1.0), wavenum=2.0 * np.pi)
    return mesh, pw


def config_dict(extra=None):
    c = {"workload": WORKLOAD["name"], "unknowns": 30720, "triangles": 20480,
         "radius_lambda": WORKLOAD["radius"], "root_box_lambda": WORKLOAD["root_leng"],
         "max_node_srcs": WORKLOAD["max_node_srcs"], "quadrature": "7-point",
         "digits": WORKLOAD["digits"], "interp_points": 2 * WORKLOAD["interp_order"],
         "precision": "complex fp64", "rhs_per_step": 1,
         "l2": "no flush: operator data read per step 0.54 GB > 126 MB L2"}
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            with open(self.path) as f:
                for line in f:
                    p = [v.strip() for v in line.split(",")]
                    if len(p) < 9:
                        continue
                    try:
                        sm.append(float(p[1]))
                        smax.append(float(p[2]))
                    except ValueError:
                        continue
                    for nm, v in zip(names, p[5:9]):
                        if v.lower().startswith("active"):
                            reasons.add(nm)
            os.unlink(self.path)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ------------------------------------------------------------------ reference arm

def parity_vector(n):
    """The seeded input vector of the reference arm's products (and of the GPU
    arm's parity check against them)."""
    return np.random.default_rng(7).standard_normal(n) + 1j * np.random.default_rng(8).standard_normal(n)


def run_reference(steps: int, warmup: int, save_y: str | None = None) -> dict:
    sys.path.insert(0, HERE)
    from oracle import ref_lib
    mesh, pw = make_problem()
    t0 = time.perf_counter()
    P = ref_lib.RefProblem("rwg", mesh, pw, digits=WORKLOAD["digits"], interp_order=WORKLOAD["interp_order"],
                           over_interp=WORKLOAD["over_interp"], root_leng=WORKLOAD["root_leng"],
                           max_node_srcs=WORKLOAD["max_node_srcs"], quad_prec=WORKLOAD["quad_prec"])
    setup_s = time.perf_counter() - t0
    x = parity_vector(P.n)
    y = None
    for _ in range(warmup):
        y = P.matvec(x)
    t0 = time.perf_counter()
    for _ in range(steps):
        y = P.matvec(x)
    dt = time.perf_counter() - t0
    if save_y:
        # the last product and how many products of x led to it (the reference
        # carries state from one product to the next)
        np.savez(save_y, y=y, products=warmup + steps)
    return {"value": steps / dt, "ms_per_step": dt / steps * 1e3, "setup_s": setup_s, "steps": steps}


def parity_vs_reference(dev, saved: str) -> dict:
    """Replays the reference arm's products of the seeded vector on a fresh
    plain-FP64 operator with the reference's rules and compares the last one
    with the reference's (the 1e-10 contract, on the benchmark workload)."""
    from mlfma_b200 import MLFMA, default_config
    f = np.load(saved)
    y_ref, count = f["y"], int(f["products"])
    mesh, pw = make_problem()
    cfg = default_config(quad_prec=WORKLOAD["quad_prec"], digits=WORKLOAD["digits"],
                         interp_order=WORKLOAD["interp_order"], over_interp=WORKLOAD["over_interp"],
                         root_leng=WORKLOAD["root_leng"], max_node_srcs=WORKLOAD["max_node_srcs"],
                         device=dev.index, precision=0)
    op = MLFMA.rwg(mesh, pw, config=cfg).setup()
    x = parity_vector(op.n)
    for _ in range(count):
        y = op.matvec(x)
    op.close()
    return {"rel_err": float(np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref)), "products": count,
            "tolerance": 1e-10,
            "what": "the reference's own product (oracle/_ref, same seeded x, same call sequence) against "
                    "mlfma_matvec, plain FP64, reference rules"}


# ------------------------------------------------------------------ our arm

def measure(torch, dev, rank, world, args, precision: int, clocks=None) -> dict:
    """Time one operator: device-resident products (value), host-buffer products
    (e2e) and per-stage CUDA-event times."""
    import torch.distributed as dist
    from mlfma_b200 import MLFMA, default_config
    mesh, pw = make_problem()
    cfg = default_config(quad_prec=WORKLOAD["quad_prec"], digits=WORKLOAD["digits"],
                         interp_order=WORKLOAD["interp_order"], over_interp=WORKLOAD["over_interp"],
                         root_leng=WORKLOAD["root_leng"], max_node_srcs=WORKLOAD["max_node_srcs"],
                         device=dev.index, precision=precision)
    t0 = time.perf_counter()
    op = MLFMA.rwg(mesh, pw, config=cfg)
    op.setup()
    setup_s = time.perf_counter() - t0
    tuning = op.autotune(1, reps=5)  # launch shapes timed on this operator (mlfma_autotune)
    st = op.stats()
    n = op.n
    g = torch.Generator(device="cpu").manual_seed(1234 + rank)
    xh = torch.complex(torch.randn(n, generator=g, dtype=torch.float64),
                       torch.randn(n, generator=g, dtype=torch.float64))
    x = xh.to(dev)
    y = torch.zeros(n, dtype=torch.complex128, device=dev)
    torch.cuda.synchronize(dev)
    # Every product runs on the operator's own stream; events are recorded there.
    stream = torch.cuda.ExternalStream(op.stream(), device=dev)

    def step():
        op.matvec_device(x.data_ptr(), y.data_ptr(), False, stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if clocks is not None:
        clocks.start()
        time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1) / args.steps
    y_dev = y.cpu().numpy().copy()

    # End to end through the C-ABI host-buffer call mlfma_matvec (the drop-in
    # boundary a C or C++ caller uses), pinned buffers, pointers prepared once;
    # each call copies x in, runs the product, copies y out and synchronises.
    import ctypes
    from mlfma_b200 import _lib
    xp = torch.empty(n, dtype=torch.complex128, pin_memory=True)
    yp = torch.empty(n, dtype=torch.complex128, pin_memory=True)
    xp.copy_(xh)
    xn, yn = xp.numpy(), yp.numpy()
    dp = ctypes.POINTER(ctypes.c_double)
    handle = _lib.lib(), op._h
    px, py = xn.view(np.float64).ctypes.data_as(dp), yn.view(np.float64).ctypes.data_as(dp)

    def e2e_time(fn, name):
        def e2e_step():
            rc = fn(handle[1], px, py, 0)
            if rc:
                raise RuntimeError(f"{name} returned {rc}")

        for _ in range(args.warmup):
            e2e_step()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        f1.record(stream)
        torch.cuda.synchronize(dev)
        return f0.elapsed_time(f1) / args.steps

    # mlfma_matvec_mapped: the gather and final kernels read x and write y in
    # the pinned buffers across the bus (the transfers inside the kernels);
    # mlfma_matvec: copies in and out around the device product
    e2e_ms = e2e_time(handle[0].mlfma_matvec_mapped, "mlfma_matvec_mapped")
    e2e_mapped_ok = bool(np.array_equal(yn, y_dev))
    e2e_copy_ms = e2e_time(handle[0].mlfma_matvec, "mlfma_matvec")
    clk = clocks.stop() if clocks is not None else None

    # Per-stage device times (stages launched back to back on the operator's stream).
    stages = [op.stage_times() for _ in range(max(5, min(args.steps, 50)))]
    avg = {k: float(np.mean([s[k] for s in stages])) for k in stages[0]}
    traffic = op.traffic()

    # Error of the product against the dense FP64 operator on DENSE_ROWS seeded
    # rows (every interaction evaluated directly, mlfma_dense_rows).
    rows = np.random.default_rng(77).choice(n, DENSE_ROWS, replace=False)
    xd = xh.numpy()
    dense = op.dense_rows(rows, xd)
    dense_err = float(np.linalg.norm(y_dev[rows] - dense) / np.linalg.norm(dense))

    op.close()

    # GMRES(50) solve of the plane-wave right-hand side to a 1e-4 relative
    # residual (FP64 residual; the mixed operator refines on it).  The solve
    # runs on the EFIE with its self terms (coincident and touching triangle
    # pairs in mixed-potential form, 1/R extracted): the reference's operator
    # leaves them out and GMRES then needs thousands of iterations.
    solve = None
    if not args.no_solve:
        scfg = default_config(quad_prec=WORKLOAD["quad_prec"], digits=WORKLOAD["digits"],
                              interp_order=WORKLOAD["interp_order"], over_interp=WORKLOAD["over_interp"],
                              root_leng=WORKLOAD["root_leng"], max_node_srcs=WORKLOAD["max_node_srcs"],
                              device=dev.index, precision=precision, self_terms=1, ref_compat=0)
        op = MLFMA.rwg(mesh, pw, config=scfg).setup()
        op.autotune(1, reps=5)
        b = op.rhs()
        op.solve(b, max_iter=5, tol=1e-12, restart=SOLVE["restart"], ref_givens=False,
                 refine=precision == 1)  # warm-up: workspace and graphs
        t0 = time.perf_counter()
        xs, info = op.solve(b, max_iter=SOLVE["max_iter"], tol=SOLVE["tol"], restart=SOLVE["restart"],
                            ref_givens=False, refine=precision == 1)
        wall = time.perf_counter() - t0
        far = op.farfield(xs, op.phi_cut(360))
        srows = np.random.default_rng(78).choice(n, DENSE_ROWS, replace=False)
        dres = float(np.linalg.norm(op.dense_rows(srows, xs) - b[srows]) / np.linalg.norm(b[srows]))
        solve = dict(seconds=wall, iterations=info.iterations, true_residual=info.true_residual,
                     converged=info.converged, refinements=info.refinements, far=far, x=xs,
                     dense_residual=dres)
        op.close()
    if world > 1:
        ms, e2e_ms, e2e_copy_ms = max_over_ranks(torch, dist, [ms, e2e_ms, e2e_copy_ms], dev)
    return dict(ms=ms, e2e_ms=e2e_ms, e2e_copy_ms=e2e_copy_ms, e2e_mapped_ok=e2e_mapped_ok, stages=avg,
                traffic=traffic, stats=st, setup_s=setup_s, n=n, y=y_dev, clocks=clk, solve=solve, tuning=tuning,
                dense_err=dense_err)


def max_over_ranks(torch, dist, values, device) -> list:
    """Each rank's timings (ms) -> their maximum over the ranks, on every rank."""
    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def job_rate(world: int, ms_per_step: float) -> float:
    """Whole-job products per second: every one of the world replicas applies
    one product per step, and the step takes the slowest rank's time."""
    return world * 1000.0 / ms_per_step


def measure_batched(torch, dev, args, precision: int) -> dict:
    """Products and the GMRES solve on NRHS incident plane waves at once
    (Fibonacci-sphere directions, theta polarisation) on the EFIE with self
    terms: device-resident matvecs/s over all right-hand sides, per-stage times,
    and the batched solve to the same 1e-4 FP64 residual."""
    from mlfma_b200 import MLFMA, default_config, inputs
    mesh, pw = make_problem()
    cfg = default_config(quad_prec=WORKLOAD["quad_prec"], digits=WORKLOAD["digits"],
                         interp_order=WORKLOAD["interp_order"], over_interp=WORKLOAD["over_interp"],
                         root_leng=WORKLOAD["root_leng"], max_node_srcs=WORKLOAD["max_node_srcs"],
                         device=dev.index, precision=precision, self_terms=1, ref_compat=0, max_rhs=NRHS)
    op = MLFMA.rwg(mesh, pw, config=cfg).setup()
    op.autotune(1, reps=5)
    tuning = op.autotune(NRHS, reps=3)
    n = op.n
    pws = inputs.fibonacci_planewaves(NRHS, wavenum=pw.wavenum)
    B = np.stack([op.rhs_planewave(p) for p in pws])
    X = torch.from_numpy(B).to(dev)
    Y = torch.zeros_like(X)
    stream = torch.cuda.ExternalStream(op.stream(), device=dev)
    for _ in range(args.warmup):
        op.matvec_multi_device(NRHS, X.data_ptr(), Y.data_ptr(), False, stream.cuda_stream)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = max(3, args.steps // 10)
    e0.record(stream)
    for _ in range(steps):
        op.matvec_multi_device(NRHS, X.data_ptr(), Y.data_ptr(), False, stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    st = op.stage_times_multi(NRHS)
    out = {"nrhs": NRHS, "ms_per_product": ms, "matvecs_per_s": NRHS * 1000.0 / ms,
           "us_per_rhs": ms * 1000.0 / NRHS, "stage_ms": st,
           "tuning": {k: v for k, v in tuning.items() if k != "m2m_rows"}}
    if not args.no_solve:
        op.solve_multi(B, max_iter=3, tol=1e-12, restart=SOLVE["restart"], refine=precision == 1)  # warm-up
        t0 = time.perf_counter()
        Xs, infos = op.solve_multi(B, max_iter=SOLVE["max_iter"], tol=SOLVE["tol"], restart=SOLVE["restart"],
                                   refine=precision == 1)
        wall = time.perf_counter() - t0
        out["solve"] = {"seconds": wall, "seconds_per_rhs": wall / NRHS,
                        "iterations_max": max(i.iterations for i in infos),
                        "iterations_mean": float(np.mean([i.iterations for i in infos])),
                        "true_residual_fp64_max": max(i.true_residual for i in infos),
                        "converged": all(i.converged for i in infos),
                        "method": f"{NRHS} simultaneous GMRES({SOLVE['restart']}) to {SOLVE['tol']:g}, x0 = 0"}
        out["_x0"] = Xs[0]
        out["_far0"] = op.farfield(Xs[0], op.phi_cut(360))
    op.close()
    return out


def batched_summary(bat, r64):
    """The many-right-hand-side block of the JSON line: per precision the
    product throughput and the solve, compared per right-hand side with the
    one-at-a-time FP64 path (matvec and solve of the benchmark's own plane wave)."""
    out = {"workload": f"{NRHS} plane waves, Fibonacci-sphere directions, theta polarisation, EFIE with self terms"}
    fp64_ms = r64["ms"]
    fp64_solve = r64["solve"]["seconds"] if r64["solve"] else None
    for p, b in bat.items():
        key = "fp64" if p == 0 else "mixed"
        d = {k: v for k, v in b.items() if not k.startswith("_")}
        d["matvec_speedup_per_rhs_vs_fp64_single"] = fp64_ms * 1000.0 / b["us_per_rhs"]
        if "solve" in b and fp64_solve:
            d["solve"]["speedup_per_rhs_vs_fp64_single_solve"] = fp64_solve / b["solve"]["seconds_per_rhs"]
        out[key] = d
    if 0 in bat and 1 in bat and "_far0" in bat[0] and "_far0" in bat[1]:
        f64, fmx = bat[0]["_far0"], bat[1]["_far0"]
        out["mixed"]["farfield_rel_err_vs_fp64_rhs0"] = float(np.linalg.norm(fmx - f64) / np.linalg.norm(f64))
    return out


def measure_problems(torch, dev, args) -> dict:
    """Many independent dipole problems of uneven size in one graph launch
    (mlfma_batch_*): NPROB problems, N log-uniform in [2,000, 50,000], seeded
    uniform positions in cubes of side 2-6 wavelengths, unit diagonal,
    complex-float far field and FP64 near field.  Device-resident batched
    product against the same products one operator at a time."""
    from mlfma_b200 import MLFMA, Batch, default_config, inputs
    rng = np.random.default_rng(2024)
    pw = inputs.PlaneWave(amplitude=1.0, pol=(1.0, 0.0, 0.0), khat=(0.0, 0.0, -1.0), wavenum=2.0 * np.pi)
    ops = []
    t0 = time.perf_counter()
    for i in range(NPROB):
        n = int(np.exp(rng.uniform(np.log(2000), np.log(50000))))
        side = float(rng.uniform(2.0, 6.0))
        d = inputs.make_dipoles(n, side=side, seed=100 + i)
        cfg = default_config(max_node_srcs=64, root_leng=side, digits=3, interp_order=3, over_interp=2.0,
                             device=dev.index, precision=1, ref_compat=0, self_terms=1)
        op = MLFMA.dipoles(d, pw, config=cfg).setup()
        op.autotune(1, reps=3)
        ops.append(op)
    setup_s = time.perf_counter() - t0
    batch = Batch(ops)
    sizes = [o.n for o in ops]
    offs = np.concatenate([[0], np.cumsum(sizes)])
    x = torch.randn(batch.total, dtype=torch.complex128, device=dev)
    y = torch.zeros_like(x)
    stream = torch.cuda.Stream(device=dev)
    steps = max(3, args.steps // 5)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.warmup):
        batch.matvec_device(x.data_ptr(), y.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    for _ in range(steps):
        batch.matvec_device(x.data_ptr(), y.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms_batch = e0.elapsed_time(e1) / steps
    # the same products one operator at a time, on one stream
    s0 = torch.cuda.ExternalStream(ops[0].stream(), device=dev)

    def one_at_a_time():
        for i, o in enumerate(ops):
            o.matvec_device(x.data_ptr() + 16 * int(offs[i]), y.data_ptr() + 16 * int(offs[i]), False,
                            s0.cuda_stream)

    for _ in range(args.warmup):
        one_at_a_time()
    torch.cuda.synchronize(dev)
    e0.record(s0)
    for _ in range(steps):
        one_at_a_time()
    e1.record(s0)
    torch.cuda.synchronize(dev)
    ms_seq = e0.elapsed_time(e1) / steps
    batch.close()
    for o in ops:
        o.close()
    return {"workload": f"{NPROB} dipole problems, N log-uniform in [2000, 50000], cubes of side 2-6 wavelengths, "
                        "unit diagonal, complex-float far field, FP64 near field",
            "unknowns_total": int(offs[-1]), "sizes_min_max": [int(min(sizes)), int(max(sizes))],
            "setup_s": setup_s, "ms_per_batched_product": ms_batch, "ms_one_operator_at_a_time": ms_seq,
            "speedup": ms_seq / ms_batch, "problem_products_per_s": NPROB * 1000.0 / ms_batch}


def measure_adjoint(torch, dev, args) -> dict:
    """The adjoint gradient on the benchmark sphere (30,720 RWGs, EFIE with
    self terms): per-edge loads z ~ U[0, 50] + j U[-20, 20] ohm, two weighted
    plane-wave excitations, J = summed far-field power in 16 seeded random
    directions.  One vector-Jacobian product = forward solve + far field +
    adjoint solve + gradient assembly (mlfma_vjp_farfield_power), timed at two
    solve tolerances, with a central-difference spot check (step 1e-4
    relative) on one load and one weight coordinate."""
    from mlfma_b200 import MLFMA, inputs
    mesh, pw = make_problem()
    t0 = time.perf_counter()
    op = MLFMA.rwg(mesh, pw, max_node_srcs=WORKLOAD["max_node_srcs"], root_leng=WORKLOAD["root_leng"],
                   device=dev.index, ref_compat=0, self_terms=1).setup()
    setup_s = time.perf_counter() - t0
    n = op.n
    r = np.random.default_rng(20)
    z = r.uniform(0, 50, n) + 1j * r.uniform(-20, 20, n)
    kh = np.random.default_rng(21).standard_normal((16, 3))
    kh /= np.linalg.norm(kh, axis=1)[:, None]
    pws = [pw] + inputs.fibonacci_planewaves(1)
    w = np.array([1.0 + 0.0j, 0.4 - 0.3j])
    op.set_loads(z)
    out = {"workload": "rwg_sphere_r2lambda_ico5 with loads U[0,50]+jU[-20,20] ohm, 2 excitations, "
                       "16 far-field directions", "unknowns": n, "setup_s": setup_s}
    op.vjp_farfield_power(pws, w, kh, max_iter=8000, tol=1e-6, restart=200)  # warm-up (graphs)
    for tol in (1e-6, 1e-10):
        t = time.perf_counter()
        J, gz, gw, _, infos = op.vjp_farfield_power(pws, w, kh, max_iter=8000, tol=tol, restart=200)
        sec = time.perf_counter() - t
        out[f"vjp_tol{tol:g}"] = {"seconds": sec, "forward_iterations": infos[0].iterations,
                                  "adjoint_iterations": infos[1].iterations,
                                  "forward_true_residual": infos[0].true_residual,
                                  "adjoint_true_residual": infos[1].true_residual, "J": J}
    B = [op.rhs_planewave(p) for p in pws]

    def J_of(zz, ww):
        op.set_loads(zz)
        x, _ = op.solve(sum(wj * bj for wj, bj in zip(ww, B)), max_iter=8000, tol=1e-12, restart=200,
                        ref_givens=False)
        F = op.farfield(x, kh)
        return float(np.vdot(F, F).real)

    k = int(np.random.default_rng(22).integers(n))
    h = 1e-4 * abs(z[k])
    zp, zm = z.copy(), z.copy()
    zp[k] += h
    zm[k] -= h
    fd_z = (J_of(zp, w) - J_of(zm, w)) / (2 * h)
    hw = 1e-4 * abs(w[1])
    wp, wm = w.copy(), w.copy()
    wp[1] += hw
    wm[1] -= hw
    fd_w = (J_of(z, wp) - J_of(z, wm)) / (2 * hw)
    op.set_loads(z)
    out["fd_check"] = {"coordinates": ["Re z[%d]" % k, "Re w[1]"],
                       "rel_err": [abs(gz[k].real - fd_z) / abs(fd_z), abs(gw[1].real - fd_w) / abs(fd_w)]}
    op.close()
    return out


def measure_large(torch, dev, args) -> dict:
    """The 8-wavelength sphere (491,520 RWGs, 7 levels) on the EFIE with self
    terms: products (FP64 and mixed), the FP64 GMRES(50) solve to 1e-4, the
    mixed solves (iterative refinement; flexible GMRES) and the mixed batched
    solve of LARGE_NRHS plane waves, each to 1e-4 on the FP64 residual; far
    field of every solution against the FP64 solution on 360 phi-cut angles."""
    from mlfma_b200 import MLFMA, default_config, inputs
    t0 = time.perf_counter()
    mesh = inputs.make_icosphere(LARGE["level"], radius=LARGE["radius"])
    pw = inputs.PlaneWave(amplitude=1.0, pol=(1.0, 0.0, 0.0), khat=(0.0, 0.0, -1.0), wavenum=2.0 * np.pi)
    mesh_s = time.perf_counter() - t0

    def cfg(precision, max_rhs=1):
        return default_config(quad_prec=LARGE["quad_prec"], digits=LARGE["digits"],
                              interp_order=LARGE["interp_order"], over_interp=LARGE["over_interp"],
                              root_leng=LARGE["root_leng"], max_node_srcs=LARGE["max_node_srcs"], device=dev.index,
                              precision=precision, self_terms=1, ref_compat=0, max_rhs=max_rhs)

    def products(op, steps):
        x = torch.randn(op.n, dtype=torch.complex128, device=dev)
        y = torch.zeros_like(x)
        stream = torch.cuda.ExternalStream(op.stream(), device=dev)
        for _ in range(3):
            op.matvec_device(x.data_ptr(), y.data_ptr(), False, stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            op.matvec_device(x.data_ptr(), y.data_ptr(), False, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / steps

    steps = max(5, min(args.steps, 20))
    out = {"workload": f"{LARGE['name']}: PEC sphere r = 8 wavelengths, icosphere level 7, root box 16, "
                       f"boxes split above {LARGE['max_node_srcs']} RWGs, EFIE with self terms",
           "mesh_s": mesh_s}
    rows = np.random.default_rng(91).choice(491520, 32, replace=False)
    phi = None
    # ---- FP64
    t0 = time.perf_counter()
    op = MLFMA.rwg(mesh, pw, config=cfg(0)).setup()
    out["unknowns"], out["levels"] = op.n, op.stats()["max_level"] + 1
    setup64 = time.perf_counter() - t0
    op.autotune(1, reps=3)
    ms64 = products(op, steps)
    st64 = op.stage_times()
    tr64 = op.traffic()
    b = op.rhs()
    xr = np.random.default_rng(92).standard_normal(op.n) + 1j * np.random.default_rng(93).standard_normal(op.n)
    yr = op.matvec(xr)
    dense_err = float(np.linalg.norm(yr[rows] - op.dense_rows(rows, xr)) / np.linalg.norm(op.dense_rows(rows, xr)))
    op.solve(b, max_iter=3, tol=1e-12, restart=LARGE_SOLVE["restart"], ref_givens=False)  # workspace, graphs
    t0 = time.perf_counter()
    x64, i64 = op.solve(b, max_iter=LARGE_SOLVE["max_iter"], tol=LARGE_SOLVE["tol"],
                        restart=LARGE_SOLVE["restart"], ref_givens=False)
    s64 = time.perf_counter() - t0
    phi = op.phi_cut(360)
    far64 = op.farfield(x64, phi)
    op.solve(b, max_iter=3, tol=1e-12, restart=LARGE_FLEX["restart"], flexible=True,
             inner_iters=LARGE_FLEX["inner_iters"])  # warm-up
    t0 = time.perf_counter()
    x64f, i64f = op.solve(b, max_iter=LARGE_SOLVE["max_iter"], tol=LARGE_SOLVE["tol"], restart=LARGE_FLEX["restart"],
                          flexible=True, inner_iters=LARGE_FLEX["inner_iters"])
    s64f = time.perf_counter() - t0
    op.close()
    out["fp64"] = {"setup_s": setup64, "ms_per_product": ms64, "matvecs_per_s": 1000.0 / ms64, "stage_ms": st64,
                   "matvec_alg_bytes": tr64["total"], "roofline": roofline(st64, tr64, "", LARGE["name"]),
                   "dense_rel_err_32_rows": dense_err,
                   "solve": {"seconds": s64, "iterations": i64.iterations, "true_residual_fp64": i64.true_residual,
                             "converged": i64.converged,
                             "method": f"GMRES({LARGE_SOLVE['restart']}) to {LARGE_SOLVE['tol']:g}, FP64"}}

    def farerr(x):
        return float(np.linalg.norm(op.farfield(x, phi) - far64) / np.linalg.norm(far64))

    # ---- mixed precision, one right-hand side
    t0 = time.perf_counter()
    op = MLFMA.rwg(mesh, pw, config=cfg(1)).setup()
    setupmx = time.perf_counter() - t0
    tune = op.autotune(1, reps=3)
    msmx = products(op, steps)
    stmx = op.stage_times()
    trmx = op.traffic()
    def flexible(o):
        t0 = time.perf_counter()
        x, info = o.solve(b, max_iter=LARGE_SOLVE["max_iter"], tol=LARGE_SOLVE["tol"], restart=LARGE_FLEX["restart"],
                          flexible=True, inner_iters=LARGE_FLEX["inner_iters"])
        return x, info, time.perf_counter() - t0

    def flex_summary(x, info, sec, what):
        return {"seconds": sec, "inner_iterations": info.iterations, "outer_iterations": info.refinements,
                "true_residual_fp64": info.true_residual, "converged": info.converged,
                "speedup_vs_fp64_gmres": s64 / sec, "farfield_rel_err_vs_fp64": farerr(x),
                "method": f"FGMRES({LARGE_FLEX['restart']}) in FP64 over inner GMRES of "
                          f"{LARGE_FLEX['inner_iters']} iterations {what}"}

    op.solve(b, max_iter=3, tol=1e-12, restart=LARGE_FLEX["restart"], flexible=True,
             inner_iters=LARGE_FLEX["inner_iters"])  # warm-up: workspaces, graphs
    xfl, ifl, sfl = flexible(op)
    out["mixed"] = {"setup_s": setupmx, "ms_per_product": msmx, "matvecs_per_s": 1000.0 / msmx,
                    "speedup_vs_fp64": ms64 / msmx, "stage_ms": stmx, "matvec_alg_bytes": trmx["total"],
                    "interp_path": tune["interp_path"], "schedule": tune["schedule"],
                    "solve_flexible": flex_summary(xfl, ifl, sfl, "on the complex-float far field")}
    out["fp64"]["solve_flexible"] = flex_summary(x64f, i64f, s64f, "on the FP64 far field")
    # the same flexible solve with its inner iterations on a cheaper operator of
    # the same sources and tree: 2-digit angular sampling, complex-float far field
    ccfg = cfg(1)
    ccfg.digits = LARGE_INNER_DIGITS
    inner = MLFMA.rwg(mesh, pw, config=ccfg).setup()
    inner.autotune(1, reps=3)
    op.set_inner_operator(inner)
    op.solve(b, max_iter=3, tol=1e-12, restart=LARGE_FLEX["restart"], flexible=True,
             inner_iters=LARGE_FLEX["inner_iters"])  # warm-up: the inner operator's graphs
    xfi, ifi, sfi = flexible(op)
    out["mixed"]["solve_flexible_inner"] = flex_summary(
        xfi, ifi, sfi, f"on a {LARGE_INNER_DIGITS}-digit complex-float inner operator (mlfma_set_inner_operator)")
    op.set_inner_operator(None)
    inner.close()
    op.close()
    # ---- mixed precision, many right-hand sides, flexible GMRES: LARGE_FLEX_NRHS
    # plane waves (the benchmark's first, then Fibonacci-sphere directions),
    # every outer step's inner solves run together through the many-rhs product
    if not args.no_large_batched_flex:
        nrf = LARGE_FLEX_NRHS
        t0 = time.perf_counter()
        op = MLFMA.rwg(mesh, pw, config=cfg(1, nrf)).setup()
        setupf = time.perf_counter() - t0
        op.autotune(1, reps=2)
        tf = op.autotune(nrf, reps=2)
        B = np.stack([b] + [op.rhs_planewave(p) for p in inputs.fibonacci_planewaves(nrf - 1)])
        X = torch.from_numpy(B).to(dev)
        Y = torch.zeros_like(X)
        stream = torch.cuda.ExternalStream(op.stream(), device=dev)
        for _ in range(2):
            op.matvec_multi_device(nrf, X.data_ptr(), Y.data_ptr(), False, stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            op.matvec_multi_device(nrf, X.data_ptr(), Y.data_ptr(), False, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        msf = e0.elapsed_time(e1) / 3
        stf = op.stage_times_multi(nrf)
        del X, Y
        op.solve_multi(B, max_iter=2, tol=1e-12, restart=LARGE_FLEX["restart"], flexible=True,
                       inner_iters=LARGE_FLEX["inner_iters"])  # warm-up: workspaces, graphs
        t0 = time.perf_counter()
        Xs, infos = op.solve_multi(B, max_iter=LARGE_SOLVE["max_iter"], tol=LARGE_SOLVE["tol"],
                                   restart=LARGE_FLEX["restart"], flexible=True,
                                   inner_iters=LARGE_FLEX["inner_iters"])
        sf = time.perf_counter() - t0
        xf0 = Xs[0]
        rows_f = rows[:8]
        dres = float(np.linalg.norm(op.dense_rows(rows_f, xf0) - b[rows_f]) / np.linalg.norm(b[rows_f]))
        ferr = farerr(xf0)
        op.close()
        torch.cuda.empty_cache()
        out["batched_flexible"] = {
            "nrhs": nrf, "setup_s": setupf, "ms_per_product": msf, "us_per_rhs": msf * 1000.0 / nrf,
            "stage_ms": stf, "matvec_speedup_per_rhs_vs_fp64": ms64 * nrf / msf,
            "matvec_speedup_per_rhs_vs_mixed": msmx * nrf / msf, "interp_path": tf["interp_path"],
            "solve": {"seconds": sf, "seconds_per_rhs": sf / nrf,
                      "inner_iterations_max": max(i.iterations for i in infos),
                      "outer_iterations_max": max(i.refinements for i in infos),
                      "true_residual_fp64_max": max(i.true_residual for i in infos),
                      "converged": all(i.converged for i in infos),
                      "speedup_per_rhs_vs_fp64_gmres": s64 * nrf / sf,
                      "farfield_rel_err_vs_fp64_rhs0": ferr,
                      "dense_residual_rhs0_8_rows": dres,
                      "method": f"{nrf} simultaneous FGMRES({LARGE_FLEX['restart']}) in FP64, inner GMRES of "
                                f"{LARGE_FLEX['inner_iters']} iterations on the complex-float far field, all "
                                "right-hand sides' inner solves through one many-rhs product per step"}}
    # ---- mixed precision, many right-hand sides (the benchmark's plane wave first);
    # measured at 16 right-hand sides: 1.04x per right-hand side (the slowest
    # column sets the iteration count), so not in the default run
    if args.large_batched:
        t0 = time.perf_counter()
        op = MLFMA.rwg(mesh, pw, config=cfg(1, LARGE_NRHS)).setup()
        setupb = time.perf_counter() - t0
        op.autotune(1, reps=3)
        tb = op.autotune(LARGE_NRHS, reps=2)
        B = np.stack([b] + [op.rhs_planewave(p) for p in inputs.fibonacci_planewaves(LARGE_NRHS - 1)])
        X = torch.from_numpy(B).to(dev)
        Y = torch.zeros_like(X)
        stream = torch.cuda.ExternalStream(op.stream(), device=dev)
        for _ in range(2):
            op.matvec_multi_device(LARGE_NRHS, X.data_ptr(), Y.data_ptr(), False, stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            op.matvec_multi_device(LARGE_NRHS, X.data_ptr(), Y.data_ptr(), False, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        msb = e0.elapsed_time(e1) / 3
        stb = op.stage_times_multi(LARGE_NRHS)
        op.solve_multi(B, max_iter=2, tol=1e-12, restart=LARGE_SOLVE["restart"], refine=True)
        t0 = time.perf_counter()
        Xs, infos = op.solve_multi(B, max_iter=LARGE_SOLVE["max_iter"], tol=LARGE_SOLVE["tol"],
                                   restart=LARGE_SOLVE["restart"], refine=True)
        sb = time.perf_counter() - t0
        out["batched"] = {"nrhs": LARGE_NRHS, "setup_s": setupb, "ms_per_product": msb,
                          "us_per_rhs": msb * 1000.0 / LARGE_NRHS, "stage_ms": stb,
                          "matvec_speedup_per_rhs_vs_fp64": ms64 * LARGE_NRHS / msb,
                          "interp_path": tb["interp_path"],
                          "solve": {"seconds": sb, "seconds_per_rhs": sb / LARGE_NRHS,
                                    "iterations_max": max(i.iterations for i in infos),
                                    "true_residual_fp64_max": max(i.true_residual for i in infos),
                                    "converged": all(i.converged for i in infos),
                                    "speedup_per_rhs_vs_fp64_single": s64 * LARGE_NRHS / sb,
                                    "farfield_rel_err_vs_fp64_rhs0": farerr(Xs[0]),
                                    "method": f"{LARGE_NRHS} simultaneous GMRES({LARGE_SOLVE['restart']}) with "
                                              "iterative refinement, complex-float far field, FP64 residual"}}
        op.close()
    best = max([out["mixed"]["solve_flexible"]["speedup_vs_fp64_gmres"],
                out["mixed"]["solve_flexible_inner"]["speedup_vs_fp64_gmres"]] +
               ([out["batched"]["solve"]["speedup_per_rhs_vs_fp64_single"]] if "batched" in out else []) +
               ([out["batched_flexible"]["solve"]["speedup_per_rhs_vs_fp64_gmres"]
                 if out["batched_flexible"]["solve"]["converged"] else 0.0] if "batched_flexible" in out else []))
    out["precision_gain"] = {"what": "FP64 vs mixed far field under the same FGMRES", "speedup": s64f / sfl}
    out["solver_gain"] = {"what": "FP64 GMRES(50) vs FP64 FGMRES", "speedup": s64 / s64f}
    out["target"] = {"what": "mixed/batched solve to 1e-4 at least 4x faster than the FP64 GPU solve, far-field "
                             "error below 1e-3", "best_speedup": best, "met": bool(best >= 4.0)}
    # where the time of the best mixed solve goes, and what a 4x solve would need
    sf = out["mixed"]["solve_flexible"]  # its product is the measured mixed product
    inner = max(1, sf["inner_iterations"])
    per_it = sf["seconds"] / inner * 1000.0
    need = s64 / 4.0
    out["target"]["gap"] = {
        "solve_s": sf["seconds"], "solve_s_for_4x": need,
        "ms_per_inner_iteration": per_it, "ms_per_mixed_product": msmx,
        "ms_per_iteration_besides_the_product": per_it - msmx,
        "ms_per_inner_iteration_for_4x": need / inner * 1000.0,
        "mixed_product_stage_ms": stmx,
        "what": "the solve's time per inner iteration = one mixed product (stage times above, the near field and "
                "the translations largest) + Arnoldi/CGS2 in FP64 and the outer FP64 steps; a 4x solve at the same "
                "iteration count needs ms_per_inner_iteration_for_4x"}
    return out


def solve_summary(sv):
    return {"seconds": sv["seconds"], "iterations": sv["iterations"], "true_residual_fp64": sv["true_residual"],
            "dense_residual": sv["dense_residual"], "converged": sv["converged"], "refinements": sv["refinements"],
            "method": f"GMRES({SOLVE['restart']}) to {SOLVE['tol']:g} relative residual, x0 = 0, plane-wave rhs",
            "operator": "EFIE with self terms (self_terms=1, ref_compat=0)"}


def roofline(avg, traffic, precision_name, workload=None):
    # The near field's tile kernel is the longest single kernel of a product
    # (launch list in profiles/); the stage time also holds its per-target sum.
    dom = "near_field"
    peaks = {}
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    achieved = traffic[dom] / (avg[dom] * 1e-3) / 1e9
    ncu_traffic = None
    try:
        with open(os.path.join(HERE, "profiles", "traffic.json")) as f:
            ncu_traffic = json.load(f).get((workload or WORKLOAD["name"]) + precision_name, {}).get(dom)
    except (OSError, ValueError):
        pass
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
            "frac": achieved / hbm_peak, "peak_source": peak_src, "traffic": ncu_traffic,
            "algorithmic_bytes": traffic[dom], "avg_launch_ms": avg[dom]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-solve", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-large", action="store_true", help="skip the 8-wavelength sphere (491,520 unknowns)")
    ap.add_argument("--large-batched", action="store_true",
                    help="also the batched solve of the 8-wavelength sphere (about 200 s)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-gradient leg")
    ap.add_argument("--no-large-batched-flex", action="store_true",
                    help="skip the 8-wavelength sphere's batched flexible solve (64 right-hand sides)")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--save-y", default=None, help="reference arm: save its last product here (.npz)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        r = run_reference(args.steps, max(args.warmup, 0), save_y=args.save_y)
        line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
                "data": "synthetic (seeded icosphere mesh)",
                "config": config_dict({"reference_setup_s": r["setup_s"]}),
                "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": 1, "kind": "reference",
                                 "sample": f"{args.steps} full matvecs of the workload after {args.warmup} "
                                           "warm-up matvecs; the reference is single-threaded"},
                "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    if args.warmup < 3:
        print("warm-up must be >= 3", file=sys.stderr)
        args.warmup = 3
    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)

    # CPU baseline in a child process (rank 0, N = 1), overlapping GPU setup.
    cpu_proc = None
    ref_y = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        fd, ref_y = tempfile.mkstemp(suffix=".npz")
        os.close(fd)
        cpu_proc = subprocess.Popen([sys.executable, os.path.abspath(__file__), "--impl", "reference",
                                     "--steps", str(args.cpu_steps), "--warmup", "1", "--save-y", ref_y],
                                    stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    sys.path.insert(0, HERE)

    r64 = measure(torch, dev, rank, world, args, precision=0, clocks=ClockSampler(local_rank))
    rmx = None if args.no_mixed else measure(torch, dev, rank, world, args, precision=1)
    # The secondary legs (many right-hand sides, many problems, the adjoint
    # gradient, the 8-wavelength sphere) run with one process only: the
    # replicas of a multi-GPU run report the headline product.
    solo = world == 1
    bat = None
    if not args.no_batched and solo:
        bat = {p: measure_batched(torch, dev, args, p) for p in ((0, 1) if not args.no_mixed else (0,))}
    probs = None if args.no_batched or not solo else measure_problems(torch, dev, args)
    adj = None if args.no_adjoint or not solo else measure_adjoint(torch, dev, args)
    large = None if args.no_large or not solo else measure_large(torch, dev, args)

    if rank == 0:
        cpu = None
        if cpu_proc is not None:
            try:
                out, _ = cpu_proc.communicate(timeout=900)
                r = json.loads(out.strip().splitlines()[-1])
                cpu = {"value": r["value"], "unit": UNIT, "cores": 1, "kind": "reference",
                       "sample": f"{args.cpu_steps} full matvecs of this workload by the reference built from its "
                                 f"sources (oracle/_ref), after 1 warm-up matvec and a "
                                 f"{r['config'].get('reference_setup_s', 0):.0f} s setup"}
            except Exception as e:  # noqa: BLE001
                cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"failed: {e}"}
        parity = None
        if ref_y is not None:
            try:
                parity = parity_vs_reference(dev, ref_y)
            except Exception as e:  # noqa: BLE001
                parity = {"rel_err": None, "error": str(e)}
            finally:
                os.unlink(ref_y)
        st, n, ms, e2e_ms = r64["stats"], r64["n"], r64["ms"], r64["e2e_ms"]
        line = {
            "metric": METRIC, "value": job_rate(world, ms), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded icosphere mesh)",
            "config": config_dict({"parallelism": f"replicas{world}", "levels": st["max_level"],
                                   "near_entries": st["near_entries"], "setup_s": r64["setup_s"],
                                   "autotuned": {"m2l_chunk": r64["tuning"]["m2l_chunk"],
                                                 "near_blocks_per_sm": r64["tuning"]["near_blocks_per_sm"],
                                                 "m2m_rows": [v for v in r64["tuning"]["m2m_rows"] if v]}}),
            "e2e": {"value": job_rate(world, e2e_ms), "unit": UNIT, "h2d_bytes_per_step": n * 16,
                    "d2h_bytes_per_step": n * 16, "call": "mlfma_matvec_mapped",
                    "what": "pinned host buffers; x read and y written across the bus by the product's first and "
                            "last kernels, synchronised every call",
                    "equals_device_product": r64["e2e_mapped_ok"],
                    "copy_path": {"value": job_rate(world, r64["e2e_copy_ms"]), "call": "mlfma_matvec",
                                  "what": "the same buffers through cudaMemcpyAsync in and out"}},
            "gpu_launches": int(st.get("launches_per_matvec", 0)) * args.steps,
            "roofline": roofline(r64["stages"], r64["traffic"], ""),
            "stage_ms": r64["stages"],
            "matvec_alg_bytes": r64["traffic"]["total"],
            "clocks": r64["clocks"],
            "cpu_baseline": cpu,
            "parity_rel_err_vs_reference": parity["rel_err"] if parity else None,
            "parity_vs_reference": parity,
            "dense_check": {"rows": DENSE_ROWS, "matvec_rel_err_fp64": r64["dense_err"],
                            "reference": "the same rows of the operator with every interaction evaluated "
                                         "directly in FP64 (mlfma_dense_rows)"},
        }
        if r64["solve"] is not None:
            line["solve_fp64"] = solve_summary(r64["solve"])
        if rmx is not None:
            err = float(np.linalg.norm(rmx["y"] - r64["y"]) / np.linalg.norm(r64["y"]))
            line["mixed"] = {"value": job_rate(world, rmx["ms"]), "ms_per_step": rmx["ms"],
                             "e2e": job_rate(world, rmx["e2e_ms"]), "speedup_vs_fp64": ms / rmx["ms"],
                             "rel_diff_vs_fp64": err, "dense_rel_err": rmx["dense_err"],
                             "dtype": "c64 far field, c128 near field",
                             "stage_ms": rmx["stages"], "roofline": roofline(rmx["stages"], rmx["traffic"], "_mixed"),
                             "matvec_alg_bytes": rmx["traffic"]["total"]}
            if rmx["solve"] is not None and r64["solve"] is not None:
                sm, s64 = rmx["solve"], r64["solve"]
                line["mixed"]["solve"] = solve_summary(sm)
                line["mixed"]["solve"]["speedup_vs_fp64"] = s64["seconds"] / sm["seconds"]
                line["mixed"]["solve"]["farfield_rel_err_vs_fp64"] = float(
                    np.linalg.norm(sm["far"] - s64["far"]) / np.linalg.norm(s64["far"]))
        if bat is not None:
            line["batched"] = batched_summary(bat, r64)
        if probs is not None:
            line["problems"] = probs
        if adj is not None:
            line["adjoint"] = adj
        if large is not None:
            line["large"] = large
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
