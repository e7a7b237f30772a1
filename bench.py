"""Benchmark: composite-geometry Poisson solves per second on B200 (solves/s and HBM GB/s).

Workload (the largest cross configuration that fits one GPU): a cross of 5 subdomains of 2048 x 2048 cells
(centre + 4 arms), h = 1/2048, Neumann arm tips, Dirichlet elsewhere, seeded zero-mean Gaussian RHS,
GMRES(m=20, tol=1e-14, maxIter=100) on the interface unknowns. One step = one full composite solve
(inputs re-filled from a resident copy first, since a solve consumes its right-hand side). Four forms are
timed (FP64, FP64 + refinement, FP32 + FP64 refinement, FP64 solve + FP32 corrections); the headline is the
fastest whose answer is within 1e-10 relative L2 of the refined solution. Every form's answer is also
compared with the reference's own answer to the same workload (the CPU leg, which times it). Further
sections: the 512-problem batched workload (`batched_uneven`; split between the ranks when N > 1;
--no-batched skips it) and the 9 x 4096^2 tree (`large_tree`, N = 1; --no-large skips it).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --probe transform|rect|composite|batch ...   (one kernel family or solve; see PROBE_USAGE)

N > 1 runs N independent replicas of the cross, one process per GPU under torchrun. Prints one JSON line on
rank 0.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s and HBM GB/s (% peak), FP32+IR vs FP64 at 1e-10 rel L2, 1 B200"
N_CELLS = 2048
GMRES = (20, 1e-14, 100)
SEED = 2024
IR_REL_TOL = 1e-11
# DRAM bytes of one k_xform_rc<double, DD, 4096> launch on 2048 x 2048 (ncu capture summarised in
# profiles/k_xform_rc_DD_2048x2048_f64.md): the input is read once, the output stays in L2
DD_TRAFFIC_BYTES = 33.752576e6 + 0.015104e6
INNER = {"f64ir": "f64", "f32ir": "f32", "mixedir": "mixed"}


def workload_config():
    return {
        "workload": f"cross 5x{N_CELLS}x{N_CELLS} (centre + 4 arms), h=1/{N_CELLS}, Neumann arm tips, "
                    f"zero-mean Gaussian RHS (seed {SEED}), GMRES(m={GMRES[0]}, tol={GMRES[1]:g}, maxIter={GMRES[2]}); "
                    f"FP32+IR to |correction| <= {IR_REL_TOL:g} |u|",
        "cells": 5 * N_CELLS * N_CELLS,
        "l2_policy": "inputs larger than L2 (5 x 33.5 MB FP64 fields re-filled each step)",
    }


# ------------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ------------------------------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def max_over_ranks(x: float, dist, device) -> float:
    """The slowest rank's time (every rank must call this, in the same order)."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(steps: int, world: int, ms: float) -> float:
    """Whole-job solves/s of `world` independent replicas, each doing `steps` solves in `ms` (the max over
    ranks)."""
    return steps * world / (ms / 1e3)


def partition_problems(cells, world: int):
    """Split independent problems over `world` ranks, balanced by cells: the largest problems first, each onto
    the rank with the fewest cells so far (ties to the lower rank). Deterministic, so every rank computes the
    same split without communicating. Returns one sorted list of problem indices per rank."""
    load = [0] * world
    parts = [[] for _ in range(world)]
    for p in sorted(range(len(cells)), key=lambda i: (-cells[i], i)):
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(p)
        load[r] += cells[p]
    return [sorted(x) for x in parts]


def sharded_value(problems: int, ms_max: float) -> float:
    """Whole-job solves/s of one batch of `problems` split over the ranks, the slowest rank taking ms_max."""
    return problems / (ms_max / 1e3)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------------------------------------
# CPU reference (the reference's own sources, oracle/_ref) -- baseline leg and --impl reference
# ------------------------------------------------------------------------------------------------
def reference_solver(n: int, threads: int):
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import refsolve as RS
    from focalors_poisson_b200 import workloads as W

    g = W.cross(n, neumann_tips=True)
    rhs = W.gaussian_rhs(g, SEED)
    # Root Schur matrices in closed form (oracle/schur_closed_form.py): the reference's own construction
    # needs one full solve per interface cell. The timed region is the reference's unmodified solve().
    return RS.reference_case(g, *GMRES), rhs


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    from oracle import refbind as R

    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfpref.so not built (needs the reference "
                                                               "sources at build time)"}))
        return
    case, rhs = reference_solver(N_CELLS, threads)
    budget = 150.0
    times = []
    for _ in range(max(0, min(args.warmup, 0))):
        case.solve(rhs)
    t_start = time.perf_counter()
    while len(times) < args.steps:
        _, t = case.solve(rhs)
        times.append(t)
        if time.perf_counter() - t_start + t > budget:
            break
    total = sum(times)
    value = len(times) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": len(times), "steps_requested": args.steps, "warmup": 0, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "reference",
                         "sample": "full solves of the same workload on the reference's own sources (FFTW r2c via "
                                   "the project shim), OpenMP Hybrid build, each solve one step; steps capped at "
                                   "~150 s of CPU time; warm-up skipped (CPU)"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def cpu_reference_leg(g, rhs):
    """The CPU baseline of the main arm and the reference's answer for the parity figures: one full
    reference solve of the same 5 x 2048^2 workload on the host cores (oracle/_ref, the reference's own
    sources; its time is the baseline), then one refinement step of that answer by the same solver
    (oracle/refsolve.py) so that the GPU forms can be compared with the reference below its own FP64
    round-off."""
    threads = os.cpu_count() or 1
    try:
        from oracle import refbind as R
        from oracle import refsolve as RS

        if not R.available():
            return {"value": None, "unit": "solves/s", "cores": threads, "kind": "reference",
                    "sample": "unavailable: oracle/_ref/libfpref.so not built"}, None
        os.environ["OMP_NUM_THREADS"] = str(threads)
        ref = RS.reference_answer(g, rhs, *GMRES)
        base = {"value": 1.0 / ref["seconds"], "unit": "solves/s", "cores": threads, "kind": "reference",
                "sample": f"one full reference solve of the same workload (5x{N_CELLS}x{N_CELLS}, "
                          f"{ref['seconds']:.1f} s), the reference's own sources with the FFTW r2c shim, "
                          "OpenMP Hybrid build", "sample_seconds": ref["seconds"]}
        return base, ref
    except Exception as e:  # the baseline leg never blocks the GPU measurement
        return {"value": None, "unit": "solves/s", "cores": threads, "kind": "reference",
                "sample": f"failed: {e}"}, None


# ------------------------------------------------------------------------------------------------
# Batched uneven workload: 512 independent L/T problems (sides 64..1024), one launch sequence
# ------------------------------------------------------------------------------------------------
BATCH_PROBLEMS = 512
BATCH_FORMS = (("f64", 0), ("f32", 2), ("f32", 3))  # (storage precision, inner solves of the refinement)


def launch_shape(info):
    """The batched solver's autotuned launch shape. The transform grid is either persistent (a fixed number of
    CTAs per SM looping over the work items) or one CTA per work item; fp_batch_info reports the latter as
    1 << 20 CTAs per SM."""
    bps = info["dst_blocks_per_sm"]
    grid = "one CTA per work item" if bps >= 1 << 20 else f"persistent, {bps} CTAs per SM"
    return {"dst_threads": info["dst_threads"], "dst_grid": grid, "chase_threads": info["chase_threads"]}


def batched_section(args, dev, rank, world=1, dist=None):
    """solves/s of the batched workload in its FP64-direct and FP32+refinement forms (each step: refill the
    right-hand sides from a resident copy, then one replay of the captured graph), their accuracy against
    the FP64 solve refined twice, the plain per-problem FP64 path on a sample, and the reference CPU build
    on a sample. With several ranks the 512 problems are split between them (partition_problems), one
    batch and one captured graph per GPU; no data crosses between GPUs, and the job's time is the slowest
    rank's."""
    import torch

    from focalors_poisson_b200 import capi
    from focalors_poisson_b200 import workloads as W

    all_probs, all_rhs = W.batched_uneven(BATCH_PROBLEMS, SEED)
    mine = partition_problems([g.cells() for g in all_probs], world)[rank]
    probs, rhs = [all_probs[p] for p in mine], [all_rhs[p] for p in mine]
    flat = [x for r in rhs for x in r]
    cells = sum(int(x.size) for x in flat)
    pristine = [torch.tensor(x, device=dev) for x in flat]
    work = [torch.empty_like(p) for p in pristine]
    starts = np.cumsum([0] + [len(g.nx) for g in probs])
    out = {"workload": f"{BATCH_PROBLEMS} L/T problems (3-4 subdomains, sides uniform in 64..1024 step 32, "
                       f"seed {SEED}), Dirichlet outer faces, N(0,1) RHS",
           "cells": sum(g.cells() for g in all_probs),
           "l2_policy": "inputs larger than L2 (4.4 GB of FP64 fields re-filled each step)", "forms": {}}
    if world > 1:
        out["sharding"] = {"ranks": world, "split": "problems balanced by cells, one batch and one graph per GPU, "
                                                    "no collective on the data path",
                           "problems_rank0": len(mine), "cells_rank0": cells}

    def refill():
        for w, p in zip(work, pristine):
            w.copy_(p)

    # arbiter: FP64 solve refined twice
    ref = capi.Batch(probs, precision="f64")
    refill()
    ref.solve(work, steps=3)
    torch.cuda.synchronize()
    exact = [w.clone() for w in work]
    del ref
    lib = capi.lib()
    # problems the reference also solves (CPU leg below, rank 0): every 128th of this rank's share
    csample = list(range(0, len(probs), 128))
    sample_out = {}
    for prec, steps in BATCH_FORMS:
        t0 = time.perf_counter()
        b = capi.Batch(probs, precision=prec)
        torch.cuda.synchronize()
        setup = time.perf_counter() - t0
        for _ in range(max(args.warmup, 3)):
            refill()
            b.solve(work, steps=steps, graph=True)
        torch.cuda.synchronize()
        l0 = lib.fp_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            refill()
            b.solve(work, steps=steps, graph=True)
        e1.record()
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, dev)
        launches = (lib.fp_launch_count() - l0) / args.steps
        perr = []
        for p in range(len(probs)):
            rng_ = range(starts[p], starts[p + 1])
            num = sum(float(((work[d] - exact[d]) ** 2).sum()) for d in rng_)
            den = sum(float((exact[d] ** 2).sum()) for d in rng_)
            perr.append((num / den) ** 0.5)
        res = b.residuals(work, pristine)
        info = b.info()
        key = f"{prec}" + (f"+ir{steps}" if steps else "")
        sample_out[key] = {p: [work[d].cpu().numpy() for d in range(starts[p], starts[p + 1])] for p in csample}
        out["forms"][key] = {
            "solves_per_s": sharded_value(BATCH_PROBLEMS, ms), "ms_per_batch": ms, "setup_s": setup,
            "max_rel_l2_vs_refined": max_over_ranks(max(perr), dist, dev),
            "max_rel_residual": max_over_ranks(float(res.max()), dist, dev),
            "gpu_launches_per_batch": launches, "graph_kernels": info["graph_kernels"],
            "launch_shape": launch_shape(info)}
        del b
        torch.cuda.empty_cache()
    ok = {k: v for k, v in out["forms"].items() if v["max_rel_l2_vs_refined"] <= 1e-10}
    out["headline_form"] = max(ok, key=lambda k: ok[k]["solves_per_s"]) if ok else None
    # plain FP64 GPU path: the single-problem C-ABI Schur GMRES solve (FP_NO_SPECTRAL), one problem after
    # another, on every 32nd problem (setup excluded)
    sample = list(range(0, len(probs), 32))
    tot = 0.0
    for p in sample:
        solver = capi.Composite(probs[p], 20, 1e-12, 100, spectral=False)
        f = [torch.tensor(x, device=dev) for x in rhs[p]]
        solver.solve([x.clone() for x in f])
        torch.cuda.synchronize()
        reps = 3
        t0 = time.perf_counter()
        for _ in range(reps):
            g = [x.clone() for x in f]
            solver.solve(g)
        torch.cuda.synchronize()
        tot += (time.perf_counter() - t0) / reps
        del solver
    out["plain_fp64_per_problem"] = {"solves_per_s": len(sample) / tot, "sample": f"{len(sample)} problems "
                                     "(every 32nd), one Schur-GMRES fp_composite_solve_f64 each, wall clock, "
                                     "setup excluded"}
    if out["headline_form"]:
        out["headline_vs_plain_fp64"] = out["forms"][out["headline_form"]]["solves_per_s"] / \
            out["plain_fp64_per_problem"]["solves_per_s"]
    # the fastest FP32-storage form within 1e-10 of the refined answer
    f32 = [k for k in out["forms"] if k.startswith("f32") and out["forms"][k]["max_rel_l2_vs_refined"] <= 1e-10]
    if f32:
        best = max(f32, key=lambda k: out["forms"][k]["solves_per_s"])
        out["batched_fp32ir_form"] = best
        out["batched_fp32ir_vs_plain_fp64"] = out["forms"][best]["solves_per_s"] / \
            out["plain_fp64_per_problem"]["solves_per_s"]
    # reference CPU build on a sample (root Schur matrices in closed form; timed region = its solve()), and
    # every form's answer on those problems against the reference's answer (refined once by its solver)
    if rank == 0 and not args.no_cpu_baseline:
        try:
            from oracle import refbind as R
            from oracle import refsolve as RS

            if R.available():
                os.environ["OMP_NUM_THREADS"] = str(os.cpu_count() or 1)
                ctot = 0.0
                worst = {k: 0.0 for k in sample_out}
                worst_plain = {k: 0.0 for k in sample_out}
                for p in csample:
                    ref = RS.reference_answer(probs[p], rhs[p], 20, 1e-12, 100)
                    ctot += ref["seconds"]
                    for k in sample_out:
                        worst[k] = max(worst[k], RS.rel_l2(sample_out[k][p], ref["refined"]))
                        worst_plain[k] = max(worst_plain[k], RS.rel_l2(sample_out[k][p], ref["plain"]))
                for k in sample_out:
                    out["forms"][k]["max_rel_l2_vs_reference"] = worst[k]
                    out["forms"][k]["max_rel_l2_vs_reference_plain"] = worst_plain[k]
                out["reference_sample"] = f"problems {csample}: the reference's own solve() (GMRES tol 1e-12), " \
                                          "refined once by the same solver"
                out["cpu_baseline"] = {"solves_per_s": len(csample) / ctot, "cores": os.cpu_count() or 1,
                                       "kind": "reference", "sample": f"{len(csample)} problems (every 128th), "
                                       "the reference's own solve() on the host cores"}
        except Exception as e:  # the baseline leg never blocks the GPU measurement
            out["cpu_baseline"] = {"solves_per_s": None, "sample": f"failed: {e}"}
    del pristine, work, exact
    torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------------------------------------------
# Large composite: 9 subdomains of 4096^2 in a depth-2 tree, periodic arms (--no-large skips; setup ~2 min)
# ------------------------------------------------------------------------------------------------
def large_section(args, dev):
    """Forward solves (FP64, FP32 + FP64 refinement) and the adjoint solve of the 9 x 4096^2 tree with
    periodic W / E arms; each step refills the RHS from a resident copy. Setup (Schur matrices, interface
    inverses) is timed separately."""
    import torch

    from focalors_poisson_b200 import capi
    from focalors_poisson_b200 import workloads as W

    g = W.tree9_large(4096)
    pristine = W.gaussian_bumps_rhs(g, SEED, device=dev)
    work = [torch.empty_like(p) for p in pristine]
    out = {"workload": "tree of 9 x 4096^2 (centre, 4 arms, 4 corners on the y-arms), W / E arms periodic in y, "
                       "Neumann arm-tip and corner x faces, Dirichlet elsewhere, sum of 32 Gaussian bumps "
                       f"(seed {SEED}); GMRES(20, 1e-12, 100)", "cells": sum(int(p.numel()) for p in pristine)}
    t0 = time.perf_counter()
    c = capi.Composite(g, 20, 1e-12, 100)
    for w, p in zip(work, pristine):
        w.copy_(p)
    c.solve(work)  # the Schur matrices and interface inverses are built at creation; first solve warms up
    torch.cuda.synchronize()
    out["setup_s"] = time.perf_counter() - t0

    def timed(fn):
        for _ in range(2):
            for w, p in zip(work, pristine):
                w.copy_(p)
            info = fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 3
        e0.record()
        for _ in range(reps):
            for w, p in zip(work, pristine):
                w.copy_(p)
            info = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, info

    ms, info = timed(lambda: c.solve(work))
    u64 = [w.clone() for w in work]
    out["f64"] = {"solves_per_s": 1e3 / ms, "ms": ms, "rel_residual": c.residual(u64, pristine),
                  "gmres_iterations": info["iterations"]}
    ms, info = timed(lambda: c.solve_ir(work, rel_tol=1e-11, max_refine=10))
    num = sum(float(((a - b) ** 2).sum()) for a, b in zip(work, u64))
    den = sum(float((b ** 2).sum()) for b in work)
    out["f32ir"] = {"solves_per_s": 1e3 / ms, "ms": ms, "rel_residual": c.residual(work, pristine),
                    "refinements": info["refinements"], "rel_l2_vs_f64": (num / den) ** 0.5}
    ms, info = timed(lambda: c.adjoint(work))
    out["adjoint_f64"] = {"solves_per_s": 1e3 / ms, "ms": ms}
    del c, work, pristine, u64
    torch.cuda.empty_cache()
    return out



def star3d(n):
    """A root box of n^3 cells with four n^3 children on its x-, x+, y- and z+ faces (h = 1/n), Dirichlet outer
    faces except Neumann x+ on the x+ child: (domains, connections, bc) for capi.Composite3D."""
    h = 1.0 / n
    doms = [(n, n, n, h, h, h)] * 5
    conns = [(0, 0, 1), (0, 1, 2), (0, 2, 3), (0, 5, 4)]
    bc = [[0] * 6, [0] * 6, [0, 1, 0, 0, 0, 0], [0] * 6, [0] * 6]
    return doms, conns, bc


def threed_section(args, dev, with_cpu):
    """3D solves. PoissonSolver3D on 256^3 (Dirichlet faces) and ConcatPoissonSolver3D on a star of five 64^3
    boxes, device-timed with CUDA events (each step refills the right-hand side from a resident copy). Beside
    them the reference's own 3D solvers (oracle/_ref) on the host cores: the rectangle at the same size, the
    composite at 32^3 per box (the reference builds its Schur matrices by one impulse solve per face cell)."""
    import torch

    from focalors_poisson_b200 import capi

    out = {}
    n = 256
    h = 1.0 / n
    bc = (0, 0, 0, 0, 0, 0)
    f0 = np.random.default_rng(SEED).standard_normal((n, n, n))
    rect = capi.Rect3D(n, n, n, h, h, h, bc)
    x = torch.tensor(f0, device=dev)
    w = torch.empty_like(x)

    def device_time(step, reps):
        for _ in range(3):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            step()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def rect_step():
        w.copy_(x)
        rect.solve(w)

    ms = device_time(rect_step, max(args.steps, 5))
    # z-transform, transpose, y-transform, chase (two passes), y-inverse, transpose back, z-inverse: 8 passes
    # that each read and write the field
    alg = 16 * n ** 3 * 8
    peak, peak_kind = measured_peaks()
    r3 = {"workload": f"PoissonSolver3D {n}^3, Dirichlet faces, h = 1/{n}, N(0,1) right-hand side (seed {SEED})",
          "solves_per_s": 1e3 / ms, "ms": ms, "algorithmic_bytes": alg, "achieved_gbs": alg / ms / 1e6,
          "frac_of_hbm": alg / ms / 1e6 / peak, "peak_source": f"{peak_kind} hbm_gbs",
          "step_note": "each step includes the 134 MB device copy that refills the right-hand side"}
    if with_cpu:
        from oracle import refbind as R

        got = w.cpu().numpy()
        t0 = time.perf_counter()
        ref, sec = R.poisson3d_solve(f0, h, h, h, bc)
        r3["cpu_reference"] = {"solves_per_s": 1.0 / sec, "seconds": sec, "cores": os.cpu_count(),
                               "what": "the reference's PoissonSolver3D::solve on the same field (oracle/_ref)",
                               "wall_s": time.perf_counter() - t0}
        r3["rel_l2_vs_reference"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    out["rect3d"] = r3
    del rect, x, w

    doms, conns, cbc = star3d(64)
    t0 = time.perf_counter()
    c3 = capi.Composite3D(doms, conns, cbc, 20, 1e-10, 100)
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    rng = np.random.default_rng(SEED + 1)
    rhs = [torch.tensor(rng.standard_normal(d[:3]), device=dev) for d in doms]
    work = [torch.empty_like(r) for r in rhs]
    info = {}

    def c3_step():
        for a, b in zip(work, rhs):
            a.copy_(b)
        info.update(c3.solve(work))

    ms = device_time(c3_step, 5)
    c3d = {"workload": "ConcatPoissonSolver3D: root 64^3 with four 64^3 children (x-, x+, y-, z+ faces), "
                       "GMRES(20, 1e-10, 100), N(0,1) right-hand sides", "solves_per_s": 1e3 / ms, "ms": ms,
           "setup_s": setup, "gmres_iterations": info.get("iterations")}
    del c3, rhs, work
    if with_cpu:
        from oracle import refbind as R

        doms, conns, cbc = star3d(32)
        rng = np.random.default_rng(SEED + 2)
        rhs = [rng.standard_normal(d[:3]) for d in doms]
        small = capi.Composite3D(doms, conns, cbc, 20, 1e-10, 100)
        got = [r.copy() for r in rhs]
        small.solve(got)
        t0 = time.perf_counter()
        ref = R.Concat3DCase([d[0] for d in doms], [d[1] for d in doms], [d[2] for d in doms],
                             [d[0] * d[3] for d in doms], [d[1] * d[4] for d in doms], [d[2] * d[5] for d in doms],
                             conns, cbc, 20, 1e-10, 100)
        construct = time.perf_counter() - t0
        refout, sec = ref.solve(rhs)
        num = sum(float(((a - b) ** 2).sum()) for a, b in zip(got, refout))
        den = sum(float((b ** 2).sum()) for b in refout)
        c3d["reference_32"] = {"what": "the same star at 32^3 per box: the reference's ConcatPoissonSolver3D "
                                       "(oracle/_ref) on the host cores against this solver",
                               "cpu_solves_per_s": 1.0 / sec, "cpu_construct_s": construct,
                               "rel_l2_vs_reference": (num / den) ** 0.5, "cores": os.cpu_count()}
    out["composite3d"] = c3d
    torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------------------------------------------
# --probe: one kernel family or solve on synthetic data, for timing and for ncu captures
# ------------------------------------------------------------------------------------------------
PROBE_USAGE = """python bench.py --probe transform --family DD --n 2048 [--dtype f64|f32] [--inverse] [--launches K]
    python bench.py --probe rect --n 2048 --bc 0 0 0 0 [--dtype f32]
    python bench.py --probe composite --n 2048 [--form f64|f64ir|f32ir|mixedir] [--launches K]
    python bench.py --probe batch --problems 512 [--precision f64|f32] [--steps S] [--launches K]

Prints the average device time (CUDA events, after warm-up) and the algorithmic bandwidth (2*N*s bytes per
transform launch, 6*N*s per rectangle solve). With --launches 1 the kernel runs once; the composite and batch
modes then print how many library kernels ran before the final call, so that `ncu -k regex:^k_ -s <that
number>` captures exactly the final call."""
FAMILIES = {"DD": (0, 0), "NN": (1, 1), "ND": (1, 0), "DN": (0, 1), "PP": (2, 2)}


def probe_main(argv):
    import torch

    from focalors_poisson_b200 import capi
    from focalors_poisson_b200 import workloads as W

    ap = argparse.ArgumentParser(usage=PROBE_USAGE)
    ap.add_argument("what", choices=["transform", "rect", "composite", "batch"])
    ap.add_argument("--form", default="f64", choices=["f64", "f64ir", "f32ir", "mixedir"])
    ap.add_argument("--problems", type=int, default=512)
    ap.add_argument("--precision", default="f64", choices=["f64", "f32"])
    ap.add_argument("--steps", type=int, default=0)
    ap.add_argument("--family", default="DD", choices=list(FAMILIES))
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--rows", type=int, default=0, help="rows (default n)")
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--inverse", action="store_true")
    ap.add_argument("--bc", type=int, nargs=4, default=[0, 0, 0, 0])
    ap.add_argument("--launches", type=int, default=20)
    args = ap.parse_args(argv)

    def timed(fn, refill=None):
        for _ in range(3):
            if refill:
                refill()
            fn()
        torch.cuda.synchronize()
        if args.launches <= 1:
            if refill:
                refill()
            torch.cuda.synchronize()
            print(f"library launches before the final call: {capi.lib().fp_launch_count()}")
            fn()
            torch.cuda.synchronize()
            return None
        tot = 0.0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(args.launches):
            if refill:
                refill()
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / args.launches

    if args.what in ("transform", "rect"):
        dt = torch.float64 if args.dtype == "f64" else torch.float32
        rows = args.rows or args.n
        x = torch.randn(rows, args.n, dtype=dt, device="cuda")
        if args.what == "transform":
            bn, bp = FAMILIES[args.family]
            fn = lambda: capi.transform(bn, bp, x, inverse=args.inverse, out=x)  # noqa: E731
            nbytes = 2 * rows * args.n * x.element_size()
            label = f"transform {args.family} {'inv' if args.inverse else 'fwd'} {rows}x{args.n} {args.dtype}"
        else:
            r = capi.Rect(rows, args.n, 1.0 / rows, 1.0 / args.n, args.bc,
                          precision=capi.FP_F64 if args.dtype == "f64" else capi.FP_F32)
            fn = lambda: r.solve(x)  # noqa: E731
            nbytes = 6 * rows * args.n * x.element_size()
            label = f"rect solve bc={tuple(args.bc)} {rows}x{args.n} {args.dtype}"
        ms = timed(fn)
        print(f"{label}: " + ("launched once" if ms is None else
                              f"{ms * 1e3:.1f} us, {nbytes / ms / 1e6:.1f} GB/s algorithmic"))
        return
    if args.what == "composite":
        g = W.cross(args.n, neumann_tips=True)
        solver = capi.Composite(g, 20, 1e-14, 100)
        pristine = [torch.tensor(r, device="cuda") for r in W.gaussian_rhs(g, SEED)]
        work = [torch.empty_like(p) for p in pristine]
        if args.form == "f64":
            fn = lambda: solver.solve(work)  # noqa: E731
        else:
            fn = lambda: solver.solve_ir(work, rel_tol=IR_REL_TOL, max_refine=10, inner=INNER[args.form])  # noqa: E731
        label = f"composite cross 5x{args.n}^2 {args.form}"
    else:
        probs, rhs = W.batched_uneven(args.problems, SEED)
        pristine = [torch.tensor(x, device="cuda") for r in rhs for x in r]
        work = [torch.empty_like(p) for p in pristine]
        b = capi.Batch(probs, precision=args.precision)
        fn = lambda: b.solve(work, steps=args.steps, graph=True)  # noqa: E731
        label = f"batch {args.problems} problems {args.precision} steps={args.steps}"

    def refill():
        for w, p in zip(work, pristine):
            w.copy_(p)

    ms = timed(fn, refill)
    extra = "" if args.what != "batch" or ms is None else f", {args.problems / ms * 1e3:.1f} solves/s"
    print(f"{label}: " + ("launched once" if ms is None else f"{ms:.3f} ms{extra}"))


# ------------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------------
def main():
    if len(sys.argv) > 1 and sys.argv[1] == "--probe":
        return probe_main(sys.argv[2:])
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-uneven section")
    ap.add_argument("--no-large", action="store_true", help="skip the 9 x 4096^2 tree section (setup ~2 min)")
    ap.add_argument("--no-3d", action="store_true", help="skip the 3D rectangle and composite section")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.warmup < 3:
        args.warmup = 3

    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from focalors_poisson_b200 import capi
    from focalors_poisson_b200 import workloads as W

    g = W.cross(N_CELLS, neumann_tips=True)
    rhs = W.gaussian_rhs(g, SEED + rank)
    t_setup = time.perf_counter()
    solver = capi.Composite(g, *GMRES)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup
    dev = torch.device("cuda", local)
    pristine = [torch.tensor(r, device=dev) for r in rhs]
    work = [torch.empty_like(p) for p in pristine]
    stream = torch.cuda.current_stream()
    lib = capi.lib()

    def barrier():
        if dist is not None:
            dist.barrier()

    def run_form(form):
        def step():
            for w, p in zip(work, pristine):
                w.copy_(p)
            if form == "f64":
                return solver.solve(work)
            return solver.solve_ir(work, rel_tol=IR_REL_TOL, max_refine=10, inner=INNER[form])

        infos = [step() for _ in range(args.warmup)]
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        barrier()
        torch.cuda.synchronize()
        clocks.start()
        launches0 = lib.fp_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            infos.append(step())
        e1.record(stream)
        torch.cuda.synchronize()
        launches = lib.fp_launch_count() - launches0
        barrier()
        clk = clocks.stop()
        ms = max_over_ranks(e0.elapsed_time(e1), dist, dev)
        return {"ms": ms, "value": replica_value(args.steps, world, ms), "launches": int(launches), "clocks": clk,
                "infos": infos[-args.steps:], "solution": [w.clone() for w in work]}

    forms_run = ("f64", "f64ir", "f32ir", "mixedir")
    res = {form: run_form(form) for form in forms_run}
    # accuracy arbiter: the FP64 residual of the composite operator and, as "exact", the refinement solve
    # driven to |correction| <= 1e-14 |u| (the single FP64 solve has a round-off floor ~ eps * cond(A))
    for w, p in zip(work, pristine):
        w.copy_(p)
    solver.solve_ir(work, rel_tol=1e-14, max_refine=20, inner="f64")
    exact = [w.clone() for w in work]

    def rel(a_list, b_list):
        num = sum(float(((a - b) ** 2).sum()) for a, b in zip(a_list, b_list))
        den = sum(float((b ** 2).sum()) for b in b_list)
        return (num / den) ** 0.5

    accuracy = {form: {"rel_l2_vs_exact": rel(res[form]["solution"], exact),
                       "rel_residual": solver.residual(res[form]["solution"], pristine)} for form in forms_run}
    exact_residual = solver.residual(exact, pristine)
    keep_host = rank == 0 and world == 1 and not args.no_cpu_baseline
    # headline form: the fastest whose answer is within 1e-10 relative L2 of the exact discrete solution
    ok = [f for f in forms_run if accuracy[f]["rel_l2_vs_exact"] <= 1e-10]
    head = max(ok, key=lambda f: res[f]["value"]) if ok else "f64"
    head_solution = res[head]["solution"]
    for form in forms_run:
        if keep_host:  # compared with the reference's answer after the GPU sections
            res[form]["host"] = [x.cpu().numpy() for x in res[form]["solution"]]
        del res[form]["solution"]
    del exact
    r = res[head]

    # e2e: the headline form through the C ABI with host buffers, the copies inside the timed region.
    # Headline: a stream of independent solves through fp_composite_solve_async (each call copies its own
    # right-hand sides in from page-locked host memory and its solution out; consecutive calls overlap their
    # copies with the neighbouring solves), timed from the first call to the wait that ends the last one.
    # Beside it: the synchronous in-place call (copy in, solve, copy out, return) timed per call.
    host = [torch.empty(p.shape, dtype=torch.float64, pin_memory=True) for p in pristine]
    host_np = [h.numpy() for h in host]
    for h, rr in zip(host_np, rhs):
        h[...] = rr
    outs = [[torch.empty(p.shape, dtype=torch.float64, pin_memory=True) for p in pristine] for _ in range(2)]
    for k in range(2):  # warm-up of the pipeline (slots, copy streams, graphs)
        solver.solve_async(host, outs[k], form=head, rel_tol=IR_REL_TOL, max_refine=10)
    solver.wait()
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        solver.solve_async(host, outs[k % 2], form=head, rel_tol=IR_REL_TOL, max_refine=10)
    solver.wait()
    e2e_t = max_over_ranks(time.perf_counter() - t0, dist, dev)
    e2e_check = rel([o.to(dev) for o in outs[(args.steps - 1) % 2]], head_solution)
    del head_solution
    sync_times = []
    for it in range(args.steps + 1):
        for h, rr in zip(host_np, rhs):
            h[...] = rr
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        if head == "f64":
            solver.solve(host_np)  # synchronous host-pointer call
        else:
            solver.solve_ir(host_np, rel_tol=IR_REL_TOL, max_refine=10, inner=INNER[head])
        if it > 0:
            sync_times.append(time.perf_counter() - t1)
    sync_t = max_over_ranks(sum(sync_times), dist, dev)
    field_bytes = sum(int(p.numel()) * 8 for p in pristine)
    # the host link alone: the same bytes copied host -> device and back from the pinned buffers, timed
    # with events, one direction after the other and both at once (a call that copies, solves, copies back
    # is bounded by 1 / (copies + solve); overlapped calls by 1 / max(both copies at once, solve))
    c0, c1, c2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    for _ in range(2):
        c0.record(stream)
        for w, h in zip(work, host):
            w.copy_(h, non_blocking=True)
        c1.record(stream)
        for w, h in zip(work, host):
            h.copy_(w, non_blocking=True)
        c2.record(stream)
        torch.cuda.synchronize()
    h2d_ms, d2h_ms = c0.elapsed_time(c1), c1.elapsed_time(c2)
    # both directions at once, as the overlapped calls run them (one copy stream each way)
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    back = [torch.empty(p.shape, dtype=torch.float64, pin_memory=True) for p in pristine]
    for _ in range(2):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        with torch.cuda.stream(s_in):
            for w, h in zip(work, host):
                w.copy_(h, non_blocking=True)
        with torch.cuda.stream(s_out):
            for p, b in zip(pristine, back):
                b.copy_(p, non_blocking=True)
        torch.cuda.synchronize()
        duplex_ms = (time.perf_counter() - t1) * 1e3
    del back
    solve_ms = r["ms"] / args.steps
    e2e = {"value": args.steps * world / e2e_t, "unit": "solves/s", "h2d_bytes_per_step": field_bytes,
           "d2h_bytes_per_step": field_bytes, "form": head,
           "api": "fp_composite_solve_async per step (host buffers, page-locked), fp_composite_wait after the last",
           "rel_l2_vs_device_solution": e2e_check,
           "sync_call": {"value": args.steps * world / sync_t, "unit": "solves/s",
                         "api": "fp_composite_solve_f32ir / _f64 with host pointers (copy in, solve, copy out)"},
           "host_link": {"h2d_ms": h2d_ms, "d2h_ms": d2h_ms, "h2d_gbs": field_bytes / h2d_ms / 1e6,
                         "d2h_gbs": field_bytes / d2h_ms / 1e6,
                         "serial_bound_solves_per_s": 1e3 / (h2d_ms + d2h_ms + solve_ms),
                         "duplex_ms": duplex_ms,
                         "overlap_bound_solves_per_s": 1e3 / max(duplex_ms, solve_ms)}}
    ms, value, launches, clk, infos = r["ms"], r["value"], r["launches"], r["clocks"], r["infos"]
    t_max = ms

    # roofline of the dominant kernel: the DD y-transform of one 2048^2 FP64 subdomain, launched in turn on
    # five fields (168 MB together, more than the 126 MB L2), so that every launch reads its input from HBM
    xs = [torch.randn(N_CELLS, N_CELLS, dtype=torch.float64, device=dev) for _ in range(5)]
    for x in xs:
        capi.transform(0, 0, x, out=x)
    torch.cuda.synchronize()
    reps = 20
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k0.record(stream)
    for i in range(reps):
        capi.transform(0, 0, xs[i % 5], out=xs[i % 5])
    k1.record(stream)
    torch.cuda.synchronize()
    t_kernel = k0.elapsed_time(k1) / reps / 1e3
    bytes_launch = 2 * N_CELLS * N_CELLS * 8
    peak, peak_kind = measured_peaks()
    achieved = bytes_launch / t_kernel / 1e9
    roofline = {"kernel": "k_xform_rc<double, DD, 0, double, double, ACC=false, M=4096> (register engine, plan by value) "
                          "(one run of 2048 rows of 2048, in place, five fields in turn; the instantiation the FP64 "
                          "solve launches)", "bound": "hbm",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} hbm_gbs", "traffic": DD_TRAFFIC_BYTES,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch "
                                  "(profiles/k_xform_rc_DD_2048x2048_f64.md)",
                "algorithmic_bytes_per_launch": bytes_launch, "avg_launch_ms": t_kernel * 1e3}
    # the chase (the solve's other kernel family): the x-direction tridiagonal solves of one 2048^2 FP64
    # subdomain, fp_rect_chase_f64 (local chunk sweeps, separator scan, correction), 2*N*8 bytes algorithmic
    rect = capi.Rect(N_CELLS, N_CELLS, 1.0 / N_CELLS, 1.0 / N_CELLS, (0, 0, 0, 0))
    for x in xs:
        rect.chase(x)
    torch.cuda.synchronize()
    k0.record(stream)
    for i in range(reps):
        rect.chase(xs[i % 5])
    k1.record(stream)
    torch.cuda.synchronize()
    t_chase = k0.elapsed_time(k1) / reps / 1e3
    ach_chase = bytes_launch / t_chase / 1e9
    roofline_chase = {"kernel": "k_chase_local + k_chase_reduced + k_chase_correct (2048x2048, FP64, one chase)",
                      "bound": "hbm", "achieved": ach_chase, "peak": peak, "unit": "GB/s", "frac": ach_chase / peak,
                      "peak_source": f"{peak_kind} hbm_gbs", "algorithmic_bytes_per_launch": bytes_launch,
                      "avg_launch_ms": t_chase * 1e3,
                      "traffic_note": "the chase reads and writes the field twice (chunk sweeps, then the "
                                      "correction): 4*N*8 bytes of DRAM traffic for 2*N*8 algorithmic"}
    del rect, xs

    forms = {}
    for form, rr in res.items():
        it = rr["infos"]
        forms[form] = {"value": rr["value"], "ms_per_step": rr["ms"] / args.steps, "gpu_launches": rr["launches"],
                       "gmres_or_refine_steps_per_solve": statistics.mean(
                           [i["iterations"] if form == "f64" else i["refinements"] for i in it]) if it else None}
    for form in forms:
        forms[form].update(accuracy[form])
    forms["exact_rel_residual"] = exact_residual
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"f64": "f64", "f64ir": "f64", "f32ir": "f32 transforms + f64 refinement",
                  "mixedir": "f64 solve + f32 corrections, f64 refinement"}[head],
        "data": "synthetic", "config": workload_config(),
        "precision_form": {"f64": "FP64 drop-in (interface-preconditioned Schur GMRES)",
                           "f64ir": "FP64 solves + FP64 iterative refinement",
                           "f32ir": "FP32 transforms + FP64 iterative refinement",
                           "mixedir": "FP64 solve, then FP32-storage corrections in FP64 iterative refinement"}[head],
        "forms": forms, "clocks": clk, "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline,
        "roofline_chase": roofline_chase,
        "setup": {"seconds": setup_s, "what": "capi.Composite creation for this workload (plans, chase tables, "
                                               "closed-form interface operators and the reduced-system inverse of "
                                               "the spectral path; on the Schur GMRES path the Schur matrices and "
                                               "interface inverses), wall clock"},
    }
    if keep_host:
        from oracle import refsolve as RS

        line["cpu_baseline"], ref = cpu_reference_leg(g, rhs)
        if ref is not None:
            for form in forms_run:
                forms[form]["rel_l2_vs_reference"] = RS.rel_l2(res[form]["host"], ref["refined"])
                forms[form]["rel_l2_vs_reference_plain"] = RS.rel_l2(res[form]["host"], ref["plain"])
            line["rel_l2_vs_reference"] = forms[head]["rel_l2_vs_reference"]
            line["reference_answer"] = {
                "what": "the reference's own solve() of this workload (oracle/_ref), refined once by the same "
                        "solver; rel_l2_vs_reference compares with the refined answer, "
                        "rel_l2_vs_reference_plain with the single solve",
                "rel_residual_plain": ref["rel_residual"],
                "plain_vs_refined": ref["rel_correction"],
                "plain_vs_refined_note": "the single FP64 solve's own round-off (~eps * cond(A)): the floor any "
                                         "single FP64 solve of this workload sits at, ours included",
                "solve_seconds": ref["seconds"], "refine_seconds": ref["refine_seconds"]}
        for form in forms_run:
            res[form].pop("host", None)
    if not args.no_batched:
        del solver, pristine, work
        torch.cuda.empty_cache()
        line["batched_uneven"] = batched_section(args, dev, rank, world, dist)
    if not args.no_large and world == 1:
        line["large_tree"] = large_section(args, dev)
    if not args.no_3d and world == 1:
        line["three_d"] = threed_section(args, dev, with_cpu=rank == 0 and not args.no_cpu_baseline)
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
