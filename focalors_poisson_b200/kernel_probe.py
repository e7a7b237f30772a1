"""Times (or, under a profiler, just launches) individual device kernels of libfpb200 on synthetic data.

    python -m focalors_poisson_b200.kernel_probe transform --family DD --n 2048 [--dtype f64] [--inverse]
    python -m focalors_poisson_b200.kernel_probe rect --n 2048 --bc 0 0 0 0 [--dtype f32]
    python -m focalors_poisson_b200.kernel_probe transform ... --launches 1     # one launch, for ncu -c 1
    python -m focalors_poisson_b200.kernel_probe composite --n 2048 [--form f64|f64ir|f32ir|mixedir] [--launches K]
    python -m focalors_poisson_b200.kernel_probe batch --problems 512 [--precision f64|f32] [--steps S]

With --launches 1 the composite and batch modes print how many library kernels ran before the final call,
so that `ncu -k regex:^k_ -s <that number>` captures exactly the final call.

Prints one line per measurement: average device time (CUDA events, after 3 warm-up launches) and the
algorithmic bandwidth (2*N*s bytes per transform launch, 6*N*s per rectangle solve).
"""
from __future__ import annotations

import argparse

FAMILIES = {"DD": (0, 0), "NN": (1, 1), "ND": (1, 0), "DN": (0, 1), "PP": (2, 2)}


def main():
    import torch

    from . import capi

    ap = argparse.ArgumentParser()
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
    args = ap.parse_args()
    if args.what == "composite":
        return composite(args)
    if args.what == "batch":
        return batch(args)
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
    if args.launches <= 1:
        fn()
        torch.cuda.synchronize()
        print(f"{label}: launched once")
        return
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.launches):
        fn()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.launches
    print(f"{label}: {ms * 1e3:.1f} us, {nbytes / ms / 1e6:.1f} GB/s algorithmic")


def _time(fn, refill, launches):
    import torch

    for _ in range(2):
        refill()
        fn()
    torch.cuda.synchronize()
    if launches <= 1:
        from . import capi

        refill()
        torch.cuda.synchronize()
        print(f"library launches before the final call: {capi.lib().fp_launch_count()}")
        fn()
        torch.cuda.synchronize()
        return None
    tot = 0.0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(launches):
        refill()
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
    return tot / launches


def composite(args):
    """One composite solve of the cross 5 x n^2 with Neumann arm tips (seeded Gaussian RHS)."""
    import torch

    from . import capi
    from . import workloads as W

    g = W.cross(args.n, neumann_tips=True)
    solver = capi.Composite(g, 20, 1e-14, 100)
    pristine = [torch.tensor(r, device="cuda") for r in W.gaussian_rhs(g, 2024)]
    work = [torch.empty_like(p) for p in pristine]

    def refill():
        for w, p in zip(work, pristine):
            w.copy_(p)

    if args.form == "f64":
        fn = lambda: solver.solve(work)  # noqa: E731
    else:
        inner = {"f64ir": "f64", "f32ir": "f32", "mixedir": "mixed"}[args.form]
        fn = lambda: solver.solve_ir(work, rel_tol=1e-11, max_refine=10, inner=inner)  # noqa: E731
    ms = _time(fn, refill, args.launches)
    print(f"composite cross 5x{args.n}^2 {args.form}: " + ("launched once" if ms is None else f"{ms:.3f} ms"))


def batch(args):
    """The batched-uneven workload (first `problems` of the 512 seeded L/T problems) in one graph."""
    import torch

    from . import capi
    from . import workloads as W

    probs, rhs = W.batched_uneven(args.problems)
    pristine = [torch.tensor(x, device="cuda") for r in rhs for x in r]
    work = [torch.empty_like(p) for p in pristine]
    b = capi.Batch(probs, precision=args.precision)

    def refill():
        for w, p in zip(work, pristine):
            w.copy_(p)

    ms = _time(lambda: b.solve(work, steps=args.steps, graph=True), refill, args.launches)
    cells = sum(int(p.numel()) for p in pristine)
    print(f"batch {args.problems} problems ({cells} cells) {args.precision} steps={args.steps}: "
          + ("launched once" if ms is None else f"{ms:.3f} ms, {args.problems / ms * 1e3:.1f} solves/s"))


if __name__ == "__main__":
    main()
