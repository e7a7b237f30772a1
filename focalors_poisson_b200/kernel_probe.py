"""Times (or, under a profiler, just launches) individual device kernels of libfpb200 on synthetic data.

    python -m focalors_poisson_b200.kernel_probe transform --family DD --n 2048 [--dtype f64] [--inverse]
    python -m focalors_poisson_b200.kernel_probe rect --n 2048 --bc 0 0 0 0 [--dtype f32]
    python -m focalors_poisson_b200.kernel_probe transform ... --launches 1     # one launch, for ncu -c 1

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
    ap.add_argument("what", choices=["transform", "rect"])
    ap.add_argument("--family", default="DD", choices=list(FAMILIES))
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--rows", type=int, default=0, help="rows (default n)")
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--inverse", action="store_true")
    ap.add_argument("--bc", type=int, nargs=4, default=[0, 0, 0, 0])
    ap.add_argument("--launches", type=int, default=20)
    args = ap.parse_args()
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


if __name__ == "__main__":
    main()
