"""Run one piece of the hot path on seeded inputs, for timing or for a profiler.

    python lhl.jl_b200/profile_case.py --n 2048 --what reduce --reps 3
    python lhl.jl_b200/profile_case.py --n 2048 --what chain --shifts 64 --reps 3

--what reduce: lhl_reduce (balance + reduction + Ht/perm) of an N(0,1) matrix.
--precision mixed: the mixed form's FP32 reduction (workspace LHL_PREC_MIXED).
--what chain:  one reduction, then per repetition the batched shift LUs, the solves and one
               refinement step for `--shifts` shifts (1, -g) with one right-hand side each.
Prints the CUDA-event time of each repetition."""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

import lhl_gpu as G  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--what", default="reduce", choices=["reduce", "chain"])
    ap.add_argument("--shifts", type=int, default=64)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--complex-j", action="store_true", help="a complex J (LHLWorkspace{ComplexF64})")
    ap.add_argument("--probes", action="store_true", help="record and print the reduction's device timers")
    args = ap.parse_args()
    n = args.n
    rng = np.random.default_rng(args.seed)
    Jh = rng.standard_normal((n, n))
    if args.complex_j:
        Jh = Jh + 1j * rng.standard_normal((n, n))
    J = torch.as_tensor(np.asfortranarray(Jh)).cuda()
    if args.complex_j:
        ws = G.LHLWorkspace(n, dtype=torch.complex128)
    else:
        ws = G.LHLWorkspace(n, G.LHL_PREC_MIXED if args.precision == "mixed" else G.LHL_PREC_FP64)
    if args.probes:
        ws.set_probes(True)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    if args.what == "reduce":
        for r in range(args.reps):
            a, b = ev(), ev()
            a.record()
            G.lhl_reduce_(ws, J, True)
            b.record()
            torch.cuda.synchronize()
            ws.check()
            form = "complex-J" if args.complex_j else args.precision
            line = f"reduce n={n} {form} rep={r} ms={a.elapsed_time(b):.3f}"
            if args.precision == "mixed" and args.probes:  # CTA 0's sub-phase times, summed over the steps (ms)
                p = [int(v) for v in ws.probe_ns()]
                names = ("wait+choice", "loads", "dots+column", "publish", "rowop", "poll", "dots")
                line += " " + " ".join(f"{nm}={p[i] / 1e6:.2f}" for i, nm in enumerate(names))
            if args.precision == "fp64" and args.probes and not args.complex_j:  # plain reduction's phase timers (ms)
                line += " " + " ".join(f"{k}={v / 1e6:.2f}" for k, v in ws.phase_ns().items())
                # finer probes (reduce.cu's tprobe slots): 0-4 the row phase of the last CTA with
                # rows (start, partials staged, row work, candidate published, barrier), 5 and 6 CTA
                # 0's pivot combine and step table, 7 CTA 1's GEMV tasks, 8 CTA 0's phase A to its end
                p = [int(v) for v in ws.probe_ns()]
                line += " probes=" + ",".join(f"{p[i] / 1e6:.2f}" for i in range(9))
            print(line, flush=True)
        return
    S = args.shifts
    G.lhl_reduce_(ws, J, True)
    sh = G.LHLShift(n, S, complex=args.complex_j)
    sig = torch.ones(S, dtype=torch.float64, device="cuda")
    tau = torch.as_tensor(-(10.0 ** rng.uniform(-4, -1, S))).cuda()
    Bh = rng.standard_normal((n, S))
    if args.complex_j:
        sig, tau = sig.to(torch.complex128), tau.to(torch.complex128)
        Bh = Bh + 1j * rng.standard_normal((n, S))
    B = torch.as_tensor(np.asfortranarray(Bh)).cuda()
    X = torch.empty_like(B)
    for r in range(args.reps):
        a, b = ev(), ev()
        a.record()
        G.lhl_shift_batched_(sh, ws, sig, tau)
        X.copy_(B)
        G.lhl_ldiv_(X, sh, ws)
        G.lhl_refine_(X, J, B, sh, ws, 1)
        b.record()
        torch.cuda.synchronize()
        print(f"chain n={n} shifts={S} rep={r} ms={a.elapsed_time(b):.3f}", flush=True)


if __name__ == "__main__":
    main()
