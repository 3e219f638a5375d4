"""Measure one of the path's configurations end to end on one GPU, both forms.

    python lhl.jl_b200/run_config.py --config c1|c3|c5 [--reps 2] [--chunk 16]

One step = the reduction, every shift LU, every solve and refinement until each solve is at
relative residual <= 1e-10 (plain form: fixed-point lhl_refine_tol; mixed form: GMRES-IR for
real shifts, fixed-point for complex ones unless --gmres-complex).  Shifts are processed in chunks of `--chunk`
(config 5's complex Gt is 1.07 GB per shift at n = 8192).  Inputs are the seeded synthetic
configurations of lhl_gpu.configs; device-resident; CUDA-event times; one JSON line per form.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import lhl_gpu as G  # noqa: E402
from lhl_gpu import configs  # noqa: E402

TOL = 1e-10


def load(name):
    if name == "c1":
        return configs.config1()
    if name == "c3":
        return configs.config3()
    if name == "c5":
        c = configs.config5()
        g = c["rng"]
        n, R, S = c["n"], c["nrhs"], len(c["sigma"])
        c["B"] = np.asfortranarray(g.standard_normal((n, S * R)) + 1j * g.standard_normal((n, S * R)))
        c["R"] = R
        return c
    raise SystemExit(f"unknown config {name}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", required=True, choices=["c1", "c3", "c5"])
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--chunk", type=int, default=16)
    ap.add_argument("--forms", default="plain,mixed")
    ap.add_argument("--steps", type=int, default=4, help="plain form: fixed-point steps at most")
    ap.add_argument("--cycles", type=int, default=4, help="mixed form: GMRES-IR cycles at most")
    ap.add_argument("--restart", type=int, default=3, help="mixed form: Arnoldi steps per cycle")
    ap.add_argument("--gmres-complex", action="store_true", help="mixed form, complex shifts: GMRES-IR too")
    args = ap.parse_args()
    c = load(args.config)
    n = c["n"]
    cplx = np.iscomplexobj(c["sigma"])
    S = len(c["sigma"])
    R = c.get("R", 1)
    Jd = torch.as_tensor(c["J"]).cuda()
    Bd = torch.as_tensor(c["B"]).cuda()
    sig = torch.as_tensor(np.asarray(c["sigma"])).cuda()
    tau = torch.as_tensor(np.asarray(c["tau"]).astype(np.asarray(c["sigma"]).dtype)).cuda()
    chunk = min(args.chunk, S)
    stream = torch.cuda.current_stream()
    for form in args.forms.split(","):
        prec = G.LHL_PREC_MIXED if form == "mixed" else G.LHL_PREC_FP64
        ws = G.LHLWorkspace(n, prec, shift_complex=cplx)
        sh = G.LHLShift(n, chunk, complex=cplx)
        dt = torch.complex128 if cplx else torch.float64
        X = torch.empty((chunk * R, n), dtype=dt, device="cuda").t()
        Rs = torch.empty((chunk * R, n), dtype=dt, device="cuda")
        res_all = torch.empty(S * R, dtype=torch.float64, device="cuda")
        # GMRES-IR pays where a few columns converge slowly (config 2's mixed form).  Where every
        # column converges in a few fixed-point steps and solves are costly (config 5's complex
        # shifts), its extra solve per cycle loses: 436 against 571 solves/s there.
        use_gmres = form == "mixed" and not (cplx and not args.gmres_complex)

        def step(times=None):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            ev[0].record(stream)
            G.lhl_reduce_(ws, Jd, True)
            ev[1].record(stream)
            for s0 in range(0, S, chunk):
                cnt = min(chunk, S - s0)
                G.lhl_shift_batched_(sh, ws, sig[s0:s0 + cnt], tau[s0:s0 + cnt])
                Xc = X[:, :cnt * R]
                Bc = Bd[:, s0 * R:(s0 + cnt) * R]
                Xc.copy_(Bc)
                G.lhl_ldiv_(Xc, sh, ws, rhs_per_shift=R)
                if use_gmres:
                    G.lhl_refine_gmres_(Xc, Jd, Bc, sh, ws, tol=TOL, max_cycles=args.cycles, restart=args.restart, rhs_per_shift=R,
                                        R=Rs, res=res_all[s0 * R:(s0 + cnt) * R])
                else:
                    G.lhl_refine_tol_(Xc, Jd, Bc, sh, ws, tol=TOL, max_steps=16 if form == "mixed" else args.steps,
                                      rhs_per_shift=R, R=Rs, res=res_all[s0 * R:(s0 + cnt) * R])
            ev[2].record(stream)
            torch.cuda.synchronize()
            ws.check()
            if times is not None:
                times.append((ev[0].elapsed_time(ev[2]), ev[0].elapsed_time(ev[1])))

        step()
        times = []
        for _ in range(args.reps):
            step(times)
        res = res_all.cpu().numpy()
        ms = float(np.mean([t[0] for t in times]))
        red = float(np.mean([t[1] for t in times]))
        print(json.dumps({"config": args.config, "form": form, "n": n, "shifts": S, "rhs_per_shift": R,
                          "complex_shifts": bool(cplx), "solves_per_s": S * R / (ms * 1e-3), "ms_per_step": ms,
                          "reduce_ms": red, "chain_ms": ms - red, "max_rel_residual": float(res.max()),
                          "all_at_tol": bool((res <= TOL).all()), "n_at_tol": int((res <= TOL).sum()),
                          "median_rel_residual": float(np.median(res)),
                          "refinement": (f"GMRES-IR, GMRES({args.restart}) x {args.cycles}" if use_gmres
                                         else f"fixed-point, {16 if form == 'mixed' else args.steps} steps at most")}),
              flush=True)
        del ws, sh, X, Rs
        torch.cuda.empty_cache()


if __name__ == "__main__":
    main()
