"""Benchmark: shifted solves per second on one B200 (LHLFactorization.jl's hot path).

Workload (config 2): J 2048x2048 FP64 N(0,1); 64 shifts (1, -g), g log-uniform in
[1e-4, 1e-1]; one N(0,1) right-hand side per shift.  One step = the whole path on one
batch: reduction J = Z H Z^-1 (balance + blocked ELMHES), 64 shift LUs, 64 solves and one
refinement step each (every solve ends at <= 1e-10 relative residual; checked after the
timed region).  value = 64 solves / step time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs independent replicas, one per GPU (the reduction of one J does not shard);
value is the aggregate.  --impl reference times the CPU restatement of the reference
algorithm (the oracle, all host threads) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "lhl.jl_b200")
for _p in (REPO, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "shifted solves/sec at 1e-10 rel. residual: mixed/batched vs plain FP64, 1 B200"
UNIT = "solves/s"
L2_FLUSH_BYTES = 256 << 20


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                parts = [x.strip() for x in out.stdout.strip().split(",")]
                if len(parts) == 6:
                    self.samples.append(parts)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[2 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_setup(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_reference_run(cfg, steps, warmup, threads_note):
    """The oracle (CPU restatement) on one full step of the workload; returns seconds per step."""
    from oracle import oracle as O
    times = []
    X = None
    for it in range(warmup + steps):
        t0 = time.perf_counter()
        R = O.reduce(cfg["J"])
        X, info = O.shift_solve_batch(R, cfg["J"], cfg["sigma"], cfg["tau"], cfg["B"], steps=cfg["steps"])
        t1 = time.perf_counter()
        if it >= warmup:
            times.append(t1 - t0)
    return times, X


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-baseline-steps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world, rank, local = dist_setup(args.gpus)

    from lhl_gpu import configs
    cfg = configs.config2()
    n, S = cfg["n"], len(cfg["sigma"])
    config = {"workload": "c2: J 2048x2048 FP64 N(0,1), 64 shifts (1,-g) g log-uniform [1e-4,1e-1], 1 RHS/shift, "
                          "reduction + shift LU + ldiv + 1 refinement per step",
              "n": n, "shifts": S, "rhs_per_shift": 1, "refine_steps": cfg["steps"], "form": "plain FP64",
              "l2": "flushed between timed steps (256 MiB write)", "replicas": world}

    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import oracle as O
        threads = O.num_threads()
        times, _ = cpu_reference_run(cfg, max(args.steps, 1), 0, threads)
        sec = float(np.mean(times))
        val = S / sec
        line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
                "steps": len(times), "warmup": 0, "ms_per_step": sec * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (numpy PCG64 seeds 2,3,4)",
                "config": config,
                "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                                 "sample": f"{len(times)} full step(s) of the workload: oracle C restatement, OpenMP"},
                "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    import lhl_gpu as G
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        pg = dist
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()

    # ---- device-resident inputs ----
    Jd = torch.as_tensor(cfg["J"]).to(dev)              # column-major (strides 1, n)
    Bd = torch.as_tensor(cfg["B"]).to(dev)
    sig = torch.as_tensor(cfg["sigma"]).to(dev)
    tau = torch.as_tensor(cfg["tau"]).to(dev)
    X = torch.empty_like(Bd)
    ws = G.LHLWorkspace(n)
    sh = G.LHLShift(n, S)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def step():
        G.lhl_reduce_(ws, Jd, True)
        G.lhl_shift_batched_(sh, ws, sig, tau)
        X.copy_(Bd)
        G.lhl_ldiv_(X, sh, ws)
        G.lhl_refine_(X, Jd, Bd, sh, ws, cfg["steps"])

    launches_per_step = 4 + 1 + 1 + 3 * cfg["steps"]  # reduce(init, coop, ht, perm), shift, ldiv, refine
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    ws.check()

    # ---- timed region: K steps, per-step events, L2 flushed between steps ----
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            evs[k][0].record(stream)
            step()
            evs[k][1].record(stream)
        torch.cuda.synchronize()
    if pg:
        pg.barrier()
    ms = [a.elapsed_time(b) for a, b in evs]
    ms_step = float(np.mean(ms))
    ws.check()

    # ---- accuracy of the timed work (outside the timed region) ----
    res = G.residual_norms(sh, Jd, Bd, X).cpu().numpy()
    assert (res <= 1e-10).all(), f"residual above 1e-10: {res.max()}"

    # ---- dominant kernel: the reduction, timed alone (events on the launching stream) ----
    red_ms = []
    for k in range(max(3, min(args.steps, 10))):
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        G.lhl_reduce_(ws, Jd, True)
        b.record(stream)
        torch.cuda.synchronize()
        red_ms.append(a.elapsed_time(b))
    phase = {}
    for name, fn in (("shift", lambda: G.lhl_shift_batched_(sh, ws, sig, tau)),
                     ("ldiv", lambda: G.lhl_ldiv_(X, sh, ws)),
                     ("refine", lambda: G.lhl_refine_(X, Jd, Bd, sh, ws, cfg["steps"]))):
        tt = []
        for k in range(3):
            flush.fill_(float(k))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            tt.append(a.elapsed_time(b))
        phase[name] = float(np.mean(tt))
    red = float(np.mean(red_ms))
    phase["reduce"] = red
    phase["reduce_inside_ms"] = {k: v / 1e6 for k, v in ws.phase_ns().items()}
    alg_bytes = 8.0 * (n ** 3) / 3.0 + 16.0 * n * n   # GEMV stream (8 n^3/3) + J in, Ht/L out
    peak, peak_kind = peaks()
    achieved = alg_bytes / (red * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(REPO, "profiles", "reduce_kernel_c2_n2048.md")
    if os.path.exists(tp):
        for line in open(tp):
            if line.startswith("dram_bytes_per_launch:"):
                traffic = float(line.split(":")[1])

    # ---- end to end through the public API: host buffers, copies inside the timed region ----
    def pinned_colmajor(a):
        t = torch.empty((a.shape[1], a.shape[0]), dtype=torch.float64, pin_memory=True).t()
        t.copy_(torch.as_tensor(a))
        return t

    Jh = pinned_colmajor(cfg["J"])
    Bh = pinned_colmajor(cfg["B"])
    sh_h = torch.as_tensor(np.stack([cfg["sigma"], cfg["tau"]])).pin_memory()
    Xh = torch.empty((S, n), dtype=torch.float64, pin_memory=True).t()
    Jd2 = torch.empty_like(Jd)
    Bd2 = torch.empty_like(Bd)
    st2 = torch.empty((2, S), dtype=torch.float64, device=dev)

    def e2e_step():
        Jd2.copy_(Jh, non_blocking=True)
        Bd2.copy_(Bh, non_blocking=True)
        st2.copy_(sh_h, non_blocking=True)
        G.lhl_reduce_(ws, Jd2, True)
        G.lhl_shift_batched_(sh, ws, st2[0], st2[1])
        X.copy_(Bd2)
        G.lhl_ldiv_(X, sh, ws)
        G.lhl_refine_(X, Jd2, Bd2, sh, ws, cfg["steps"])
        Xh.copy_(X, non_blocking=True)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    e_ms = []
    for k in range(args.steps):
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e2e_step()
        b.record(stream)
        torch.cuda.synchronize()
        e_ms.append(a.elapsed_time(b))
    e2e_ms = float(np.mean(e_ms))
    h2d = Jh.numel() * 8 + Bh.numel() * 8 + sh_h.numel() * 8
    d2h = Xh.numel() * 8

    # ---- max over ranks ----
    vals = torch.tensor([ms_step, e2e_ms], dtype=torch.float64, device=dev)
    if pg:
        pg.all_reduce(vals, op=pg.ReduceOp.MAX)
    ms_step, e2e_ms = float(vals[0]), float(vals[1])
    value = world * S / (ms_step * 1e-3)
    e2e_value = world * S / (e2e_ms * 1e-3)

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            from oracle import oracle as O
            times, Xc = cpu_reference_run(cfg, args.cpu_baseline_steps, 0, None)
            sec = float(np.mean(times))
            cpu = {"value": S / sec, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
                   "sample": f"{len(times)} full step(s) (reduction + 64 shift LUs + solves + 1 refinement), "
                             f"oracle C restatement with OpenMP, {sec:.2f} s/step"}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (numpy PCG64 seeds 2,3,4)",
                "config": config,
                "phases_ms": phase, "max_rel_residual": float(res.max()),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                             "kernel": "reduce_kernel (balance + blocked ELMHES, one cooperative launch)",
                             "algorithmic_bytes": alg_bytes},
                "cpu_baseline": cpu,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "ms_per_step": e2e_ms},
                "gpu_launches": launches_per_step * args.steps,
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
