"""Benchmark: shifted solves per second on one B200 (LHLFactorization.jl's hot path).

Workload (config 2): J 2048x2048 FP64 N(0,1); 64 shifts (1, -g), g log-uniform in
[1e-4, 1e-1]; one N(0,1) right-hand side per shift.  One step = the whole path on one
batch: reduction J = Z H Z^-1, 64 shift LUs, 64 solves, then FP64 refinement until every
solve is at <= 1e-10 relative residual (lhl_refine_tol; the final residuals are checked
after the timed region).  value = 64 solves / step time of the mixed form (FP32 reduction);
the plain FP64 form (bit-identical to the reference's operation order) is timed the same
way and reported beside it, with the ratio.

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


def max_over_ranks(times_ms, device, dist=None):
    """Every rank's per-step times, reduced to the maximum over ranks (the job is as fast as
    its slowest rank); `dist` is torch.distributed once the process group exists, else None."""
    import torch
    vals = torch.tensor([float(v) for v in times_ms], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(vals, op=dist.ReduceOp.MAX)
    return [float(v) for v in vals]


def whole_job_rate(world, units_per_rank, ms_per_step):
    """Units per second of the whole job: every rank processes units_per_rank per step."""
    return world * units_per_rank / (ms_per_step * 1e-3)


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


def time_events(stream, fn, reps, flush):
    out = []
    for k in range(reps):
        flush.fill_(float(k))
        import torch
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        out.append(a.elapsed_time(b))
    return float(np.mean(out))


def cpu_config_sample(name, shifts_sample):
    """The oracle on a bounded sample of configuration c1, c3 or c5: the full reduction once,
    then `shifts_sample` of its shifts (c1: all three), each with its right-hand sides solved and
    refined by one step.  Returns (seconds for the whole step, scaled from the sample by the
    shift count; solves per step; a description of the sample)."""
    from oracle import oracle as O
    from lhl_gpu import configs
    c = {"c1": configs.config1, "c3": configs.config3, "c5": configs.config5}[name]()
    J, sig, tau = c["J"], np.asarray(c["sigma"]), np.asarray(c["tau"])
    n, S, R = J.shape[0], len(sig), int(c.get("nrhs", 1))
    k = S if name == "c1" else max(1, min(shifts_sample, S))
    t0 = time.perf_counter()
    Rd = O.reduce(J)
    t_red = time.perf_counter() - t0
    t0 = time.perf_counter()
    if np.iscomplexobj(sig) or np.iscomplexobj(tau):
        g = np.random.default_rng(12)
        for s in range(k):
            Sh = O.shift_complex(Rd, sig[s], tau[s])
            for _ in range(R):
                b = g.standard_normal(n) + 1j * g.standard_normal(n)
                x = O.ldiv_complex(Rd, Sh, b)
                Jx = J @ x.real + 1j * (J @ x.imag)  # a real J: no complex copy of it
                x = x + O.ldiv_complex(Rd, Sh, b - (sig[s] * x + tau[s] * Jx))
    else:
        O.shift_solve_batch(Rd, J, sig[:k], tau[:k], np.asfortranarray(c["B"][:, :k]), steps=1)
    t_sh = time.perf_counter() - t0
    desc = (f"{name}: FP64 reduction of n = {n} once ({t_red:.2f} s), then {k} of {S} shifts with {R} right-hand "
            f"side(s) each, shift LU + solve + 1 refinement step ({t_sh:.2f} s), scaled to {S} shifts")
    return t_red + t_sh * S / k, S * R, desc


class Form:
    """One form of the path on the device: the workspace, the shift batch and one step.
    refine = ("fixed", max_steps): lhl_refine_tol; ("gmres", max_cycles, restart): lhl_refine_gmres
    with the host stopping once every column is at the tolerance."""

    def __init__(self, G, torch, precision, n, S, dev, refine):
        self.G, self.torch = G, torch
        self.precision = precision
        self.ws = G.LHLWorkspace(n, precision)
        self.sh = G.LHLShift(n, S)
        self.X = torch.empty((S, n), dtype=torch.float64, device=dev).t()
        self.Rs = torch.empty((S, n), dtype=torch.float64, device=dev)
        self.res = torch.empty(S, dtype=torch.float64, device=dev)
        self.refine = refine

    def reduce(self, Jd):
        self.G.lhl_reduce_(self.ws, Jd, True)

    def chain(self, Jd, Bd, sig, tau):
        G = self.G
        G.lhl_shift_batched_(self.sh, self.ws, sig, tau)
        self.X.copy_(Bd)
        G.lhl_ldiv_(self.X, self.sh, self.ws)
        if self.refine[0] == "gmres":
            G.lhl_refine_gmres_(self.X, Jd, Bd, self.sh, self.ws, tol=TOL, max_cycles=self.refine[1],
                                restart=self.refine[2], host_check=True, R=self.Rs, res=self.res)
        else:
            G.lhl_refine_tol_(self.X, Jd, Bd, self.sh, self.ws, tol=TOL, max_steps=self.refine[1], R=self.Rs,
                              res=self.res)

    def step(self, Jd, Bd, sig, tau):
        self.reduce(Jd)
        self.chain(Jd, Bd, sig, tau)


def count_launches(torch, fn):
    """Kernels of this library launched by one call of fn, counted from the CUDA activity
    trace of an untimed run (torch.profiler); None where the trace is unavailable."""
    try:
        from torch.profiler import ProfilerActivity, profile
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            fn()
            torch.cuda.synchronize()
        names = [e.name for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA]
        ours = [nm for nm in names if "lhl::" in nm]
        return len(ours) if ours else None
    except Exception:  # pragma: no cover - profiler missing on the box
        return None


TOL = 1e-10
MIXED_REFINE = ("gmres", 4, 3)   # GMRES(3), at most 4 cycles
PLAIN_REFINE = ("fixed", 2)
FIXED_POINT_REPLAY_STEPS = 16


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-baseline-steps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-c4", action="store_true", help="skip the batched config-4 measurement")
    ap.add_argument("--no-launch-count", action="store_true",
                    help="skip the profiler-based kernel count (for runs under ncu)")
    ap.add_argument("--cpu-config", choices=["c1", "c3", "c5"],
                    help="with --impl reference: time the oracle on a bounded sample of this configuration "
                         "instead (thread count from OMP_NUM_THREADS; set OPENBLAS_NUM_THREADS alike)")
    ap.add_argument("--cpu-shifts", type=int, default=4, help="--cpu-config: shifts in the sample")
    args = ap.parse_args()
    world, rank, local = dist_setup(args.gpus)

    from lhl_gpu import configs
    cfg = configs.config2()
    n, S = cfg["n"], len(cfg["sigma"])
    config = {"workload": "c2: J 2048x2048 FP64 N(0,1), 64 shifts (1,-g) g log-uniform [1e-4,1e-1], 1 RHS/shift; "
                          "one step = reduction + 64 shift LUs + 64 solves + refinement until every solve is at "
                          "<= 1e-10 relative residual",
              "n": n, "shifts": S, "rhs_per_shift": 1, "tolerance": TOL,
              "form": "mixed: FP32 reduction (FP64-accumulated column updates), FP64 balancing, shift LU, solves, "
                      "residuals and refinement",
              "l2": "flushed between timed steps (256 MiB write)", "replicas": world}

    if args.impl == "reference" and args.cpu_config:
        if rank != 0:
            return
        from oracle import oracle as O
        sec, units, desc = cpu_config_sample(args.cpu_config, args.cpu_shifts)
        val = units / sec
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "ms_per_step": sec * 1e3,
                          "higher_is_better": True, "dtype": "f64", "config": {"workload": args.cpu_config},
                          "cpu_baseline": {"value": val, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
                                           "sample": desc + "; oracle C restatement, OpenMP"}}), flush=True)
        return

    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import oracle as O
        threads = O.num_threads()
        warm = max(args.warmup, 0)
        times, _ = cpu_reference_run(cfg, max(args.steps, 1), warm, threads)
        sec = float(np.mean(times))
        val = S / sec
        line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
                "steps": len(times), "warmup": warm, "ms_per_step": sec * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (numpy PCG64 seeds 2,3,4)",
                "config": config,
                "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                                 "sample": f"{len(times)} full step(s) of the workload (FP64 reduction + 64 shift "
                                           f"LUs + solves + 1 refinement): oracle C restatement, OpenMP"},
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
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    mixed = Form(G, torch, G.LHL_PREC_MIXED, n, S, dev, MIXED_REFINE)
    plain = Form(G, torch, G.LHL_PREC_FP64, n, S, dev, PLAIN_REFINE)

    def timed(form):
        for _ in range(max(args.warmup, 3)):
            form.step(Jd, Bd, sig, tau)
        torch.cuda.synchronize()
        form.ws.check()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            for k in range(args.steps):
                flush.fill_(float(k))
                evs[k][0].record(stream)
                form.step(Jd, Bd, sig, tau)
                evs[k][1].record(stream)
            torch.cuda.synchronize()
        if pg:
            pg.barrier()
        form.ws.check()
        ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
        # every solve of the timed work is at <= 1e-10 (final residuals from the refinement)
        res = form.res.cpu().numpy()
        assert (res <= TOL).all(), f"residual above {TOL}: {res.max()}"
        return ms, clk.summary(), float(res.max())

    ms_mixed, clk_mixed, res_mixed = timed(mixed)
    ms_plain, clk_plain, res_plain = timed(plain)

    # ---- phases, each timed alone with events on the launching stream ----
    def phases(form):
        ph = {"reduce": time_events(stream, lambda: form.reduce(Jd), 5, flush),
              "chain": time_events(stream, lambda: form.chain(Jd, Bd, sig, tau), 3, flush)}
        ph["shift"] = time_events(stream, lambda: G.lhl_shift_batched_(form.sh, form.ws, sig, tau), 3, flush)
        ph["ldiv"] = time_events(stream, lambda: G.lhl_ldiv_(form.X, form.sh, form.ws), 3, flush)
        return ph

    ph_mixed = phases(mixed)
    ph_plain = phases(plain)
    # what the mixed form's refinement needed: fixed-point steps per column (a replay of
    # lhl_refine_tol with growing step counts) against GMRES-IR cycles
    G.lhl_shift_batched_(mixed.sh, mixed.ws, sig, tau)
    X0 = Bd.clone()
    G.lhl_ldiv_(X0, mixed.sh, mixed.ws)
    need = np.full(S, -1)
    for st in range(FIXED_POINT_REPLAY_STEPS + 1):
        Xs = X0.clone()
        r = G.lhl_refine_tol_(Xs, Jd, Bd, mixed.sh, mixed.ws, tol=0.0, max_steps=st).cpu().numpy()
        need[(need < 0) & (r <= TOL)] = st
        if (need >= 0).all():
            break
    gm_cycles = None
    for cyc in range(1, MIXED_REFINE[1] + 1):
        Xs = X0.clone()
        r = G.lhl_refine_gmres_(Xs, Jd, Bd, mixed.sh, mixed.ws, tol=TOL, max_cycles=cyc,
                                restart=MIXED_REFINE[2]).cpu().numpy()
        if (r <= TOL).all():
            gm_cycles = cyc
            break
    fixed_chain_ms = time_events(stream, lambda: (G.lhl_shift_batched_(mixed.sh, mixed.ws, sig, tau),
                                                  mixed.X.copy_(Bd), G.lhl_ldiv_(mixed.X, mixed.sh, mixed.ws),
                                                  G.lhl_refine_tol_(mixed.X, Jd, Bd, mixed.sh, mixed.ws, tol=TOL,
                                                                    max_steps=FIXED_POINT_REPLAY_STEPS, R=mixed.Rs,
                                                                    res=mixed.res)), 3, flush)
    launches = None if args.no_launch_count else count_launches(torch, lambda: mixed.step(Jd, Bd, sig, tau))

    # ---- whole-step lower bound: the compulsory HBM bytes of each phase at the measured copy
    # bandwidth (every phase here is HBM- or latency-bound; none is tensor-core work):
    # reduction 4n^3/3 (FP32 GEMV stream) + 16n^2; shift LUs 4n^2 (Ht, shared) + S 4n^2 (Gt);
    # one solve pass S 4n^2 (Gt) + 8n^2 (L, shared); one residual pass 8n^2 (J, shared)
    def step_lower_ms(peak_gbs):
        b = (4.0 * n ** 3 / 3 + 16.0 * n * n) + (4.0 * n * n + S * 4.0 * n * n) \
            + (S * 4.0 * n * n + 8.0 * n * n) + 8.0 * n * n
        return b / (peak_gbs * 1e9) * 1e3

    # ---- roofline of the dominant kernel: the mixed reduction ----
    alg_bytes = 4.0 * (n ** 3) / 3.0 + 16.0 * n * n   # FP32 GEMV stream (4 n^3/3) + J in, factors out (FP64)
    peak, peak_kind = peaks()
    red = ph_mixed["reduce"]
    achieved = alg_bytes / (red * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(REPO, "profiles", "reduce_mixed_kernel_c2_n2048.md")
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
    # Two device input slots: a Jacobian stream is served double-buffered, the copy of step t+1's
    # inputs (on a copy stream) overlapping step t's work.  Every step still copies its own J, B
    # and shifts from pinned host memory and reads its solutions back, all inside the timed region;
    # the L2 flush is inside it too.
    slots = [(torch.empty_like(Jd), torch.empty_like(Bd), torch.empty((2, S), dtype=torch.float64, device=dev))
             for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    ready = [torch.cuda.Event() for _ in range(2)]
    freed = [torch.cuda.Event() for _ in range(2)]

    def load_inputs(s):
        Js, Bs, sts = slots[s]
        with torch.cuda.stream(copy_stream):
            copy_stream.wait_event(freed[s])
            Js.copy_(Jh, non_blocking=True)
            Bs.copy_(Bh, non_blocking=True)
            sts.copy_(sh_h, non_blocking=True)
            ready[s].record(copy_stream)

    def e2e_run(K):
        """K steps: the first step's copy, then per step t: the copy of step t+1 issued, the wait
        for step t's inputs, the L2 flush, the step, the read-back of X."""
        for s in range(2):
            freed[s].record(stream)
        load_inputs(0)
        for t in range(K):
            s = t & 1
            if t + 1 < K:
                load_inputs(1 - s)
            stream.wait_event(ready[s])
            flush.fill_(float(t))
            Js, Bs, sts = slots[s]
            mixed.step(Js, Bs, sts[0], sts[1])
            freed[s].record(stream)
            Xh.copy_(mixed.X, non_blocking=True)

    e2e_run(2)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    e2e_run(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = ev0.elapsed_time(ev1) / args.steps
    h2d = Jh.numel() * 8 + Bh.numel() * 8 + sh_h.numel() * 8
    d2h = Xh.numel() * 8

    # ---- config 4: 4096 independent Jacobians of uneven order, batched (FP64) ----
    c4 = None
    if not args.no_c4:
        from lhl_gpu.sharding import jacobian_partition
        cfg4 = configs.config4()
        total4 = len(cfg4["ns"])
        mine = jacobian_partition([int(v) for v in cfg4["ns"]], world)[rank]  # all of them on one GPU
        ns4 = [int(cfg4["ns"][i]) for i in mine]
        S4, R4 = 8, 4
        bt = G.LHLBatch(ns4, S4)
        J4 = torch.as_tensor(bt.pack_matrices([cfg4["mats"][i] for i in mine])).to(dev)
        B4 = torch.as_tensor(bt.pack_rhs([cfg4["rhs"][i][:, :S4 * R4] for i in mine])).to(dev)
        X4 = torch.empty_like(B4)
        sg4 = torch.as_tensor(cfg4["sigma"][mine].ravel()).to(dev)
        ta4 = torch.as_tensor(cfg4["tau"][mine].ravel()).to(dev)
        res4 = torch.empty(len(ns4) * S4 * R4, dtype=torch.float64, device=dev)

        def c4_step():
            G.lhl_reduce_batched_(bt, J4, True)
            G.lhl_shift_batched_all_(bt, sg4, ta4)
            G.lhl_solve_batched_(bt, J4, B4, X4, R4, tol=TOL, max_steps=6, res=res4)

        for _ in range(3):
            c4_step()
        torch.cuda.synchronize()
        c4_ms = time_events(stream, c4_step, max(3, min(args.steps, 5)), flush)
        r4 = res4.cpu().numpy()
        assert (r4 <= TOL).all(), f"config 4 residual above {TOL}: {r4.max()}"
        c4 = {"workload": "c4: 4096 J, n uniform [16,256], N(0,1) - 5I; 8 shifts (1,-g) g log-uniform "
                          "[1e-3,1e-1]; 4 RHS/shift; reduction + shift LUs + solves refined to 1e-10, "
                          "three launches, FP64 (plain form)",
              "value": None, "unit": UNIT, "ms_per_step": None, "ranks": world,
              "partition": "matrices balanced across ranks by n^3 (lhl_gpu.sharding.jacobian_partition)",
              "phases_ms": {"reduce_batched": time_events(stream, lambda: G.lhl_reduce_batched_(bt, J4, True), 3,
                                                          flush),
                            "shift_batched_all": time_events(stream, lambda: G.lhl_shift_batched_all_(bt, sg4, ta4),
                                                             3, flush),
                            "solve_batched": time_events(stream, lambda: G.lhl_solve_batched_(
                                bt, J4, B4, X4, R4, tol=TOL, max_steps=6, res=res4), 3, flush)},
              "max_rel_residual": float(r4.max()), "_ms": c4_ms}

    # ---- max over ranks ----
    ms_mixed, ms_plain, e2e_ms, c4_max = max_over_ranks(
        [ms_mixed, ms_plain, e2e_ms, c4["_ms"] if c4 else 0.0], dev, pg)
    if c4:
        c4.pop("_ms")
        c4["ms_per_step"] = c4_max
        c4["value"] = total4 * S4 * R4 / (c4_max * 1e-3)
    value = whole_job_rate(world, S, ms_mixed)
    plain_value = whole_job_rate(world, S, ms_plain)

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            from oracle import oracle as O
            times, Xc = cpu_reference_run(cfg, args.cpu_baseline_steps, 0, None)
            sec = float(np.mean(times))
            cpu = {"value": S / sec, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
                   "sample": f"{len(times)} full step(s) (FP64 reduction + 64 shift LUs + solves + 1 refinement), "
                             f"oracle C restatement with OpenMP, {sec:.2f} s/step"}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64 (mixed form: f32 reduction)",
                "data": "synthetic (numpy PCG64 seeds 2,3,4)", "config": config,
                "plain_fp64": {"value": plain_value, "unit": UNIT, "ms_per_step": ms_plain,
                               "max_rel_residual": res_plain, "phases_ms": ph_plain,
                               "form": "plain: FP64 throughout, bit-identical reduction and shift LUs",
                               "clocks": clk_plain},
                "mixed_vs_plain": value / plain_value,
                "excluding_reduction": {"mixed": S / (ph_mixed["chain"] * 1e-3), "plain": S / (ph_plain["chain"] * 1e-3),
                                        "unit": UNIT, "note": "S*R / T(shift + solve + refine), reduction excluded"},
                "phases_ms": ph_mixed, "max_rel_residual": res_mixed,
                "refinement": {"method": f"GMRES-IR: GMRES({MIXED_REFINE[2]}) cycles left-preconditioned by the "
                                         f"shift's factorisation, host check per cycle",
                               "gmres_cycles_needed": gm_cycles,
                               "fixed_point_steps_needed": {
                                   "max": int(need.max()), "mean": float(need.mean()),
                                   "histogram": {int(k): int((need == k).sum()) for k in np.unique(need)}},
                               "chain_ms_with_fixed_point": fixed_chain_ms},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                             "kernel": "lhl_reduce, mixed form (balance + FP32 ELMHES, cooperative launches)",
                             "algorithmic_bytes": alg_bytes},
                "roofline_step": {"t_lower_ms": step_lower_ms(peak), "t_measured_ms": ms_mixed,
                                  "frac": step_lower_ms(peak) / ms_mixed,
                                  "counts": "reduction + all shift LUs + one solve pass + one residual pass, "
                                            "compulsory HBM bytes at the measured copy bandwidth"},
                "cpu_baseline": cpu,
                "e2e": {"value": world * S / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                        "timing": "K steps in one event-timed region through the public API: per step the "
                                  "pinned host->device copy of J, B and the shifts (double-buffered: step "
                                  "t+1's copy overlaps step t), the L2 flush, the step, the read-back of X"},
                "batched_c4": c4,
                "gpu_launches": launches * args.steps if launches is not None else None,
                "clocks": clk_mixed}
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
