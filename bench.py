"""Benchmark: shifted solves per second on one B200 (LHLFactorization.jl's hot path).

Headline workload, config 5 (the largest configuration; the one whose stated form is the mixed
one): a real J 8192 x 8192 FP64 with iid N(0,1)/sqrt(n) entries; 128 complex shifts
s = a + ib, a ~ U[-2, 0], b ~ U[0, 10], (sigma, tau) = (s, -1); 32 complex N(0,1) right-hand
sides per shift.  One step = the whole path on one batch: the reduction J = Z H Z^-1, the 128
complex shift LUs, the 4096 complex solves, then FP64 refinement until every solve is at
<= 1e-10 relative residual (lhl_refine_tol; the final residuals are checked after the timed
region).  value = 4096 solves / step time of the mixed form (FP32 reduction); the plain FP64
form (bit-identical to the reference's operation order) is timed the same way and reported
beside it, with the ratio.  Configurations 1, 2 and 3 (both forms) and the batched config 4
are reported as extra fields of the same line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config c5|c2|c3|c1]

N > 1 runs independent replicas, one per GPU (one reduction does not shard); value is the
aggregate.  --impl reference times the oracle (the CPU restatement of the reference's
algorithm, all host threads) on a bounded sample of the same workload; it never loads the
CUDA library.  --case runs one phase of one configuration alone (the small cases that the ncu
summaries under profiles/ were captured on).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import importlib.util
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
TOL = 1e-10
EPS = float(np.finfo(float).eps)


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_configs():
    """lhl_gpu/configs.py by its path: the seeded input generator, without importing the
    package (whose import loads the CUDA library; the reference arm must not)."""
    spec = importlib.util.spec_from_file_location("lhl_configs", os.path.join(PKG, "lhl_gpu", "configs.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


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


# ---------------------------------------------------------------------------------------
# Workloads: the seeded configurations and how each form refines them

DESCR = {
    "c1": "c1: J 400x400 FP64 N(0,1), 3 shifts (1,-g) g in {0.01,0.013,0.021}, 1 RHS/shift",
    "c2": "c2: J 2048x2048 FP64 N(0,1), 64 shifts (1,-g) g log-uniform [1e-4,1e-1], 1 RHS/shift",
    "c3": "c3: stiff J 4096x4096 = Q diag(-lam) Q^-1 + 0.01 N(0,1), lam log-uniform [1,1e4]; 256 shifts "
          "(-1/(dt g), 1), dt g log-uniform [1e-5,1e-2]; 1 RHS/shift",
    "c5": "c5: real J 8192x8192 FP64 N(0,1)/sqrt(n); 128 complex shifts (s,-1), s = a+ib, a~U[-2,0], b~U[0,10]; "
          "32 complex RHS/shift (4096 complex solves)",
}
# refinement per (configuration, form): ("fixed", max steps) = lhl_refine_tol;
# ("gmres", max cycles, restart) = lhl_refine_gmres with a host check per cycle
REFINE = {
    ("c1", "mixed"): ("gmres", 4, 3), ("c1", "plain"): ("fixed", 2),
    ("c2", "mixed"): ("gmres", 4, 3), ("c2", "plain"): ("fixed", 2),
    ("c3", "mixed"): ("gmres", 12, 8), ("c3", "plain"): ("fixed", 4),
    ("c5", "mixed"): ("fixed", 16), ("c5", "plain"): ("fixed", 4),
}


def workload(name, cfgs):
    c = {"c1": cfgs.config1, "c2": cfgs.config2, "c3": cfgs.config3, "c5": cfgs.config5}[name]()
    w = {"name": name, "n": int(c["J"].shape[0]), "J": c["J"], "sigma": np.asarray(c["sigma"]),
         "tau": np.asarray(c["tau"])}
    w["S"] = len(w["sigma"])
    w["cplx"] = bool(np.iscomplexobj(w["sigma"]))
    if name == "c5":
        g = c["rng"]
        n, S, R = c["n"], len(c["sigma"]), c["nrhs"]
        re = g.standard_normal((n, S * R))
        im = g.standard_normal((n, S * R))
        B = np.empty((n, S * R), dtype=np.complex128, order="F")
        B.real = re
        B.imag = im
        w["B"], w["R"] = B, R
        w["tau"] = w["tau"].astype(np.complex128)
    else:
        w["B"], w["R"] = np.asfortranarray(c["B"]), 1
    fx = os.path.join(REPO, "tests", "golden", f"config_{name}.npz")
    w["fixture"] = dict(np.load(fx)) if os.path.exists(fx) else None
    return w


def forward_errors(w, X):
    """Forward error of the sampled columns against the oracle's refined FP64 solutions
    (tests/golden/config_<c>.npz); None where no fixture exists."""
    fx = w["fixture"]
    if fx is None:
        return None
    out = []
    for i, col in enumerate(fx["rhs_columns"]):
        x = X[:, int(col)].cpu().numpy()
        xr = fx["x_ref"][:, i]
        out.append(float(np.linalg.norm(x - xr) / np.linalg.norm(xr)))
    return {"max": max(out), "columns": [int(v) for v in fx["rhs_columns"]], "values": out,
            "against": "the oracle's FP64 solution refined by two steps (tests/golden)"}


class Form:
    """One form of the path on the device for workload w: workspace, the shift object (shared
    between forms when given), solution and residual scratch, and one step."""

    def __init__(self, G, torch, w, form, dev, sh=None, choice=None):
        self.G, self.torch, self.w, self.form = G, torch, w, form
        n, S, R = w["n"], w["S"], w["R"]
        dt = torch.complex128 if w["cplx"] else torch.float64
        self.ws = G.LHLWorkspace(n, G.LHL_PREC_MIXED if form == "mixed" else G.LHL_PREC_FP64,
                                 shift_complex=w["cplx"])
        self.sh = sh if sh is not None else G.LHLShift(n, S, complex=w["cplx"])
        self.X = torch.empty((S * R, n), dtype=dt, device=dev).t()
        self.Rs = torch.empty((S * R, n), dtype=dt, device=dev)
        self.res = torch.empty(S * R, dtype=torch.float64, device=dev)
        self.refine = REFINE[(w["name"], form)]
        self.choice = None
        if choice:  # the tuner's choices for this workload (lhl_gpu/tune.py)
            self.apply(choice)

    def apply(self, choice):
        sv = choice.get("shift_variant") or [0, 0]
        self.ws.set_shift_variant(int(sv[0]), int(sv[1]))
        if self.form == "mixed" and choice.get("mixed_kernel"):
            self.ws.set_mixed_kernel(int(choice["mixed_kernel"]))
        if choice.get("refine"):
            self.refine = tuple(choice["refine"])
        self.choice = {k: choice[k] for k in ("shift_variant", "mixed_kernel", "refine", "measured") if k in choice}

    def reduce(self, Jd):
        self.G.lhl_reduce_(self.ws, Jd, True)

    def shift(self, sig, tau):
        self.G.lhl_shift_batched_(self.sh, self.ws, sig, tau)

    def solve(self, Bd):
        self.X.copy_(Bd)
        self.G.lhl_ldiv_(self.X, self.sh, self.ws, rhs_per_shift=self.w["R"])

    def refine_(self, Jd, Bd):
        G, R = self.G, self.w["R"]
        if self.refine[0] == "gmres":
            G.lhl_refine_gmres_(self.X, Jd, Bd, self.sh, self.ws, tol=TOL, max_cycles=self.refine[1],
                                restart=self.refine[2], rhs_per_shift=R, host_check=True, R=self.Rs, res=self.res)
        elif self.refine[0] == "hybrid":  # fixed-point steps for the bulk, then GMRES-IR for what is left
            G.lhl_refine_tol_(self.X, Jd, Bd, self.sh, self.ws, tol=TOL, max_steps=self.refine[1],
                              rhs_per_shift=R, R=self.Rs, res=self.res)
            G.lhl_refine_gmres_(self.X, Jd, Bd, self.sh, self.ws, tol=TOL, max_cycles=self.refine[2],
                                restart=self.refine[3], rhs_per_shift=R, host_check=True, R=self.Rs, res=self.res)
        else:
            G.lhl_refine_tol_(self.X, Jd, Bd, self.sh, self.ws, tol=TOL, max_steps=self.refine[1],
                              rhs_per_shift=R, R=self.Rs, res=self.res)

    def chain(self, Jd, Bd, sig, tau):
        self.shift(sig, tau)
        self.solve(Bd)
        self.refine_(Jd, Bd)

    def step(self, Jd, Bd, sig, tau):
        self.reduce(Jd)
        self.chain(Jd, Bd, sig, tau)

    def describe_refine(self):
        r = self.refine
        if r[0] == "gmres":
            return f"GMRES-IR: GMRES({r[2]}) x {r[1]} cycles at most, host check per cycle"
        if r[0] == "hybrid":
            return (f"{r[1]} fixed-point lhl_refine_tol steps, then GMRES-IR GMRES({r[3]}) x {r[2]} cycles at most "
                    f"on the columns still above the tolerance")
        return f"fixed-point lhl_refine_tol, {r[1]} steps at most"


def device_name(torch):
    try:
        return torch.cuda.get_device_name()
    except Exception:  # pragma: no cover
        return "unknown"


def cached_choice(torch, w, form):
    """The tuner's cached choice for workload w and form (lhl_gpu/tuning.json), or None."""
    from lhl_gpu import tune as T
    return T.lookup(device_name(torch), w["cplx"], w["n"], form, w["R"])


def solves_accepted(w, f):
    """Every solve at the tolerance (config 3: at the tolerance or at its FP64 floor)."""
    if w["name"] == "c3":
        return floor_counts(w, f)["neither"] == 0
    return bool((f.res.cpu().numpy() <= TOL).all())


def tune_config(G, torch, name, cfgs, dev):
    """Timed trials of the open choices of configuration `name` for both forms (lhl_gpu/tune.py):
    the mixed reduction kernel, the shift LU's launch shape, the refinement scheme.  Writes the
    cache and returns the choices."""
    from lhl_gpu import tune as T
    w = workload(name, cfgs)
    Jd = torch.as_tensor(w["J"]).to(dev)
    Bd = torch.as_tensor(w["B"]).to(dev)
    sig = torch.as_tensor(w["sigma"]).to(dev)
    tau = torch.as_tensor(w["tau"]).to(dev)
    sh = G.LHLShift(w["n"], w["S"], complex=w["cplx"])
    cache = T.load_cache()
    out = {}
    for fm in ("mixed", "plain"):
        f = Form(G, torch, w, fm, dev, sh)
        choice = {}
        if fm == "mixed":
            choice["mixed_kernel"], choice["kernel_trials"] = T.tune_mixed_kernel(torch, f.ws, lambda: f.reduce(Jd))
        f.reduce(Jd)
        v, choice["shift_trials"] = T.tune_shift_variant(G, torch, f.ws, f.sh, sig, tau)
        choice["shift_variant"] = [0, v] if w["cplx"] else [v, 0]
        f.ws.set_shift_variant(*choice["shift_variant"])

        def run_chain(ch, f=f):
            f.refine = tuple(ch)
            f.chain(Jd, Bd, sig, tau)

        cands = [c for c in T.REFINE_CANDIDATES[fm] if not (w["cplx"] and c[0] == "gmres" and c[2] > 4)]
        best, choice["refine_trials"] = T.tune_refine(torch, fm, run_chain, lambda f=f: solves_accepted(w, f),
                                                      candidates=cands)
        choice["refine"] = list(best) if best else list(REFINE[(name, fm)])
        key = T.workload_key(device_name(torch), w["cplx"], w["n"], fm, w["R"])
        T.record(cache, key, choice)
        out[key] = cache[key]
        del f
    T.save_cache(cache)
    del sh
    torch.cuda.empty_cache()
    return out


def time_events(torch, stream, fn, reps, flush):
    out = []
    for k in range(reps):
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        out.append(a.elapsed_time(b))
    return float(np.mean(out))


def timed_steps(torch, form, dev_in, steps, warmup, flush, stream, pg=None, clocks=None):
    """warmup untimed steps, then `steps` steps each bracketed by CUDA events on the launching
    stream (L2 flushed before each); returns (mean ms, clock summary)."""
    Jd, Bd, sig, tau = dev_in
    for _ in range(warmup):
        form.step(Jd, Bd, sig, tau)
    torch.cuda.synchronize()
    form.ws.check()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with ClockSampler(clocks if clocks is not None else 0) as clk:
        for k in range(steps):
            flush.fill_(float(k))
            evs[k][0].record(stream)
            form.step(Jd, Bd, sig, tau)
            evs[k][1].record(stream)
        torch.cuda.synchronize()
    if pg:
        pg.barrier()
    form.ws.check()
    return float(np.mean([a.elapsed_time(b) for a, b in evs])), clk.summary()


def floor_counts(w, form):
    """Config 3: FP64's attainable relative residual eps (|sigma| + |tau| ||J||_1) ||x|| / ||b||
    per solve, and how many solves are at 1e-10, or else at their floor (within 10x)."""
    J1 = float(np.abs(w["J"]).sum(axis=0).max())
    X = form.X.cpu().numpy()
    res = form.res.cpu().numpy()
    B = w["B"]
    fl = np.array([EPS * (abs(w["sigma"][c]) + abs(w["tau"][c]) * J1) * np.linalg.norm(X[:, c])
                   / np.linalg.norm(B[:, c]) for c in range(X.shape[1])])
    at_tol = res <= TOL
    floor_limited = (~at_tol) & (fl > TOL / 10) & (res <= 10 * fl)
    return {"at_1e-10": int(at_tol.sum()), "floor_limited": int(floor_limited.sum()),
            "neither": int((~at_tol & ~floor_limited).sum()), "max_floor": float(fl.max()),
            "max_rel_residual": float(res.max()),
            "note": "a solve above 1e-10 whose FP64 floor eps ||W||_1 ||x|| / ||b|| exceeds 1e-11 and whose residual "
                    "is within 10x of that floor counts as floor_limited"}


def config_extra(G, torch, name, cfgs, dev, stream, flush, steps):
    """Both forms of configuration `name` (c1, c2, c3) timed over `steps` steps after one warm-up."""
    w = workload(name, cfgs)
    Jd = torch.as_tensor(w["J"]).to(dev)
    Bd = torch.as_tensor(w["B"]).to(dev)
    sig = torch.as_tensor(w["sigma"]).to(dev)
    tau = torch.as_tensor(w["tau"]).to(dev)
    sh = G.LHLShift(w["n"], w["S"], complex=w["cplx"])
    out = {"workload": DESCR[name], "steps": steps, "warmup": 1}
    X_plain = None
    for fm in ("mixed", "plain"):
        f = Form(G, torch, w, fm, dev, sh, cached_choice(torch, w, fm))
        ms, _ = timed_steps(torch, f, (Jd, Bd, sig, tau), steps, 1, flush, stream)
        red = time_events(torch, stream, lambda: f.reduce(Jd), 2, flush)
        res = f.res.cpu().numpy()
        d = {"value": w["S"] * w["R"] / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "reduce_ms": red,
             "chain_ms": ms - red, "max_rel_residual": float(res.max()), "n_at_1e-10": int((res <= TOL).sum()),
             "solves": int(res.size), "refinement": f.describe_refine(),
             "tuning": f.choice or "defaults (no cached choice for this device)"}
        fe = forward_errors(w, f.X)
        if fe is not None:
            d["forward_error"] = fe
        if name == "c3":
            d["floor"] = floor_counts(w, f)
        if fm == "plain":
            X_plain = f.X.clone()
        else:
            X_mixed = f.X.clone()
        out[fm] = d
        del f
    out["mixed_vs_plain"] = out["mixed"]["value"] / out["plain"]["value"]
    if out["mixed"].get("forward_error") is None:
        e = torch.linalg.vector_norm(X_mixed - X_plain, dim=0) / torch.linalg.vector_norm(X_plain, dim=0)
        out["mixed"]["forward_error_vs_plain"] = {"max": float(e.max()), "median": float(e.median()),
                                                  "against": "the plain form's refined FP64 solution"}
    del sh
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------------------
# CPU baseline: the oracle (C restatement of the reference's Float64 path, OpenMP reduction;
# the per-right-hand-side solves of a shift spread over host threads), on a bounded sample

def _sub_workload(w, sel):
    """Workload w restricted to the shifts `sel` (same J, so the cached reduction serves it)."""
    R = w["R"]
    sub = dict(w)
    sub["sigma"], sub["tau"], sub["S"] = w["sigma"][sel], w["tau"][sel], len(sel)
    sub["B"] = np.asfortranarray(np.concatenate([w["B"][:, s * R:(s + 1) * R] for s in sel], axis=1))
    return sub


def _oracle_reduce(w):
    """The oracle's FP64 reduction of w's J (OpenMP), kept for the chains that follow; seconds."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    _RED_CACHE["key"] = id(w["J"])
    _RED_CACHE["R"] = O.reduce(w["J"])
    return time.perf_counter() - t0


def _chain_only(w, threads):
    """The oracle's per-shift chain for every shift of w, on the reduction _oracle_reduce kept:
    shift LU, every right-hand side solved (spread over host threads; ctypes releases the GIL),
    one lhl_refine! step with the residual J X as one BLAS product over the shift's vectors."""
    from oracle import oracle as O
    assert _RED_CACHE.get("key") == id(w["J"]), "reduce first"
    Rd = _RED_CACHE["R"]
    pool = _POOL.setdefault(threads, cf.ThreadPoolExecutor(max_workers=threads))
    J, R = w["J"], w["R"]
    for s in range(w["S"]):
        cols = slice(s * R, (s + 1) * R)
        if w["cplx"]:
            Sh = O.shift_complex(Rd, w["sigma"][s], w["tau"][s])
            solve = lambda b: O.ldiv_complex(Rd, Sh, b)  # noqa: E731
        else:
            Sh = O.shift(Rd, w["sigma"][s], w["tau"][s])
            solve = lambda b: O.ldiv(Rd, Sh, b)  # noqa: E731
        Bs = w["B"][:, cols]
        X = np.stack(list(pool.map(solve, [Bs[:, i] for i in range(Bs.shape[1])])), axis=1)
        JX = (J @ X.real + 1j * (J @ X.imag)) if w["cplx"] else J @ X
        Rr = Bs - (w["sigma"][s] * X + w["tau"][s] * JX)
        X = X + np.stack(list(pool.map(solve, [Rr[:, i] for i in range(Rr.shape[1])])), axis=1)


_RED_CACHE = {}
_POOL = {}


def cpu_sample(w, shifts, threads):
    """The oracle on a bounded sample of workload w: the full FP64 reduction once, then `shifts`
    of its shifts spread over the set, each with its whole chain (_chain_only).  Returns (seconds
    of the whole step scaled from the sample by the shift count, reduction seconds, seconds per
    shift, a description)."""
    n, S, R = w["n"], w["S"], w["R"]
    t_red = _oracle_reduce(w)
    idx = np.linspace(0, S - 1, shifts).round().astype(int) if shifts < S else np.arange(S)
    t0 = time.perf_counter()
    _chain_only(_sub_workload(w, list(idx)), threads)
    t_sh = (time.perf_counter() - t0) / len(idx)
    desc = (f"{w['name']}: the oracle's FP64 reduction of n = {n} once ({t_red:.2f} s, OpenMP), then {len(idx)} of "
            f"{S} shifts, each: shift LU, {R} solve(s) over {threads} host threads, one refinement step (BLAS "
            f"residual) ({t_sh:.2f} s per shift); step time = reduction + per-shift time x {S}")
    return t_red + t_sh * S, t_red, t_sh, desc


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_arm(args, cfgs, rank):
    """--impl reference: the oracle on the box's host cores, bounded: the reduction once, then
    each of warmup + steps steps one shift's whole chain (--cpu-shifts shifts per step, cycling
    through the set); the step time reported is the reduction plus the mean per-shift time times
    the shift count.  Never imports the CUDA library."""
    if rank != 0:
        return
    from oracle import oracle as O
    name = args.config
    w = workload(name, cfgs)
    threads = host_threads()
    per_step = max(1, args.cpu_shifts)
    S = w["S"]
    t_red = _oracle_reduce(w)
    shift_times = []
    for it in range(args.warmup + args.steps):
        s0 = (it * per_step) % S
        sub = _sub_workload(w, [(s0 + j) % S for j in range(per_step)])
        t1 = time.perf_counter()
        _chain_only(sub, threads)
        if it >= args.warmup:
            shift_times.append((time.perf_counter() - t1) / per_step)
    t_sh = float(np.mean(shift_times))
    sec = t_red + t_sh * S
    val = S * w["R"] / sec
    sample = (f"{name}: oracle (C restatement of the reference's Float64 path; the reference is Julia, absent on "
              f"this box): FP64 reduction of n = {w['n']} once ({t_red:.2f} s, OpenMP, {O.num_threads()} threads); "
              f"each of the {args.steps} timed steps ({args.warmup} untimed first) = {per_step} shift(s) with shift "
              f"LU, {w['R']} solve(s) over {threads} threads and one refinement step ({t_sh:.3f} s per shift); "
              f"step time = reduction + mean shift time x {S} shifts")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (numpy PCG64 seeds)",
            "config": {"workload": DESCR[name], "n": w["n"], "shifts": S, "rhs_per_shift": w["R"]},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


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


PLAIN_STEPS_MAX = 5
E2E_STEPS_MAX = 10


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c5", choices=["c5", "c2", "c3", "c1"],
                    help="headline workload (default config 5)")
    ap.add_argument("--cpu-shifts", type=int, default=1, help="CPU sample: shifts per sampled step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip configurations 1-3 and 4 beside the headline")
    ap.add_argument("--no-launch-count", action="store_true",
                    help="skip the profiler-based kernel count (for runs under ncu)")
    ap.add_argument("--case", choices=["reduce", "shift", "ldiv", "step"],
                    help="run one phase of --config's --form alone, --reps times (profiling cases)")
    ap.add_argument("--form", default="mixed", choices=["mixed", "plain"])
    ap.add_argument("--mixed-kernel", type=int, default=0, choices=[0, 1, 2],
                    help="--case, mixed form: 1 the eager FP32 reduction kernel, 2 the panel-delayed one "
                         "(0: the cached choice)")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--shifts", type=int, default=0, help="--case: use only the first SHIFTS shifts")
    ap.add_argument("--tune", default="", help="comma-separated configurations (c1,c2,c3,c5) to tune by timed "
                                               "trials (lhl_gpu/tune.py); writes lhl_gpu/tuning.json and exits")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.case is None else args.warmup
    world, rank, local = dist_setup(args.gpus)
    cfgs = load_configs()

    if args.impl == "reference":
        return reference_arm(args, cfgs, rank)

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
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    if args.tune:
        res = {nm: tune_config(G, torch, nm, cfgs, dev) for nm in args.tune.split(",") if nm}
        print(json.dumps({"tuned": res}), flush=True)
        return

    w = workload(args.config, cfgs)
    if args.case is not None and args.shifts:
        k = args.shifts
        w["S"], w["sigma"], w["tau"] = k, w["sigma"][:k], w["tau"][:k]
        w["B"] = np.asfortranarray(w["B"][:, :k * w["R"]])
    n, S, R = w["n"], w["S"], w["R"]
    Jd = torch.as_tensor(w["J"]).to(dev)
    Bd = torch.as_tensor(w["B"]).to(dev)
    sig = torch.as_tensor(w["sigma"]).to(dev)
    tau = torch.as_tensor(w["tau"]).to(dev)
    dev_in = (Jd, Bd, sig, tau)

    if args.case is not None:  # one phase alone (profiling)
        f = Form(G, torch, w, args.form, dev, None, cached_choice(torch, w, args.form))
        if args.mixed_kernel and args.form == "mixed":
            f.ws.set_mixed_kernel(args.mixed_kernel)
        f.step(Jd, Bd, sig, tau)
        torch.cuda.synchronize()
        fn = {"reduce": lambda: f.reduce(Jd), "shift": lambda: f.shift(sig, tau), "ldiv": lambda: f.solve(Bd),
              "step": lambda: f.step(Jd, Bd, sig, tau)}[args.case]
        ms = time_events(torch, stream, fn, max(args.reps, 1), flush)
        f.ws.check()
        print(json.dumps({"case": args.case, "config": args.config, "form": args.form, "n": n, "shifts": S,
                          "rhs_per_shift": R, "ms": ms}), flush=True)
        return

    sh = G.LHLShift(n, S, complex=w["cplx"])
    mixed = Form(G, torch, w, "mixed", dev, sh, cached_choice(torch, w, "mixed"))
    plain = Form(G, torch, w, "plain", dev, sh, cached_choice(torch, w, "plain"))
    ms_mixed, clk_mixed = timed_steps(torch, mixed, dev_in, args.steps, args.warmup, flush, stream, pg, local)
    res_mixed = mixed.res.cpu().numpy()
    fe_mixed = forward_errors(w, mixed.X)
    steps_plain = min(args.steps, PLAIN_STEPS_MAX)
    ms_plain, clk_plain = timed_steps(torch, plain, dev_in, steps_plain, 1, flush, stream, pg, local)
    res_plain = plain.res.cpu().numpy()
    fe_plain = forward_errors(w, plain.X)
    if args.config != "c3":
        assert (res_mixed <= TOL).all(), f"mixed residual above {TOL}: {res_mixed.max()}"
        assert (res_plain <= TOL).all(), f"plain residual above {TOL}: {res_plain.max()}"

    # ---- phases, each timed alone with events on the launching stream ----
    def phases(f):
        reps = 2 if n >= 4096 else 3
        ph = {"reduce": time_events(torch, stream, lambda: f.reduce(Jd), reps, flush),
              "shift": time_events(torch, stream, lambda: f.shift(sig, tau), reps, flush),
              "ldiv": time_events(torch, stream, lambda: f.solve(Bd), reps, flush)}
        f.step(Jd, Bd, sig, tau)
        ph["refine"] = time_events(torch, stream, lambda: (f.solve(Bd), f.refine_(Jd, Bd)), reps, flush) - ph["ldiv"]
        return ph

    ph_mixed = phases(mixed)
    ph_plain = phases(plain)
    launches = None if args.no_launch_count else count_launches(torch, lambda: mixed.step(Jd, Bd, sig, tau))
    mixed_choice = mixed.choice or "defaults (no cached choice for this device)"
    plain_choice = plain.choice or "defaults (no cached choice for this device)"
    mixed_refine, plain_refine = mixed.describe_refine(), plain.describe_refine()

    # ---- roofline of the dominant kernel: the mixed form's reduction (its launches alone) ----
    # algorithmic bytes: the FP32 GEMV stream 4 n^3 / 3 (every step re-reads the trailing block)
    # + 16 n^2 (J in, factors and Ht out in FP64)
    alg_bytes = 4.0 * n ** 3 / 3.0 + 16.0 * n * n
    peak, peak_kind = peaks()
    red = ph_mixed["reduce"]
    achieved = alg_bytes / (red * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(REPO, "profiles", f"reduce_mixed_{args.config}.md")
    if os.path.exists(tp):
        for line in open(tp):
            if line.startswith("dram_bytes_per_launch:"):
                traffic = float(line.split(":")[1])

    # ---- end to end through the public API: host buffers, copies inside the timed region ----
    def pinned(a):
        t = torch.empty((a.shape[1], a.shape[0]), dtype=torch.from_numpy(a[:1, :1].copy()).dtype,
                        pin_memory=True).t()
        t.copy_(torch.as_tensor(a))
        return t

    Jh = pinned(w["J"])
    Bh = pinned(w["B"])
    sh_h = torch.as_tensor(np.stack([w["sigma"], w["tau"]]).astype(w["B"].dtype if w["cplx"] else np.float64)).pin_memory()
    Xh = torch.empty((S * R, n), dtype=mixed.X.dtype, pin_memory=True).t()
    # Two device input slots: a stream of Jacobians is served double-buffered, the copy of step
    # t+1's inputs (on a copy stream) overlapping step t's work.  Every step still copies its own
    # J, B and shifts from pinned host memory and reads its solutions back, inside the timed region.
    slots = [(torch.empty_like(Jd), torch.empty_like(Bd), torch.empty_like(sh_h, device=dev)) for _ in range(2)]
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

    e2e_steps = min(args.steps, E2E_STEPS_MAX)
    e2e_run(1)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    e2e_run(e2e_steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = ev0.elapsed_time(ev1) / e2e_steps
    h2d = Jh.numel() * Jh.element_size() + Bh.numel() * Bh.element_size() + sh_h.numel() * sh_h.element_size()
    d2h = Xh.numel() * Xh.element_size()
    e2e_res = G.residual_norms(sh, Jd, Bd, torch.as_tensor(Xh.numpy()).to(dev).t().contiguous().t(),
                               rhs_per_shift=R).cpu().numpy() if w["cplx"] else None
    del slots, Jh, Bh, Xh

    # ---- extras: the other configurations (both forms) and the batched config 4 ----
    extras = {}
    if not args.no_extras:
        del mixed, plain, sh
        torch.cuda.empty_cache()
        for nm, st in (("c1", 3), ("c2", 3), ("c3", 2)):
            if nm != args.config:
                extras[nm] = config_extra(G, torch, nm, cfgs, dev, stream, flush, st)
        extras["c4"] = batched_c4(G, torch, cfgs, dev, stream, flush, world, rank)

    ms_mixed, ms_plain, e2e_ms = max_over_ranks([ms_mixed, ms_plain, e2e_ms], dev, pg)
    value = whole_job_rate(world, S * R, ms_mixed)
    plain_value = whole_job_rate(world, S * R, ms_plain)

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            threads = host_threads()
            sec, t_red, t_sh, desc = cpu_sample(w, max(1, args.cpu_shifts), threads)
            cpu = {"value": S * R / sec, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": desc + "; oracle C restatement (the reference is Julia, absent on this box)"}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64 (mixed form: f32 reduction)",
                "data": "synthetic (numpy PCG64 seeds; no public dataset)",
                "config": {"workload": DESCR[args.config] + "; one step = reduction + every shift LU + every solve "
                                                             "+ refinement until every solve is at <= 1e-10",
                           "n": n, "shifts": S, "rhs_per_shift": R, "tolerance": TOL,
                           "form": "mixed: FP32 reduction, FP64 balancing, shift LUs, solves, residuals and "
                                   "refinement", "l2": "flushed between timed steps (256 MiB write)",
                           "replicas": world},
                "max_rel_residual": float(res_mixed.max()), "forward_error": fe_mixed,
                "refinement": mixed_refine,
                "plain_fp64": {"value": plain_value, "unit": UNIT, "ms_per_step": ms_plain, "steps": steps_plain,
                               "warmup": 1, "max_rel_residual": float(res_plain.max()), "forward_error": fe_plain,
                               "phases_ms": ph_plain, "refinement": plain_refine,
                               "form": "plain: FP64 throughout, bit-identical reduction and shift LUs",
                               "clocks": clk_plain},
                "mixed_vs_plain": value / plain_value,
                "tuning": {"mixed": mixed_choice, "plain": plain_choice,
                           "cache": "lhl.jl_b200/lhl_gpu/tuning.json (bench.py --tune)"},
                "phases_ms": ph_mixed,
                "excluding_reduction": {"mixed": S * R / ((ms_mixed - ph_mixed["reduce"]) * 1e-3),
                                        "plain": S * R / ((ms_plain - ph_plain["reduce"]) * 1e-3), "unit": UNIT,
                                        "note": "S*R / T(shift + solve + refine), reduction excluded"},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                             "kernel": "lhl_reduce, mixed form (its launches alone)",
                             "algorithmic_bytes": alg_bytes,
                             "algorithmic": "4 n^3 / 3 (FP32 GEMV stream) + 16 n^2 (J in, factors and Ht out)"},
                "cpu_baseline": cpu,
                "e2e": {"value": world * S * R / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms, "steps": e2e_steps,
                        "max_rel_residual": float(e2e_res.max()) if e2e_res is not None else None,
                        "timing": "K steps in one event-timed region through the public API: per step the pinned "
                                  "host->device copy of J, B and the shifts (double-buffered: step t+1's copy "
                                  "overlaps step t), the L2 flush, the step, the read-back of X"},
                "extras": extras,
                "gpu_launches": launches * args.steps if launches is not None else None,
                "clocks": clk_mixed}
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


def batched_c4(G, torch, cfgs, dev, stream, flush, world, rank):
    """Config 4: 4096 independent Jacobians of uneven order, batched (FP64), this rank's share."""
    from lhl_gpu.sharding import jacobian_partition
    cfg4 = cfgs.config4()
    total4 = len(cfg4["ns"])
    mine = jacobian_partition([int(v) for v in cfg4["ns"]], world)[rank]
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
    c4_ms = time_events(torch, stream, c4_step, 5, flush)
    r4 = res4.cpu().numpy()
    assert (r4 <= TOL).all(), f"config 4 residual above {TOL}: {r4.max()}"
    return {"workload": "c4: 4096 J, n uniform [16,256], N(0,1) - 5I; 8 shifts (1,-g) g log-uniform [1e-3,1e-1]; "
                        "4 RHS/shift; reduction + shift LUs + solves refined to 1e-10, three launches, FP64",
            "value": len(ns4) * S4 * R4 / (c4_ms * 1e-3) * world, "unit": UNIT, "ms_per_step": c4_ms,
            "matrices": total4, "partition": "matrices balanced across ranks by n^3 (lhl_gpu.sharding)",
            "phases_ms": {"reduce_batched": time_events(torch, stream, lambda: G.lhl_reduce_batched_(bt, J4, True),
                                                        3, flush),
                          "shift_batched_all": time_events(torch, stream, lambda: G.lhl_shift_batched_all_(bt, sg4,
                                                                                                          ta4),
                                                           3, flush),
                          "solve_batched": time_events(torch, stream, lambda: G.lhl_solve_batched_(
                              bt, J4, B4, X4, R4, tol=TOL, max_steps=6, res=res4), 3, flush)},
            "max_rel_residual": float(r4.max())}


if __name__ == "__main__":
    main()
