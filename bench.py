"""Benchmark of the batch Monte Carlo pricing path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step"): the Heston batch -- 1024 European calls, full-truncation
Euler, 200 time steps, 262144 paths each (5.37e10 path-steps), seeded synthetic
parameters (quantkernel_b200.workloads.heston).  Metric: path-steps per second
(and Heston prices per second) for the whole job.

* value  -- device-resident: a plan holds the packed options in HBM; each step
  is one execute() (simulate + finalize kernels), timed with CUDA events on
  the launching stream, L2 flushed (256 MiB write) between steps.
* e2e    -- the same batch through the drop-in C call
  qk_mcm_heston_monte_carlo_price_batch with host buffers: validation, packing,
  host->device copy, kernels and device->host copy inside the timed region.
* roofline -- the simulate kernel's algorithmic issue rate against the SM
  issue peak at the measured clock (a compute-bound kernel: no HBM stream).
* cpu_baseline -- the reference's own CPU implementation (compiled from its
  sources into oracle/_ref) on a bounded sample, all host threads.

Multi-GPU (torchrun): options are independent, so every rank prices its own
1024-option batch (different seeds) with no collective on the data path;
value = all ranks' path-steps / max-over-ranks time ("weak" scaling).

--impl reference times the reference CPU path (oracle/_ref, else the oracle
port) on the same workload, rank 0 only, each step a bounded sample.
"""

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "quant-kernel_b200"))

METRIC = "Heston prices/sec at <=5e-4*S err: surrogate vs plain GPU MC; path-steps/sec"
UNIT = "path-steps/s"
N_OPT, PATHS, STEPS = 1024, 262144, 200
WORKLOAD = f"heston full-truncation Euler: {N_OPT} calls x {PATHS} paths x {STEPS} steps"
# Algorithmic cost per path-step, counted from the reference formulas
# (model_concepts.h) under antithetic pairing, where the two paths of a pair
# share their normals:
#   Heston      one Box-Muller pair per pair-step (log, sqrt, sin, cos) and per
#               path sqrt(v) and exp: 8 XU per pair-step = 4 per path-step;
#               ALU ~30 per path-step: the step's ~12 FMA-fused FP32 ops, half
#               a Box-Muller pair's ~6 FP ops, a quarter of a Philox4x32-10
#               call (~60 integer instructions per call)
#   Euler / LV  one normal per pair-step (half a Box-Muller pair: 2 XU): 1 XU
#               per path-step; ALU ~13 (step ~4, Box-Muller ~1.5, Philox 1/8
#               call ~7.5)
#   Milstein    as Euler plus 3 FP32 ops: 1 XU, ALU ~16
XU_PER_UNIT, ALU_PER_UNIT = 4, 30
STEP_COST = {2: (1, 13), 3: (1, 16), 4: (1, 13), 6: (XU_PER_UNIT, ALU_PER_UNIT)}  # model: (XU, ALU)
# FP64 operations per antithetic pair of the terminal model (make_bsm_terminal
# with one normal per pair): half a Box-Muller pair (log 20, sqrt 6, sin+cos
# 17 and ~6 arithmetic: ~25), two exp (16 each), d0 + d1 z twice with one
# multiply (3), two spot * exp (2), two payoffs (4): ~66, on the FP64 pipe.
# (exp, log, sin/cos and sqrt are costed as textbook range reduction plus a
# polynomial of the degree FP64 accuracy needs.)
FP64_PER_PAIR = 66
SMS, ISSUE_PER_CLK, XU_PER_CLK, FP64_PER_CLK = 148, 128, 16, 64
# Per-SM-clock pipe widths the rooflines divide by: the nominal B200 figures,
# replaced at start-up by the library's throughput probe on the GPU at hand
# (qk_b200_pipe_probe, include/qk_diag.h) when it runs.
PIPES = {"issue": float(ISSUE_PER_CLK), "xu": float(XU_PER_CLK), "fp64": float(FP64_PER_CLK),
         "source": "nominal per-clock SM widths (148 SMs x 128 issue / 16 XU / 64 FP64 lanes per clk)"}
PROBE_KINDS = (("issue", 1), ("xu", 0), ("fp64", 3), ("ffma2_lanes", 2), ("xu_in_heston_mix", 4))


def measure_pipes(qk, device):
    """Measure the pipe widths on `device` with the library's probe (FP32 FMA
    lanes = the issue width, MUFU lanes, FP64 FMA lanes, packed-FMA lanes, and
    MUFU lanes inside a Heston-like instruction mix), in lane-operations per
    SM per clock, and make them the rooflines' denominators.  Returns the
    measured dict, or None (and the nominal widths stay) if the probe fails."""
    import ctypes as ct

    fn = getattr(qk._lib, "qk_b200_pipe_probe", None)
    if fn is None:
        return None
    out = {}
    for key, kind in PROBE_KINDS:
        v = ct.c_double(0.0)
        if fn(int(device), int(kind), ct.byref(v)) != 0 or not v.value > 0:
            return None
        out[key] = v.value
    PIPES.update(issue=out["issue"], xu=out["xu"], fp64=out["fp64"],
                 source=("measured per-SM-clock widths on this GPU (qk_b200_pipe_probe: "
                         f"{out['issue']:.1f} FP32 FMA = issue, {out['xu']:.2f} MUFU, "
                         f"{out['fp64']:.1f} FP64 lanes per clk) x 148 SMs"))
    return out
SUR_CHECKPOINT = ROOT / "quant-kernel_b200" / "quantkernel_b200" / "data" / "heston_surrogate.qksur"
SUR_FLOP_PER_ROW = 2 * (9 * 256 + 256 * 256 * 2 + 256)  # forward multiply-adds x 2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--options", type=int, default=N_OPT,
                    help="options per GPU (profiling runs use a smaller batch)")
    ap.add_argument("--profile", action="store_true",
                    help="device-resident leg only (no e2e, no CPU baseline): for ncu captures")
    ap.add_argument("--surrogate-train", action="store_true",
                    help="label 4e6 Heston tuples with the GPU MC, train the surrogate, save it")
    ap.add_argument("--surrogate", action="store_true",
                    help="surrogate inference leg only (1e6 queries, MC fallback, MC judge)")
    ap.add_argument("--heston-cf", action="store_true",
                    help="Heston characteristic-function leg only")
    ap.add_argument("--cf-options", type=int, default=65536)
    ap.add_argument("--pipe-probe", action="store_true",
                    help="print the measured per-SM-clock pipe widths (qk_b200_pipe_probe) and exit")
    ap.add_argument("--mixed", action="store_true",
                    help="mixed-model leg only (with --profile: the first --options options, "
                         "persistent kernel and per-family grids, two executes each)")
    ap.add_argument("--bsm", action="store_true",
                    help="FP64 terminal BSM leg only (with --profile: three plain executes)")
    ap.add_argument("--vr", action="store_true",
                    help="variance-reduction leg only (device + e2e; no CPU with --profile)")
    ap.add_argument("--sur-device-rows", type=int, default=0,
                    help="time device-resident surrogate inference on this many rows and exit")
    ap.add_argument("--sur-train-n", type=int, default=4_000_000)
    ap.add_argument("--sur-hold-n", type=int, default=100_000)
    ap.add_argument("--sur-epochs", type=int, default=300)
    ap.add_argument("--sur-checkpoint", default=str(SUR_CHECKPOINT))
    ap.add_argument("--cpu-leg", default=None, help=argparse.SUPPRESS)
    return ap.parse_args()


# --------------------------------------------------------------------------- CPU legs
def _cpu_sample_batch(n_opt, paths):
    from quantkernel_b200 import workloads

    h = workloads.heston(N_OPT, paths=paths, steps=STEPS)
    return {k: v[:n_opt] for k, v in h.items()}


HESTON_KEYS = ("spot", "strike", "t", "r", "q", "v0", "kappa", "theta", "sigma", "rho",
               "option_type", "paths", "steps", "seed")
CPU_TIMER = ROOT / "oracle" / "_ref" / "cpu_timer"


def _time_cpu_cxx(b, symbol="qk_mcm_heston_monte_carlo_price_batch"):
    """The compiled reference's batch entry point `symbol` timed by the C++
    harness (oracle/cpu_timer.cpp, std::chrono around the call)."""
    from oracle import oracle as orc

    return orc.time_reference_batch(symbol, b)[0][0]


def _time_cpu(impl, n_opt, paths, threads):
    """One bounded sample of the CPU path; returns (seconds, path_steps).  The
    reference is timed from C++ (std::chrono around its batch call); the
    oracle port, used only where the reference could not be built, from
    Python around its C call."""
    from oracle import oracle as orc

    b = _cpu_sample_batch(n_opt, paths)
    if impl == "reference" and CPU_TIMER.exists():
        return _time_cpu_cxx(b), int(n_opt) * int(paths) * STEPS
    t0 = time.perf_counter()
    if impl == "reference":
        orc.Reference().heston_batch(**b)
    else:
        orc.Oracle().heston_batch(**b)
    dt = time.perf_counter() - t0
    return dt, int(n_opt) * int(paths) * STEPS


def _cos_batch(n=65536):
    """The CF workload's options for the COS pricer at the reference's
    defaults (256 terms, truncation width 10)."""
    from quantkernel_b200 import workloads

    b = workloads.heston_cf(n)
    out = {k: b[k] for k in ("spot", "strike", "t", "r", "q", "v0", "kappa", "theta", "sigma",
                             "rho", "option_type")}
    out["n_terms"] = np.full(n, 256, np.int32)
    out["truncation_width"] = np.full(n, 10.0)
    return out


def _cf_cpu_leg(s):
    """Reference (or oracle) Heston CF or COS batch on a bounded sample of the
    Fourier workload."""
    from oracle import oracle as orc
    from quantkernel_b200 import workloads

    cos = s.get("method") == "cos"
    b = _cos_batch() if cos else workloads.heston_cf()
    cap = len(b["spot"])
    port = orc.Oracle()
    fn = port.heston_cos if cos else port.heston_cf
    n = 16
    while True:
        t0 = time.perf_counter()
        if s["impl"] == "reference":
            ref = orc.Reference()
            (ref.heston_cos_batch if cos else ref.heston_cf_batch)(**{k: v[:n] for k, v in b.items()})
        else:
            for i in range(n):
                fn(*(b[k][i].item() for k in b))
        dt = time.perf_counter() - t0
        if dt >= 0.5 * s["seconds"] or n >= cap:
            break
        n = min(cap, max(2 * n, int(n * s["seconds"] / max(dt, 1e-3))))
    print(json.dumps({"options": n, "seconds": dt}))


VR_METHODS = {8: "control_variates", 9: "importance_sampling", 10: "stratified_sampling",
              11: "quasi_monte_carlo_sobol", 12: "quasi_monte_carlo_halton"}


def _vr_batch(n=64, paths=1 << 20):
    from quantkernel_b200 import workloads

    b = workloads.bsm_terminal(n, paths=paths, seed=11)
    b["shift"] = np.full(n, 0.25)
    return b


def _vr_cpu_leg(s):
    """The reference's OpenMP batch of each variance-reduction method on the
    64-option workload with paths scaled to about s["seconds"] per method."""
    from oracle import oracle as orc

    lib = orc.Reference() if s["impl"] == "reference" else None
    out = {}
    for m, name in VR_METHODS.items():
        paths = 1024
        while True:
            b = _vr_batch(paths=paths)
            t0 = time.perf_counter()
            if lib is not None:
                lib.vr_batch(m, b["spot"], b["strike"], b["t"], b["vol"], b["r"], b["q"],
                             b["option_type"], b["paths"], seed=b["seed"], shift=b["shift"])
            else:
                o = orc.Oracle()
                for i in range(64):
                    o.price(m, b["spot"][i], b["strike"][i], b["t"][i], b["vol"][i], b["r"][i],
                            b["q"][i], int(b["option_type"][i]), int(b["paths"][i]),
                            seed=int(b["seed"][i]), shift=float(b["shift"][i]))
            dt = time.perf_counter() - t0
            if dt >= 0.5 * s["seconds"] or paths >= (1 << 20):
                break
            paths = min(1 << 20, max(2 * paths, int(paths * s["seconds"] / max(dt, 1e-3))))
        out[name] = {"paths_per_option": paths, "seconds": dt, "paths_per_s": 64 * paths / dt}
    print(json.dumps(out))


def _bsm_cpu_leg(s):
    """The reference's qk_mcm_antithetic_variates_price_batch (OpenMP over
    options, FP64) on the 64-option terminal workload, timed from C++, paths
    scaled to about s["seconds"] (cost is linear in paths)."""
    from oracle import oracle as orc
    from quantkernel_b200 import workloads

    paths = 4096
    while True:
        b = workloads.bsm_terminal(64, paths=paths)
        if s["impl"] == "reference" and orc.timer_available():
            dt = _time_cpu_cxx(b, "qk_mcm_antithetic_variates_price_batch")
        else:
            o = orc.Oracle()
            t0 = time.perf_counter()
            for i in range(64):
                o.price(orc.ANTITHETIC, *(b[k][i].item() for k in ("spot", "strike", "t", "vol",
                                                                     "r", "q", "option_type",
                                                                     "paths")),
                        seed=int(b["seed"][i]))
            dt = time.perf_counter() - t0
        if dt >= 0.5 * s["seconds"] or paths >= (1 << 24):
            break
        paths = min(1 << 24, max(2 * paths, int(paths * s["seconds"] / max(dt, 1e-3))))
    print(json.dumps({"paths_per_option": paths, "seconds": dt, "paths": 64 * paths}))


def mixed_cpu_batch(div):
    """The mixed workload with every option's paths divided by `div` (at least
    16): the same options, models, steps and weighting of path-steps by model."""
    from quantkernel_b200 import workloads

    b = workloads.mixed()
    b["paths"] = np.maximum(16, b["paths"] // div).astype(np.int32)
    return b


def _mixed_cpu_leg(s):
    """The reference's own batch entry point per model (Euler-Maruyama,
    Milstein, local vol, Heston; each an OpenMP loop over its options) on the
    mixed workload with paths divided by a factor that brings the four calls
    to about s["seconds"]; timed from C++ and summed."""
    from oracle import oracle as orc

    div = 4096
    while True:
        b = mixed_cpu_batch(div)
        tot, units = 0.0, 0
        per = {}
        for m in np.unique(b["model"]):
            idx = np.nonzero(b["model"] == m)[0]
            sub = {k: v[idx] for k, v in b.items()}
            if s["impl"] == "reference" and orc.timer_available():
                dt = _time_cpu_cxx(sub, orc.MODEL_BATCH_SYMBOL[int(m)])
            else:
                o = orc.Oracle()
                t0 = time.perf_counter()
                if int(m) == orc.HESTON:
                    o.heston_batch(**{k: sub[k] for k in HESTON_KEYS})
                else:
                    o.bsm_family_batch(int(m), *(sub[k] for k in ("spot", "strike", "t", "vol",
                                                                   "r", "q", "option_type",
                                                                   "paths", "steps", "seed")))
                dt = time.perf_counter() - t0
            u = int((sub["paths"].astype(np.int64) * sub["steps"]).sum())
            per[int(m)] = {"seconds": dt, "path_steps": u}
            tot += dt
            units += u
        if tot >= 0.5 * s["seconds"] or div <= 1:
            break
        div = max(1, min(div // 2, int(div * tot / s["seconds"])))
    print(json.dumps({"paths_divisor": div, "seconds": tot, "path_steps": units, "per_model": per}))


def cpu_leg(spec):
    """Runs in a subprocess with OMP_NUM_THREADS set; prints one JSON line."""
    s = json.loads(spec)
    if s.get("kind") == "heston_cf":
        return _cf_cpu_leg(s)
    if s.get("kind") == "vr":
        return _vr_cpu_leg(s)
    if s.get("kind") == "bsm":
        return _bsm_cpu_leg(s)
    if s.get("kind") == "mixed":
        return _mixed_cpu_leg(s)
    target = s["seconds"]
    reps = s.get("reps", 1)
    n_opt, paths = 8, 4096
    dt, units = _time_cpu(s["impl"], n_opt, paths, s["threads"])  # calibration
    rate = units / max(dt, 1e-9)
    paths = max(1024, min(PATHS, int(rate * target / (64 * STEPS))))
    out = []
    for _ in range(reps):
        dt, units = _time_cpu(s["impl"], 64, paths, s["threads"])
        out.append({"seconds": dt, "path_steps": units})
    print(json.dumps({"samples": out, "n_opt": 64, "paths": paths}))


def run_cpu(impl, threads, seconds, reps=1, kind="heston_mc", **extra):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    spec = json.dumps({"impl": impl, "threads": threads, "seconds": seconds, "reps": reps,
                       "kind": kind, **extra})
    r = subprocess.run([sys.executable, str(Path(__file__).resolve()), "--cpu-leg", spec],
                       env=env, capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(f"cpu leg failed: {r.stderr[-2000:]}")
    return json.loads(r.stdout.strip().splitlines()[-1])


def cpu_kind():
    from oracle import oracle as orc

    return "reference" if orc.reference_available() else "port"


def cpu_timer_name():
    return ("C++ std::chrono::steady_clock around the batch call (oracle/cpu_timer.cpp)"
            if cpu_kind() == "reference" and CPU_TIMER.exists() else
            "Python time.perf_counter around the batch call")


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), for the baseline record."""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    kind = cpu_kind()
    threads = host_threads()
    res = run_cpu(kind, threads, seconds=max(1.0, 150.0 / (args.steps + args.warmup)),
                  reps=args.steps + args.warmup)
    timed = res["samples"][args.warmup:]
    secs = sum(x["seconds"] for x in timed)
    units = sum(x["path_steps"] for x in timed)
    value = units / secs
    sample = (f"64 options of the workload, {res['paths']} paths x {STEPS} steps per step "
              f"({64 * res['paths'] * STEPS:.3g} path-steps)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * secs / max(len(timed), 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "options": N_OPT, "paths": PATHS, "steps": STEPS,
                   "cpu_sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "cpu_model": cpu_model(), "timer": cpu_timer_name(), "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "prices_per_sec": value / (PATHS * STEPS),
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        import tempfile

        try:
            fd, name = tempfile.mkstemp(prefix=f"qk_clocks_gpu{self.index}_", suffix=".csv")
            self.path = Path(name)
            self.fh = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.index)], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        text = self.path.read_text()
        self.path.unlink(missing_ok=True)
        for line in text.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, flag in zip(names, f[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "samples": len(sm), "reasons": sorted(reasons)}


# --------------------------------------------------------------------------- GPU arm
NCU_FIGURES = ("dram_bytes_per_launch_full", "thread_instructions_per_path_step",
               "xu_per_path_step", "issue_busy", "xu_pipe_busy")


def ncu_figures(path=None):
    """The `<key>: <number>` lines of the committed ncu summary of the Heston
    simulate kernel (the figures the roofline block reports), as floats."""
    path = Path(path) if path else ROOT / "profiles" / "heston_simulate_ncu.md"
    out = {}
    if path.exists():
        for line in path.read_text().splitlines():
            key, sep, val = line.partition(":")
            if sep and key in NCU_FIGURES:
                out[key] = float(val)
    return out


def main_gpu(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    from quantkernel_b200 import (QK_MC_HESTON, QK_PLAN_AUTOTUNE, QK_PLAN_TIMING, QuantKernel,
                                  workloads)

    qk = QuantKernel()
    qk.set_device(local)
    pipes = measure_pipes(qk, local)  # the rooflines' measured denominators
    # one batch split across all ranks (run first, while every rank still
    # builds plans at the default launch shape: the ranks' tilings must agree)
    strong = None
    if not args.profile:
        strong = sharded_leg(qk, world, rank, dev, args.steps, args.warmup)
    n_opt = args.options
    h = workloads.heston(n_opt, paths=PATHS, steps=STEPS, seed=2 + 1000 * rank,
                         seed_base=5000 + 10_000_000 * rank)
    units_per_step = int(n_opt) * PATHS * STEPS
    # a dedicated (non-default) stream: the plan's kernels, the L2 flush and the
    # timing events are all ordered on it
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    # the autotuner picks block size, paths per thread and step unrolling by
    # timing each candidate (best of three, before the timed region);
    # --profile keeps the default shape so that an ncu capture sees the
    # launch it names
    plan = qk.plan(model=np.full(n_opt, QK_MC_HESTON, np.int32),
                   flags=QK_PLAN_TIMING | (0 if args.profile else QK_PLAN_AUTOTUNE), **h)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # ---- value: device-resident
    for _ in range(args.warmup):
        flush.zero_()
        plan.execute(stream.cuda_stream)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    kern_ms = []
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        flush.zero_()
        plan.execute(stream.cuda_stream)
        kern_ms.append(plan.stats()["simulate_ms"])
    ev1.record(stream)
    barrier()
    clk = clocks.stop()
    total_ms = ev0.elapsed_time(ev1)
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    prices, se = plan.results()
    plan_cfg = plan.config()
    assert np.all(np.isfinite(prices)) and np.all(se > 0), "non-finite result"
    launches = plan.stats()["launches"] * args.steps
    if args.profile:
        if world > 1:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"profile": True, "options": n_opt, "ms_per_step": total_ms / args.steps,
                              "simulate_ms": statistics.mean(kern_ms)}), flush=True)
        return 0

    # ---- e2e: drop-in C call with host buffers
    for _ in range(max(1, args.warmup // 2)):
        qk.heston_monte_carlo_price_batch(**h)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        out = qk.heston_monte_carlo_price_batch(**h)
    barrier()
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_s = float(te.item())
    assert np.allclose(out, prices, rtol=1e-12, atol=0), "e2e result differs from plan result"

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0

    value = world * units_per_step * args.steps / (total_ms / 1e3)
    sim_ms = statistics.mean(kern_ms)
    f_mhz = clk.get("sm_mhz") or 1965.0
    roofline = step_roofline({6: units_per_step}, sim_ms / 1e3, f_mhz)
    roofline.update({
        "kernel": ("mc_simulate_kernel<Heston,{block},{units_per_thread},antithetic,"
                   "step_unroll {step_unroll}>").format(**plan_cfg),
        "launch_config": {**plan_cfg,
                          "chosen_by": "autotuner (block x paths per thread x step unrolling)"},
        "kernel_ms": sim_ms,
        "measured": {"source": "ncu, profiles/heston_simulate_ncu.md"},
        "pipe_probe": pipes,
    })
    # DRAM bytes per full launch, from the committed ncu summary (a small case
    # of the same kernel scaled by the option count; see that file)
    figs = ncu_figures()
    if "dram_bytes_per_launch_full" in figs:
        roofline["traffic"] = int(figs.pop("dram_bytes_per_launch_full")) * n_opt // N_OPT
    roofline["measured"].update(figs)
    m = roofline["measured"]
    if "thread_instructions_per_path_step" in m and "xu_per_path_step" in m:
        # the same peaks against this kernel's own (ncu-measured) instruction
        # mix: how close the kernel runs to what its own instructions allow
        issue_peak = SMS * PIPES["issue"] * f_mhz * 1e6
        xu_peak = SMS * PIPES["xu"] * f_mhz * 1e6
        own = min(issue_peak / m["thread_instructions_per_path_step"],
                  xu_peak / m["xu_per_path_step"])
        roofline["frac_of_own_mix_bound"] = (units_per_step / (sim_ms / 1e3)) / own

    threads = host_threads()
    try:
        if world > 1:  # measured once, at N = 1; all N GPUs stay held meanwhile
            raise RuntimeError("measured in the 1-GPU run only")
        cres = run_cpu(cpu_kind(), threads, seconds=10.0)
        cs = cres["samples"][0]
        cpu_value = cs["path_steps"] / cs["seconds"]
        cpu = {"value": cpu_value, "unit": UNIT, "cores": threads, "kind": cpu_kind(),
               "cpu_model": cpu_model(), "timer": cpu_timer_name(),
               "sample": f"64 options x {cres['paths']} paths x {STEPS} steps of the workload"}
        c1 = run_cpu(cpu_kind(), 1, seconds=4.0)["samples"][0]
        cpu["value_1_core"] = c1["path_steps"] / c1["seconds"]
    except Exception as exc:  # the CPU baseline never blocks the GPU line
        cpu = {"value": None, "unit": UNIT, "cores": threads, "kind": cpu_kind(),
               "sample": (f"skipped: {exc}" if world > 1 else f"failed: {exc}")[:200]}

    extras = {}
    try:
        if world > 1:  # the secondary 1-GPU workloads run in the N = 1 line only
            raise RuntimeError("secondary legs run in the 1-GPU run only")
        extras["mixed"] = mixed_leg(qk, f_mhz=f_mhz)
        extras["bsm_terminal"] = bsm_terminal_leg(qk, f_mhz=f_mhz)
        extras["heston_cf"] = heston_cf_leg(qk)
        extras["variance_reduction"] = vr_leg(qk)
        if Path(args.sur_checkpoint).exists():
            extras["surrogate"] = surrogate_infer_leg(qk, args.sur_checkpoint,
                                                      mc_prices_per_s=value / (PATHS * STEPS))
    except Exception as exc:  # secondary workloads never block the headline line
        if world > 1:
            extras["secondary"] = f"skipped: {exc}"
        else:
            extras["secondary_error"] = f"{type(exc).__name__}: {exc}"[:300]

    h2d = n_opt * 128 + (n_opt + 1) * 8  # packed option records + tile offsets
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "options_per_gpu": n_opt, "paths": PATHS,
                   "steps": STEPS, "antithetic": True, "accumulate": "f64 double-double",
                   "l2": "flushed between steps (256 MiB write inside the timed region)",
                   "parallelism": f"dp{world} (options sharded per rank, no collective)"},
        "prices_per_sec": world * n_opt * args.steps / (total_ms / 1e3),
        "e2e": {"value": world * units_per_step * args.steps / e2e_s, "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": n_opt * 8,
                "api": "qk_mcm_heston_monte_carlo_price_batch (host buffers)"},
        "gpu_launches": launches,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clk,
        "strong_scaling": strong,
        **extras,
    }
    print(json.dumps(line), flush=True)
    return 0


def sharded_leg(qk, world, rank, dev, steps, warmup):
    """Strong scaling through the library's own multi-GPU path: the same
    1024-option Heston batch on every rank, each rank simulating its share of
    the tiles (qk_mcm_plan_execute_sharded: NCCL exchange of the tile sums,
    finalize on every rank).  Timed with CUDA events, max over ranks; at one
    GPU the results are checked against a plain execute bit for bit."""
    import torch
    import torch.distributed as dist

    from quantkernel_b200 import QK_MC_HESTON, workloads
    from quantkernel_b200.sharding import DistContext, new_id

    ident = new_id(qk) if rank == 0 else None
    if world > 1:
        obj = [ident]
        dist.broadcast_object_list(obj, src=0)
        ident = obj[0]
    ctx = DistContext(ident, world, rank, qk)
    h = workloads.heston(N_OPT, paths=PATHS, steps=STEPS)
    plan = qk.plan(model=np.full(N_OPT, QK_MC_HESTON, np.int32), **h)
    # a dedicated stream: the flush, the plan's kernels, the exchange and the
    # timing events are all ordered on it
    stream = torch.cuda.Stream(dev)
    assert stream.cuda_stream != 0
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    with torch.cuda.stream(stream):
        for _ in range(warmup):
            flush.zero_()
            ctx.execute(plan, stream.cuda_stream)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            flush.zero_()
            ctx.execute(plan, stream.cuda_stream)
        e1.record(stream)
        barrier()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item()) / steps
    p, se = plan.results()
    same = None
    if world == 1:
        plan.execute()
        p1, se1 = plan.results()
        same = bool(np.array_equal(p, p1) and np.array_equal(se, se1))
        assert same, "sharded execute differs from execute"
    bounds = plan.shard_bounds(world)
    plan.close()
    ctx.close()
    units = N_OPT * PATHS * STEPS
    return {"workload": WORKLOAD + " (one batch for all ranks)", "n_gpus": world,
            "value": units / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "scaling": "strong",
            "api": "qk_mcm_plan_execute_sharded (NCCL broadcast of tile sums, finalize on every "
                   "rank)",
            "tiles_per_rank": [int(b) for b in np.diff(bounds)],
            "equals_single_gpu_bitwise": same,
            "l2": "flushed between steps"}


# --------------------------------------------------------------------------- surrogate
def _sur_label(qk, n, paths, steps, seed, chunk):
    """Features, price/S and SE/S of n box-uniform Heston calls priced by the GPU MC."""
    from quantkernel_b200.surrogate import features_of, sample_box

    b = sample_box(n, seed)
    price = np.empty(n)
    se = np.empty(n)
    for i0 in range(0, n, chunk):
        sl = slice(i0, min(n, i0 + chunk))
        m = sl.stop - sl.start
        price[sl], se[sl] = qk.heston_monte_carlo_price_se_batch(
            *(b[k][sl] for k in ("spot", "strike", "t", "r", "q", "v0", "kappa", "theta", "sigma", "rho")),
            np.zeros(m, np.int32), np.full(m, paths, np.int32), np.full(m, steps, np.int32),
            np.arange(sl.start, sl.stop, dtype=np.uint64) + np.uint64(seed << 32))
    f = features_of(*(b[k] for k in ("spot", "strike", "t", "r", "q", "v0", "kappa", "theta", "sigma", "rho")))
    return f, price / b["spot"], se / b["spot"], b


def surrogate_train_leg(args):
    """Training workload: 4e6 tuples labelled at 200 x 65536, hold-out 1e5 at
    200 x 1048576, MLP trained with Adam (lr 1e-3 cosine, batch 8192) on the
    residual over the Black-Scholes mean-variance base."""
    import torch

    from quantkernel_b200 import QuantKernel
    from quantkernel_b200.surrogate import HestonSurrogate

    torch.cuda.set_device(0)
    qk = QuantKernel()
    qk.set_device(0)
    t0 = time.perf_counter()
    f, y, se, _ = _sur_label(qk, args.sur_train_n, 65536, 200, seed=31, chunk=65536)
    t_label = time.perf_counter() - t0
    t0 = time.perf_counter()
    hf, hy, hse, _ = _sur_label(qk, args.sur_hold_n, 1048576, 200, seed=32, chunk=16384)
    t_hold = time.perf_counter() - t0
    sur = HestonSurrogate(qk, seed=2024)
    sur.set_dataset(f, y)
    t0 = time.perf_counter()
    losses = sur.train(epochs=args.sur_epochs, batch=8192, lr=1e-3, shuffle_seed=7)
    t_train = time.perf_counter() - t0
    err = np.abs(sur.predict(hf) - hy)
    Path(args.sur_checkpoint).parent.mkdir(parents=True, exist_ok=True)
    sur.save(args.sur_checkpoint)
    steps = args.sur_epochs * (args.sur_train_n // 8192)
    flop = steps * 8192 * SUR_FLOP_PER_ROW * 3  # forward + backward (2x forward)
    out = {
        "leg": "surrogate_train", "train_n": args.sur_train_n, "hold_n": args.sur_hold_n,
        "label_seconds": t_label, "label_path_steps_per_s": args.sur_train_n * 65536 * 200 / t_label,
        "holdout_label_seconds": t_hold, "epochs": args.sur_epochs, "optimizer_steps": steps,
        "train_seconds": t_train, "ms_per_step": 1e3 * t_train / steps,
        "train_tflops": flop / t_train / 1e12,
        "epoch_loss_first_last": [float(losses[0]), float(losses[-1])],
        "holdout_abs_err_over_S": {"mean": float(err.mean()), "p50": float(np.median(err)),
                                   "p99": float(np.quantile(err, 0.99)), "max": float(err.max()),
                                   "frac_le_5e-4": float((err <= 5e-4).mean())},
        "holdout_label_se_over_S_mean": float(hse.mean()),
        "checkpoint": str(args.sur_checkpoint),
    }
    print(json.dumps(out), flush=True)
    return out


def surrogate_infer_leg(qk, checkpoint, n_query=1_000_000, n_judge=10_000, mc_prices_per_s=None):
    """Inference workload: 1e6 queries (90% in the training box, 10% with one
    parameter pushed up to 20% of its range outside), out-of-box queries priced
    by plain GPU MC (200 x 262144); 1e4 in-box queries re-priced by MC judge the
    surrogate's error."""
    import torch

    from quantkernel_b200.surrogate import (HESTON_BOX_HI, HESTON_BOX_LO, HestonSurrogate,
                                            features_of, sample_box)

    sur = HestonSurrogate(qk, seed=0)
    sur.load(checkpoint)
    rng = np.random.default_rng(41)
    b = sample_box(n_query, seed=40)
    out_mask = rng.uniform(size=n_query) < 0.10
    dims = np.array(["strike", "t", "r", "v0", "kappa", "theta", "sigma", "rho"])
    cols = {"strike": 0, "t": 1, "r": 2, "v0": 4, "kappa": 5, "theta": 6, "sigma": 7, "rho": 8}
    for i in np.nonzero(out_mask)[0]:
        d = dims[rng.integers(len(dims))]
        c = cols[d]
        lo, hi = HESTON_BOX_LO[c], HESTON_BOX_HI[c]
        push = rng.uniform(0.0, 0.2) * (hi - lo)
        if d == "strike":  # feature is S/K: push S/K outside, keep S
            sk = (hi + push) if rng.uniform() < 0.5 else max(lo - push, 1e-3)
            b["strike"][i] = b["spot"][i] / sk
        else:
            v = (hi + push) if rng.uniform() < 0.5 else (lo - push)
            if d in ("v0", "kappa", "theta", "sigma"):
                v = max(v, 1e-4)
            if d == "rho":
                v = min(max(v, -0.999), 0.999)
            b[d][i] = v
    keys = ("spot", "strike", "t", "r", "q", "v0", "kappa", "theta", "sigma", "rho")
    ot = np.zeros(n_query, np.int32)
    # e2e through the C ABI: routing, surrogate, MC fallback
    sur.price_batch(*(b[k][:2048] for k in keys), ot[:2048], fallback_paths=262144,
                    fallback_steps=200)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    price, src = sur.price_batch(*(b[k] for k in keys), ot, fallback_paths=262144, fallback_steps=200,
                                 fallback_seed=123)
    t_e2e = time.perf_counter() - t0
    n_sur = int((src == 0).sum())
    n_mc = int((src == 1).sum())
    # device-resident surrogate throughput (FP64 features already in HBM:
    # features kernel + fused network)
    f = features_of(*(b[k] for k in keys))
    inbox = src == 0
    feats = torch.from_numpy(np.ascontiguousarray(f[inbox])).cuda()
    dev_s, net_s = _time_sur_device(sur, feats, False)
    sur_dev_rate = feats.shape[0] / dev_s
    # judge: 1e4 in-box queries re-priced by MC at 200 x 262144
    jidx = rng.choice(np.nonzero(inbox)[0], n_judge, replace=False)
    jp, jse = qk.heston_monte_carlo_price_se_batch(
        *(b[k][jidx] for k in keys), np.zeros(n_judge, np.int32), np.full(n_judge, 262144, np.int32),
        np.full(n_judge, 200, np.int32), np.arange(n_judge, dtype=np.uint64) + np.uint64(777))
    err = np.abs(price[jidx] - jp) / b["spot"][jidx]
    # a second judge with 16x the paths (SE / S ~ 5e-5) on 2000 of them: the
    # network's own error, nearly free of the judge's noise
    hidx = jidx[:2000]
    hp, hse = qk.heston_monte_carlo_price_se_batch(
        *(b[k][hidx] for k in keys), np.zeros(hidx.size, np.int32),
        np.full(hidx.size, 4194304, np.int32), np.full(hidx.size, 200, np.int32),
        np.arange(hidx.size, dtype=np.uint64) + np.uint64(991))
    herr = np.abs(price[hidx] - hp) / b["spot"][hidx]
    res = {
        "workload": "1e6 Heston queries, 10% outside the box -> MC 200 x 262144; judge 1e4 at "
                    "200 x 262144 (and 2000 of them at 200 x 4194304)",
        "queries": n_query, "surrogate_priced": n_sur, "mc_fallback": n_mc,
        "e2e_prices_per_s": n_query / t_e2e, "e2e_seconds": t_e2e,
        "surrogate_prices_per_s_device": sur_dev_rate,
        "surrogate_device_note": "FP64 features in HBM -> features kernel (bf16 rows + "
                                 "Black-Scholes base) -> fused network (+ base)",
        "surrogate_network_only_prices_per_s": feats.shape[0] / net_s,
        "surrogate_tflops_device": feats.shape[0] / net_s * SUR_FLOP_PER_ROW / 1e12,
        "judge_abs_err_over_S": {"mean": float(err.mean()), "p50": float(np.median(err)),
                                 "p99": float(np.quantile(err, 0.99)), "max": float(err.max()),
                                 "frac_le_5e-4": float((err <= 5e-4).mean())},
        "judge_se_over_S_mean": float((jse / b["spot"][jidx]).mean()),
        "judge_4m_paths_abs_err_over_S": {"n": int(hidx.size), "mean": float(herr.mean()),
                                          "p99": float(np.quantile(herr, 0.99)),
                                          "max": float(herr.max()),
                                          "frac_le_5e-4": float((herr <= 5e-4).mean()),
                                          "judge_se_over_S_mean": float((hse / b["spot"][hidx]).mean())},
    }
    if mc_prices_per_s:
        res["plain_mc_prices_per_s"] = mc_prices_per_s
        res["surrogate_vs_plain_mc"] = sur_dev_rate / mc_prices_per_s
        res["e2e_vs_plain_mc"] = res["e2e_prices_per_s"] / mc_prices_per_s
    sur.close()
    return res


def _time_plan(plan, stream, flush, reps):
    import torch

    for _ in range(2):
        flush.zero_()
        plan.execute(stream.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tot = 0.0
    for _ in range(reps):
        flush.zero_()
        e0.record(stream)
        plan.execute(stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
    return tot / reps


def step_roofline(units_by_model, seconds, f_mhz):
    """Roofline of the stepwise simulate kernels: each model's path-steps at the
    tighter of its XU and issue bounds (STEP_COST, the PIPES per-clock SM widths
    at the sampled SM clock); frac = that bound time / the measured time."""
    issue_peak = SMS * PIPES["issue"] * f_mhz * 1e6  # thread-instructions/s
    xu_peak = SMS * PIPES["xu"] * f_mhz * 1e6
    bound_s, xu_ops, alu_ops, limiters = 0.0, 0.0, 0.0, set()
    for model, units in units_by_model.items():
        xu, alu = STEP_COST[int(model)]
        xu_b, alu_b = xu_peak / xu, issue_peak / alu
        limiters.add("xu" if xu_b <= alu_b else "alu")
        bound_s += units / min(xu_b, alu_b)
        xu_ops += units * xu
        alu_ops += units * alu
    bound = limiters.pop() if len(limiters) == 1 else "xu+alu"
    ops, peak = (xu_ops, xu_peak) if bound == "xu" else (alu_ops, issue_peak)
    out = {"bound": bound, "unit": "Gop/s", "frac": bound_s / seconds, "traffic": None,
           "per_unit": {str(m): {"xu": STEP_COST[int(m)][0], "alu": STEP_COST[int(m)][1]}
                        for m in units_by_model},
           "unit_of_work": "path-step (antithetic pairs share normals)",
           "bound_ms": 1e3 * bound_s, "sm_mhz": f_mhz,
           "peak_source": (PIPES["source"] + " at the SM clock sampled during the timed "
                           "region; the HBM-copy and bf16-GEMM peaks do not bound this kernel"),
           "pipe_widths_per_sm_clk": {k: PIPES[k] for k in ("issue", "xu", "fp64")}}
    if bound in ("xu", "alu"):
        out["achieved"] = ops / seconds / 1e9
        out["peak"] = peak / 1e9
    else:  # mixed limiters: report the time-weighted fraction only
        out["achieved"] = out["frac"]
        out["peak"] = 1.0
        out["unit"] = "fraction of the per-model bound time"
    return out


def _time_plan_kernel(plan, stream, flush, reps):
    """(ms per execute, ms of the simulate kernels) of a plan built with
    QK_PLAN_TIMING and no graph, CUDA events on `stream`, L2 flushed."""
    import torch

    for _ in range(3):
        flush.zero_()
        plan.execute(stream.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tot, kern = 0.0, 0.0
    for _ in range(reps):
        flush.zero_()
        e0.record(stream)
        plan.execute(stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
        kern += plan.stats()["simulate_ms"]
    return tot / reps, kern / reps


def mixed_leg(qk, reps=5, f_mhz=1965.0, cpu=True):
    """Uneven batch: 4096 options, BSM-Euler / Milstein / local vol / Heston
    1:1:1:1, paths log-uniform 2^12..2^20, steps 16..512, as one plan in a
    CUDA graph: the persistent work-stealing kernel, per-family grids, and the
    autotuner's choice between them; against one plan per model back to back."""
    import torch

    from quantkernel_b200 import (QK_PLAN_AUTOTUNE, QK_PLAN_FAMILY_GRIDS, QK_PLAN_GRAPH,
                                  QK_PLAN_PERSISTENT, QK_PLAN_TIMING, workloads)

    b = workloads.mixed()
    units = workloads.path_steps(b)
    stream = torch.cuda.current_stream()
    assert stream.cuda_stream != 0, "time on a non-default stream"
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    plan = qk.plan(**b, flags=QK_PLAN_PERSISTENT | QK_PLAN_GRAPH | QK_PLAN_TIMING)
    ms_pers = _time_plan(plan, stream, flush, reps)
    p_pers, _ = plan.results()
    plan.close()
    plan = qk.plan(**b, flags=QK_PLAN_FAMILY_GRIDS | QK_PLAN_GRAPH | QK_PLAN_TIMING)
    ms_grids = _time_plan(plan, stream, flush, reps)
    plan.close()
    plan = qk.plan(**b, flags=QK_PLAN_GRAPH | QK_PLAN_AUTOTUNE | QK_PLAN_TIMING)
    ms = _time_plan(plan, stream, flush, reps)
    cfg = plan.config()
    plan.close()
    per_model = 0.0
    out = np.empty(len(b["model"]))
    for m in np.unique(b["model"]):
        idx = np.nonzero(b["model"] == m)[0]
        sub = qk.plan(**{k: v[idx] for k, v in b.items()})
        per_model += _time_plan(sub, stream, flush, reps)
        out[idx] = sub.results()[0]
        sub.close()
    assert np.allclose(out, p_pers, rtol=1e-12, atol=0)
    # a small uneven batch (the first 48 options): per-family grids of a few
    # waves each leave tails that the persistent kernel's work stealing fills
    small = {k: v[:48] for k, v in b.items()}
    sm = {}
    for name, fl in (("persistent_graph_ms", QK_PLAN_PERSISTENT),
                     ("family_grids_graph_ms", QK_PLAN_FAMILY_GRIDS),
                     ("autotuned_graph_ms", QK_PLAN_AUTOTUNE)):
        plan = qk.plan(**small, flags=fl | QK_PLAN_GRAPH | QK_PLAN_TIMING)
        sm[name] = _time_plan(plan, stream, flush, reps)
        if fl == QK_PLAN_AUTOTUNE:
            sm["launch_config"] = plan.config()
        plan.close()
    sm["workload"] = (f"the first 48 options of the batch, "
                      f"{workloads.path_steps(small):.3g} path-steps")
    # kernel time of the autotuned launch (no graph: events around the
    # simulate kernels only) for the roofline
    plan = qk.plan(**b, flags=QK_PLAN_AUTOTUNE | QK_PLAN_TIMING)
    _, kern_ms = _time_plan_kernel(plan, stream, flush, reps)
    plan.close()
    by_model = {int(m): workloads.path_steps({k: v[b["model"] == m] for k, v in b.items()})
                for m in np.unique(b["model"])}
    roof = step_roofline(by_model, kern_ms / 1e3, f_mhz)
    roof["kernel_ms"] = kern_ms
    res = {"workload": "4096 options, Euler/Milstein/local-vol/Heston 1:1:1:1, paths 2^U[12,20], "
                       "steps 2^U[4,9]", "path_steps": units,
           "autotuned_graph_ms": ms, "path_steps_per_s": units / (ms / 1e3),
           "persistent_graph_ms": ms_pers, "family_grids_graph_ms": ms_grids,
           "per_model_plans_ms": per_model, "speedup_vs_per_model": per_model / ms,
           "launch_config": cfg,
           "launch_config_note": "units_per_thread 0 = persistent kernel, -1 = one grid per "
                                 "family group",
           "small_batch": sm,
           "roofline": roof}
    if cpu:
        res["cpu_baseline"] = _rate_baseline("mixed", "path_steps", "path-steps/s", 10.0, 4.0,
                                             lambda c: (f"the 4096 options with paths divided by "
                                                        f"{c['paths_divisor']} (at least 16): "
                                                        f"{c['path_steps']:.3g} path-steps, one "
                                                        f"reference batch call per model"))
    return res


def _rate_baseline(kind, units_key, unit, seconds, seconds_1core, describe):
    """A CPU-leg rate on all host threads and on one core, as a cpu_baseline
    record; never raises (the GPU line is printed either way)."""
    threads = host_threads()
    try:
        c = run_cpu(cpu_kind(), threads, seconds=seconds, kind=kind)
        out = {"value": c[units_key] / c["seconds"], "unit": unit, "cores": threads,
               "kind": cpu_kind(), "cpu_model": cpu_model(), "timer": cpu_timer_name(),
               "sample": describe(c)}
        c1 = run_cpu(cpu_kind(), 1, seconds=seconds_1core, kind=kind)
        out["value_1_core"] = c1[units_key] / c1["seconds"]
        out["sample_1_core"] = describe(c1)
        return out
    except Exception as exc:
        return {"value": None, "unit": unit, "cores": threads, "kind": cpu_kind(),
                "sample": f"failed: {exc}"[:200]}


def bsm_terminal_leg(qk, reps=20, f_mhz=1965.0, cpu=True):
    """64 BSM options x 131072 paths, terminal GBM with antithetic pairs in
    FP64 (FP64 normals and exponent, as the reference's make_bsm_terminal):
    device time of a graph-replayed plan, the simulate kernel alone, end to
    end through qk_mcm_antithetic_variates_price_batch with host buffers, and
    the reference's own antithetic batch on the host cores."""
    import torch

    from quantkernel_b200 import QK_MC_ANTITHETIC, QK_PLAN_GRAPH, QK_PLAN_TIMING, workloads

    b = workloads.bsm_terminal()
    n = len(b["spot"])
    stream = torch.cuda.current_stream()
    assert stream.cuda_stream != 0, "time on a non-default stream"
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    plan = qk.plan(model=np.full(n, QK_MC_ANTITHETIC, np.int32), flags=QK_PLAN_GRAPH, **b)
    ms = _time_plan(plan, stream, flush, reps)
    plan.close()
    plan = qk.plan(model=np.full(n, QK_MC_ANTITHETIC, np.int32), flags=QK_PLAN_TIMING, **b)
    _, kern_ms = _time_plan_kernel(plan, stream, flush, reps)
    plan.close()
    args = [b[k] for k in ("spot", "strike", "t", "vol", "r", "q", "option_type", "paths", "seed")]
    qk.antithetic_variates_price_batch(*args)
    t0 = time.perf_counter()
    for _ in range(reps):
        qk.antithetic_variates_price_batch(*args)
    e2e = (time.perf_counter() - t0) / reps
    paths = int(b["paths"].sum())
    pairs = paths // 2
    fp64_peak = SMS * PIPES["fp64"] * f_mhz * 1e6
    res = {"workload": "64 BSM calls/puts x 131072 paths (terminal GBM, antithetic pairs)",
           "dtype": "f64", "ms": ms, "paths_per_s": paths / (ms / 1e3), "e2e_ms": 1e3 * e2e,
           "e2e_paths_per_s": paths / e2e, "api": "qk_mcm_antithetic_variates_price_batch",
           "h2d_bytes": n * 128 + (n + 1) * 8, "d2h_bytes": n * 8,
           "roofline": {"bound": "fp64", "unit": "GFLOP/s",
                        "achieved": pairs * FP64_PER_PAIR / (kern_ms / 1e3) / 1e9,
                        "peak": fp64_peak / 1e9,
                        "frac": pairs * FP64_PER_PAIR / (kern_ms / 1e3) / fp64_peak,
                        "traffic": None, "kernel_ms": kern_ms,
                        "per_unit": {"fp64_ops": FP64_PER_PAIR, "unit": "antithetic pair"},
                        "peak_source": PIPES["source"] + " at the sampled SM clock (FP64 lanes)"}}
    if cpu:
        res["cpu_baseline"] = _rate_baseline(
            "bsm", "paths", "paths/s", 6.0, 3.0,
            lambda c: f"the 64 options with {c['paths_per_option']} paths each "
                      f"(qk_mcm_antithetic_variates_price_batch)")
    return res


def _time_sur_device(sur, feats, layered, reps=10):
    """Seconds per pass of device-resident inference over the FP64 feature
    rows `feats` (torch, n x 9, on the GPU): the features kernel (normalised
    bf16 rows + base) then the network, CUDA events on a dedicated stream.
    Returns (pipeline seconds, network-only seconds)."""
    import torch

    n = feats.shape[0]
    st = torch.cuda.Stream()
    rows = torch.empty((n, 64), dtype=torch.int16, device="cuda")
    base = torch.empty(n, dtype=torch.float32, device="cuda")
    y = torch.empty(n, dtype=torch.float32, device="cuda")

    def feat():
        sur.features_device(feats.data_ptr(), n, rows.data_ptr(), base.data_ptr(), st.cuda_stream)

    def net():
        sur.predict_device(rows.data_ptr(), base.data_ptr(), n, y.data_ptr(), st.cuda_stream,
                           layered=layered)

    out = []
    with torch.cuda.stream(st):
        for fns in ((feat, net), (net,)):
            for _ in range(3):
                for fn in fns:
                    fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(reps):
                for fn in fns:
                    fn()
            e1.record(st)
            st.synchronize()
            out.append(e0.elapsed_time(e1) / 1e3 / reps)
    return out[0], out[1]


def surrogate_device_leg(qk, checkpoint, n_rows):
    """Device-resident inference on n_rows box-uniform normalised rows: the
    fused kernel and the layer-by-layer GEMMs, CUDA events on a dedicated
    stream."""
    import torch

    from quantkernel_b200.surrogate import HestonSurrogate, features_of, sample_box

    sur = HestonSurrogate(qk, seed=0)
    sur.load(checkpoint)
    b = sample_box(n_rows, 99)
    f = features_of(*(b[k] for k in ("spot", "strike", "t", "r", "q", "v0", "kappa", "theta",
                                      "sigma", "rho")))
    feats = torch.from_numpy(f).cuda()
    pipe, fused = _time_sur_device(sur, feats, False)
    _, layered = _time_sur_device(sur, feats, True)
    return {"rows": n_rows, "pipeline_ms": 1e3 * pipe, "pipeline_prices_per_s": n_rows / pipe,
            "features_ms": 1e3 * (pipe - fused),
            "fused_ms": 1e3 * fused, "fused_prices_per_s": n_rows / fused,
            "fused_tflops": n_rows / fused * SUR_FLOP_PER_ROW / 1e12,
            "layered_ms": 1e3 * layered, "layered_prices_per_s": n_rows / layered}


def vr_leg(qk, reps=5, cpu=True):
    """64 BSM calls/puts x 2^20 paths for each terminal variance-reduction
    estimator: device time of a graph-replayed plan (L2 flushed), end to end
    through the drop-in batch call, and the reference's OpenMP batch on a
    bounded sample."""
    import torch

    from quantkernel_b200 import QK_PLAN_GRAPH, QK_PLAN_TIMING

    b = _vr_batch()
    n = len(b["spot"])
    paths = int(b["paths"].sum())
    stream = torch.cuda.current_stream()
    assert stream.cuda_stream != 0, "time on a non-default stream"
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    res = {"workload": f"{n} BSM calls/puts x 2^20 paths, shift 0.25 (importance sampling)"}
    for m, name in VR_METHODS.items():
        arr = {k: b[k] for k in ("spot", "strike", "t", "vol", "r", "q", "option_type", "paths",
                                 "seed")}
        plan = qk.plan(model=np.full(n, m, np.int32), v0=b["shift"],
                       flags=QK_PLAN_GRAPH | QK_PLAN_TIMING, **arr)
        ms = _time_plan(plan, stream, flush, reps)
        plan.close()
        fn = getattr(qk, name + "_price_batch")
        args = [b[k] for k in ("spot", "strike", "t", "vol", "r", "q", "option_type", "paths")]
        if m == 9:
            args.append(b["shift"])
        if m not in (11, 12):
            args.append(b["seed"])
        fn(*args)
        t0 = time.perf_counter()
        for _ in range(reps):
            fn(*args)
        e2e = (time.perf_counter() - t0) / reps
        res[name] = {"ms": ms, "paths_per_s": paths / (ms / 1e3), "e2e_ms": 1e3 * e2e,
                     "e2e_paths_per_s": paths / e2e}
    if cpu:
        try:
            threads = host_threads()
            c = run_cpu(cpu_kind(), threads, seconds=2.0, kind="vr")
            for name, v in c.items():
                res[name]["cpu_baseline"] = {"paths_per_s": v["paths_per_s"], "cores": threads,
                                             "kind": cpu_kind(),
                                             "sample": f"64 options x {v['paths_per_option']} paths"}
        except Exception as exc:
            res["cpu_baseline_error"] = f"{exc}"[:200]
    return res


def heston_cf_leg(qk, reps=5, n=65536, cpu=True):
    """65536 Heston calls/puts by the characteristic-function pricer (1024
    Gauss-Legendre nodes on [1e-8, 120], 2048 FP64 characteristic-function
    evaluations per option) through qk_cf_heston_price_cf_batch, and by the
    COS pricer (256 terms, width 10) through
    qk_ftm_cos_fang_oosterlee_heston_price_batch, with host buffers; beside
    each the reference's OpenMP CPU batch on a bounded sample."""
    from quantkernel_b200 import workloads

    def e2e_time(fn, batch):
        for _ in range(2):
            fn(**batch)
        t0 = time.perf_counter()
        for _ in range(reps):
            out = fn(**batch)
        dt = (time.perf_counter() - t0) / reps
        assert np.all(np.isfinite(out))
        return dt

    def cpu_rate(**extra):
        try:
            threads = host_threads()
            c = run_cpu(cpu_kind(), threads, seconds=5.0, kind="heston_cf", **extra)
            return {"value": c["options"] / c["seconds"], "unit": "options/s", "cores": threads,
                    "kind": cpu_kind(), "sample": f"first {c['options']} options of the workload"}
        except Exception as exc:
            return {"value": None, "sample": f"failed: {exc}"[:200]}

    e2e = e2e_time(qk.heston_price_cf_batch, workloads.heston_cf(n))
    res = {"workload": f"{n} Heston calls/puts, CF with 1024 steps, limit 120",
           "e2e_ms": 1e3 * e2e, "e2e_options_per_s": n / e2e,
           "h2d_bytes": n * 128, "d2h_bytes": n * 8}
    e2e = e2e_time(qk.cos_method_fang_oosterlee_heston_price_batch, _cos_batch(n))
    cos = {"workload": f"{n} Heston calls/puts, COS with 256 terms, width 10",
           "e2e_ms": 1e3 * e2e, "e2e_options_per_s": n / e2e,
           "h2d_bytes": n * 128, "d2h_bytes": n * 8}
    if cpu:
        res["cpu_baseline"] = cpu_rate()
        cos["cpu_baseline"] = cpu_rate(method="cos")
    res["cos"] = cos
    return res


def profile_plans(qk, which, n_opt):
    """Small launches for ncu captures: the mixed workload's first n_opt
    options as the persistent kernel, then as per-family grids (two executes
    each), or the FP64 terminal workload (three executes)."""
    import torch

    from quantkernel_b200 import (QK_MC_ANTITHETIC, QK_PLAN_FAMILY_GRIDS, QK_PLAN_PERSISTENT,
                                  workloads)

    out = {"profile": which}
    if which == "mixed":
        b = {k: v[:n_opt] for k, v in workloads.mixed().items()}
        for name, fl in (("persistent", QK_PLAN_PERSISTENT), ("grids", QK_PLAN_FAMILY_GRIDS)):
            plan = qk.plan(**b, flags=fl)
            for _ in range(2):
                plan.execute(torch.cuda.current_stream().cuda_stream)
            out[name] = float(plan.results()[0].sum())
            plan.close()
        out["options"] = n_opt
    else:
        b = workloads.bsm_terminal()
        plan = qk.plan(model=np.full(len(b["spot"]), QK_MC_ANTITHETIC, np.int32), **b)
        for _ in range(3):
            plan.execute(torch.cuda.current_stream().cuda_stream)
        out["price_sum"] = float(plan.results()[0].sum())
        plan.close()
    return out


def main():
    args = parse()
    if args.pipe_probe:
        from quantkernel_b200 import QuantKernel

        qk = QuantKernel()
        runs = [measure_pipes(qk, 0) for _ in range(3)]
        print(json.dumps({"leg": "pipe_probe", "unit": "lane-operations per SM per SM clock",
                          "runs": runs, "nominal": {"issue": ISSUE_PER_CLK, "xu": XU_PER_CLK,
                                                    "fp64": FP64_PER_CLK}}), flush=True)
        return 0 if all(runs) else 1
    if args.surrogate_train:
        surrogate_train_leg(args)
        return 0
    if args.surrogate:
        from quantkernel_b200 import QuantKernel

        qk = QuantKernel()
        print(json.dumps({"leg": "surrogate", **surrogate_infer_leg(qk, args.sur_checkpoint)}), flush=True)
        return 0
    if args.cpu_leg:
        cpu_leg(args.cpu_leg)
        return 0
    if args.sur_device_rows:
        from quantkernel_b200 import QuantKernel

        print(json.dumps({"leg": "surrogate_device", **surrogate_device_leg(
            QuantKernel(), args.sur_checkpoint, args.sur_device_rows)}), flush=True)
        return 0
    if args.vr:
        import torch

        from quantkernel_b200 import QuantKernel

        torch.cuda.set_stream(torch.cuda.Stream())
        leg = vr_leg(QuantKernel(), cpu=not args.profile)
        print(json.dumps({"leg": "variance_reduction", **leg}), flush=True)
        return 0
    if args.mixed or args.bsm:
        import torch

        from quantkernel_b200 import QuantKernel

        torch.cuda.set_stream(torch.cuda.Stream())
        qk = QuantKernel()
        if args.profile:
            print(json.dumps(profile_plans(qk, "mixed" if args.mixed else "bsm", args.options)),
                  flush=True)
        elif args.mixed:
            print(json.dumps({"leg": "mixed", **mixed_leg(qk)}), flush=True)
        else:
            print(json.dumps({"leg": "bsm_terminal", **bsm_terminal_leg(qk)}), flush=True)
        return 0
    if args.heston_cf:
        from quantkernel_b200 import QuantKernel

        leg = heston_cf_leg(QuantKernel(), n=args.cf_options, cpu=not args.profile)
        print(json.dumps({"leg": "heston_cf", **leg}), flush=True)
        return 0
    if args.impl == "reference":
        return reference_arm(args)
    return main_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
