"""HEOM propagation benchmark: ADO-steps/s of the fused FP64 propagator.

Workload (default): transverse-field Ising spin glass, N=6 spins (d=64),
J_ij ~ N(0,1) (seeded splitmix64/Box-Muller), h=1, one Drude-Lorentz bath
per spin (lambda=0.1, gamma=1, T=1), Pade K=2 (18 modes), depth L=4
(max_depth 5) -> 7315 ADOs of 64x64 complex128 (0.479 GB per state),
RK4 (4-term Taylor, Horner form), dt=0.005.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N>1).  A single hierarchy does not shard:
N>1 runs N independent replicas (seed + rank), value = total ADO-steps/s.
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

from helix_b200 import systems as S  # noqa: E402

METRIC = "ADO-steps/s on 1 B200, chosen form vs plain FP64, at rho0 trace-dist <=1e-6"
UNIT = "ADO-steps/s"

CONFIGS = {
    "c2": dict(n=6, depth=4, K=2, h=1.0, dt=0.005, seed=2025,
               workload="spin_glass_d64_L4_K2_7315ados_fp64"),
    "c1": dict(n=4, depth=3, K=2, h=1.0, dt=0.01, seed=2024,
               workload="spin_glass_d16_L3_K2_455ados_fp64"),
    # the reference's compiled default: d=1024, one collective bath (3 modes), 10 ADOs, dt=0.1
    "legacy": dict(legacy=True, dim=1024, workload="legacy_spin_glass_d1024_10ados_fp64"),
    # mixed precision: N=8 (d=256), h=0.5, Pade K=1 (16 modes), depth L=3 -> 969 ADOs, dt=0.005, 500 steps
    "c3": dict(n=8, depth=3, K=1, h=0.5, dt=0.005, seed=2027, mixed=True, error_steps=500,
               workload="spin_glass_d256_L3_K1_969ados_complex64_mixed"),
    # dense H on the tensor cores: the C3 hierarchy (N=8, d=256, K=1, L=3: 969 ADOs, dt=0.005) with
    # H = E + h sum sx + 0.5 G, G a seeded dense Hermitian matrix (every entry non-zero); complex64
    # hierarchy, rho_0 in FP64, commutator as 3-term TF32 split products; error against the FP64 CSR path
    "c3dense": dict(n=8, depth=3, K=1, h=0.5, eps=0.5, dt=0.005, seed=2027, dense=True, error_steps=100,
                    workload="dense_h_d256_L3_K1_969ados_complex64_tf32x3"),
    # learned closure: N=5 (d=32), K=2 (15 modes), L=2 + MLP closure of tier 3; trained on 64 seeds of plain
    # L=5 FP64 runs (dt=0.01, 1000 steps), tested on 16 held-out seeds against plain L=5
    "c5": dict(n=5, K=2, h=1.0, dt=0.01, closure=True, coarse_depth=2, fine_depth=5, train_seeds=64,
               test_seeds=16, traj_steps=1000, every=50, hidden=512, iters=3000, mlp_batch=8192, lr=3e-3,
               time_seeds=4, time_steps=250,
               workload="spin_glass_d32_K2_L2_plus_mlp_closure_vs_L5"),
    # batched disorder average: 512 seeded instances, N in {3,4,5}, L in {2,3,4}, K=2, dt=0.01
    "c4": dict(batch=True, count=512, seed=2026, dt=0.01, workload="disorder_batch_512_N3-5_L2-4_K2_fp64"),
}


def make_problem(cfg: dict, rank: int = 0):
    if cfg.get("legacy"):
        return S.legacy_spin_glass(cfg["dim"])
    if cfg.get("dense"):
        return S.dense_h_problem(cfg["n"], seed=cfg["seed"] + rank, eps=cfg["eps"], h=cfg["h"], depth=cfg["depth"],
                                 K=cfg["K"], dt=cfg["dt"])
    return S.spin_glass(cfg["n"], seed=cfg["seed"] + rank, depth=cfg["depth"], K=cfg["K"], h=cfg["h"],
                        dt=cfg["dt"])


L2_BYTES_NOMINAL = 126 * 2**20  # B200 L2 (the timing code reads the device's own figure)


def workload_config(cfg: dict, p, world: int) -> dict:
    """The `config` object of the JSON line, identical in both arms: it
    describes the workload (one hierarchy per rank), not the implementation."""
    H = p.hierarchy_size()
    full_bytes = H * p.dim * p.dim * 16
    small = full_bytes < L2_BYTES_NOMINAL
    return {"workload": cfg["workload"], "ados": H, "dim": p.dim, "modes": p.modes, "depth_L": p.max_depth - 1,
            "dt": p.dt, "integrator": "RK4 (4-term Taylor, Horner form)",
            "parallelism": f"{world} independent replicas" if world > 1 else "single",
            "l2": ("L2 flushed before every timed step (the state fits in L2; steps timed one by one with "
                   "CUDA events, the flush outside the events)") if small
            else f"inputs larger than L2 (hierarchy {H} x {p.dim} x {p.dim} complex128)"}


def batch_config(cfg: dict, problems, world: int) -> dict:
    """The `config` object of the batched workload, identical in both arms."""
    return {"workload": cfg["workload"], "instances": len(problems),
            "ados": sum(q.hierarchy_size() for q in problems), "dt": cfg["dt"],
            "integrator": "RK4 (4-term Taylor, Horner form)",
            "parallelism": f"instances sharded over {world} rank(s)" if world > 1 else "single",
            "l2": "inputs larger than L2 (all instances' states)"}


def load_peaks() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# reference benchmark record (helix_benchmark_summary.md:61): 10 ADOs / 85.718 ms
LEGACY_PUBLISHED_ADO_STEPS = 10 / 0.085718


def info_kernels_per_stage(ctx) -> int:
    return int(ctx.info.kernels_per_step) // 4


def profiled_traffic(config: str, kernel: str = "fused_kernel") -> float | None:
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{config}_ncu.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    INTERVAL_MS = 50

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[tuple[float, str]] = []
        self.thread = None
        self.t0 = None

    def start(self):
        """Start sampling and return once the first sample has arrived (or
        after 5 s), so that the timed region that follows is covered."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", str(self.INTERVAL_MS)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
            return
        deadline = time.monotonic() + 5.0
        while not self.lines and time.monotonic() < deadline and self.proc.poll() is None:
            time.sleep(0.01)
        self.t0 = time.monotonic()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def stop(self) -> dict:
        """Stop after one more sample has arrived; keep the samples taken
        between start() returning and that sample."""
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        t1 = time.monotonic()
        deadline = t1 + 2.0
        while time.monotonic() < deadline and self.proc.poll() is None and not any(t >= t1 for t, _ in self.lines):
            time.sleep(0.005)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0 = self.t0 if self.t0 is not None else 0.0
        after = [t for t, _ in self.lines if t >= t1]
        t_end = after[0] if after else float("inf")
        for t, ln in self.lines:
            if t < t0 or t > t_end:
                continue
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


class L2Flush:
    """Device timing of single steps with L2 flushed in between: for a state
    smaller than L2 every timed step starts from a cold L2 (the flush buffer,
    twice the L2 size, is written on the same stream between the timed
    events)."""

    def __init__(self, stream, device: int):
        import torch

        self.torch = torch
        self.stream = stream
        l2 = int(getattr(torch.cuda.get_device_properties(device), "L2_cache_size", 0)) or 126 * 2**20
        self.l2_bytes = l2
        self.buf = torch.empty(2 * l2, dtype=torch.uint8, device=f"cuda:{device}")

    def flush(self):
        with self.torch.cuda.stream(self.stream):
            self.buf.zero_()

    def time_steps(self, step_one, steps: int) -> float:
        """Sum of the device times of `steps` calls of step_one() (ms)."""
        torch = self.torch
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, b in ev:
            self.flush()
            a.record(self.stream)
            step_one()
            b.record(self.stream)
        torch.cuda.synchronize()
        return float(sum(a.elapsed_time(b) for a, b in ev))


def stage_kernels_label(ctx, p, packed: bool, per_stage: int) -> str:
    """The kernels one stage of this context launches (from its stage path)."""
    logd = p.dim.bit_length() - 1
    path = ctx.stage_path
    if path == "flip":
        return "comm_kernel + combine_kernel per stage (spin-flip coupling path)"
    if path == "csr":
        return "csr_comm_kernel + csr_combine_kernel per stage (general sparse operators)"
    if path == "band":
        return "band kernels per stage" + (" (Hermitian-packed slabs)" if packed else "")
    if path == "fused":
        k = f"herm_kernel<{logd}>" if packed else f"fused_kernel<{logd}>"
        return k + (" + upterm_kernel" if per_stage == 2 else "") + " per stage" + \
            (" (Hermitian-packed slabs)" if packed else "")
    if path == "small":
        if int(ctx.info.kernels_per_step) == 1:
            return "small_step_kernel per step (d <= 16; the 4 stages in one cooperative launch, grid barriers)"
        return "small_kernel per stage (d <= 16, batched neighbour gathers)"
    return "stage_kernel per stage (generic path)"


def reference_cuda(cfg: dict, p, steps: int) -> dict:
    """Time the reference's own CUDA propagator (oracle/_ref/ref_cuda_propagator:
    its initialize() + develop() with cuSPARSE/cuBLAS, built from its sources for
    sm_100a in FP64) at this workload's work shape: d, modes (one collective
    bath with modes - 1 Pade poles) and depth bound as the workload, on the
    reference's own model (collective V with sigma_x flips, diagonal H).  Same
    ADOs, same neighbour terms per ADO, same integrator; the physics differs
    (the reference fixes its model at compile time).  CUDA events on the
    legacy default stream around K develop() calls after a warm-up step."""
    from oracle import build as ob

    res = {"unit": UNIT, "shape": {"dim": p.dim, "modes": p.modes, "max_depth": p.max_depth, "dt": p.dt}}
    H = p.hierarchy_size()
    k = 3 if H > 1000 else max(3, min(steps, 50))
    out = {}
    for name, binary in (("fp64", ob.REF_CUDA_BIN), ("fp32", ob.REF_CUDA_BIN_FP32)):
        if name == "fp32" and not cfg.get("legacy"):
            continue
        if not os.path.exists(binary):
            out[name] = {"unavailable": f"{os.path.relpath(binary, ROOT)} not built (needs the reference tree)"}
            continue
        env = dict(os.environ, HX_REF_DIM=str(p.dim), HX_REF_KMAX=str(p.modes - 1), HX_REF_JMAX=str(p.max_depth),
                   HX_REF_DT=repr(p.dt), CUBLAS_WORKSPACE_CONFIG=":16:8")
        try:
            r = subprocess.run([binary, "--time", str(k), "--warmup", "1"], env=env, capture_output=True,
                               text=True, timeout=900)
            # the reference prints its own diagnostics on stdout too; the driver's line is the last JSON object
            line = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
        except (subprocess.SubprocessError, ValueError, IndexError) as e:
            out[name] = {"unavailable": f"run failed: {type(e).__name__}"}
            continue
        if r.returncode != 0 or line.get("cuda_error"):
            out[name] = {"unavailable": f"exit {r.returncode}: {line.get('cuda_error', '')}"}
            continue
        out[name] = {"value": line["ado_steps_per_s"], "ms_per_step": line["ms_per_step"],
                     "wall_ms_per_step": line["wall_ms_per_step"], "steps": line["timed_steps"],
                     "ados": line["hierarchy_size"], "init_ms": line["init_ms"],
                     "device_bytes_in_use": line["device_bytes_in_use"]}
    res.update(out)
    return res


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(cfg: dict, steps: int) -> dict:
    """Time the FP64 CPU oracle (the reference has no CPU path) on all host
    threads, then one full step on one thread."""
    from oracle import oracle as O
    p = make_problem(cfg)
    o = O.Oracle(p)
    cores = O.threads()
    o.run(1)  # warm
    t0 = time.perf_counter()
    o.run(steps)
    dt = time.perf_counter() - t0
    size = o.size
    O.set_threads(1)
    t0 = time.perf_counter()
    o.run(1)
    dt1 = time.perf_counter() - t0
    O.set_threads(cores)
    o.close()
    return {"value": size * steps / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} full steps of the {size}-ADO hierarchy ({cfg['workload']}), FP64 oracle, OpenMP",
            "one_core": {"value": size / dt1, "unit": UNIT, "sample": "1 full step on 1 thread"},
            "nproc": os.cpu_count(), "cpu_model": cpu_model()}


REFERENCE_BUDGET_S = 60.0  # timed CPU work of the reference arm
MIN_WINDOWS, MAX_WINDOWS, WINDOW_TARGET_MS = 5, 200, 1000.0  # repeats of the timed --steps window


def timed_steps(step_all, steps: int, budget_s: float = REFERENCE_BUDGET_S) -> tuple[int, float]:
    """Run whole steps until `steps` are done or `budget_s` has passed (at
    least one); returns (steps run, seconds)."""
    done = 0
    t0 = time.perf_counter()
    while done < steps:
        step_all()
        done += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    return done, time.perf_counter() - t0


def run_reference(args, cfg: dict) -> None:
    """The reference arm: the FP64 oracle on the host's threads, whole steps of
    the same workload, timed until --steps steps are done or 60 s of CPU work
    have passed (the line gives the steps timed)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    if cfg.get("batch"):
        # bounded sample of the batch: its first 16 instances of at most 1000 ADOs
        sample = [q for q in S.disorder_batch(cfg["count"], cfg["seed"], dt=cfg["dt"])
                  if q.hierarchy_size() <= 1000][:16]
        ors = [O.Oracle(q) for q in sample]
        for _ in range(args.warmup):
            for o in ors:
                o.run(1)
        n, sec = timed_steps(lambda: [o.run(1) for o in ors], args.steps)
        size = sum(o.size for o in ors)
        for o in ors:
            o.close()
        value = size * n / sec
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": n, "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sec / n,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": batch_config(cfg, S.disorder_batch(cfg["count"], cfg["seed"], dt=cfg["dt"]), args.gpus),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": O.threads(), "kind": "port",
                             "sample": f"{len(sample)} instances (<= 1000 ADOs each), {n} steps; the "
                                       "reference has no CPU path, so its FP64 restatement stands in"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    p = make_problem(cfg)
    o = O.Oracle(p)
    for _ in range(args.warmup):
        o.run(1)
    n, sec = timed_steps(lambda: o.run(1), args.steps)
    value = o.size * n / sec
    threads = O.threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": n, "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sec / n,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(cfg, p, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{n} full steps of the {o.size}-ADO hierarchy; the reference has no "
                                   "CPU path, so its FP64 restatement (oracle/heom_oracle.cpp) stands in"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    o.close()
    print(json.dumps(line), flush=True)


def run_ours(args, cfg: dict) -> None:
    import torch
    import torch.distributed as dist

    from helix_b200 import capi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    p = make_problem(cfg, rank)
    ctx = capi.Context(p)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    H = ctx.size
    state_bytes = int(ctx.info.state_bytes)

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- device-resident throughput (value) --------------------------------
    # a state smaller than L2 is timed step by step with L2 flushed in between
    flusher = L2Flush(stream, local)
    small = H * p.dim * p.dim * 16 < L2_BYTES_NOMINAL  # as workload_config states it
    for _ in range(args.warmup):
        ctx.step(1)
    ctx.sync()
    c0 = ctx.counters()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()

    def window() -> float:
        """Device time (ms) of one window of --steps steps."""
        if small:
            return flusher.time_steps(lambda: ctx.step(1), args.steps)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        ctx.step(args.steps)
        ev1.record(stream)
        ctx.sync()
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1)

    # the --steps window is repeated (every rank the same number of times,
    # fixed by rank 0's first window) until about 1 s of device time has
    # passed, so the clock sampler sees the GPU under load; ms = the median
    # window
    windows = [window()]
    reps = max(MIN_WINDOWS, min(MAX_WINDOWS, int(np.ceil(WINDOW_TARGET_MS / max(windows[0], 1e-3)))))
    if args.windows:
        reps = args.windows
    if world > 1:
        t = torch.tensor([reps], device="cuda")
        dist.broadcast(t, 0)
        reps = int(t.item())
    for _ in range(reps - 1):
        windows.append(window())
    ms = float(np.median(windows))
    clk = clocks.stop()
    del flusher
    c1 = ctx.counters()
    launches = int(c1.kernel_launches - c0.kernel_launches) // len(windows)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    barrier()
    value = world * H * args.steps / (ms / 1000.0)

    # roofline of one stage (one RHS evaluation with its Horner epilogue, all
    # kernels of the stage): the Horner form moves 11 state volumes per step
    # (stage 1: read rho, write u1; stages 2-4: read u, read rho, write)
    stages = 4
    alg_bytes_per_step = (3 * stages - 1) * state_bytes
    # launches per step: one per stage, or one for the whole step (small_step_kernel)
    step_launch = ctx.stage_path == "small" and int(ctx.info.kernels_per_step) == 1
    launches_per_step = 1 if step_launch else stages
    per_launch_bytes = alg_bytes_per_step / launches_per_step
    launch_ms = ms / (args.steps * launches_per_step)
    achieved = per_launch_bytes / (launch_ms / 1000.0) / 1e9
    peak, peak_kind = load_peaks()
    packed = bool(ctx.hermitian_packed)
    kernel = ("small_step_kernel" if step_launch else "small_kernel") if ctx.stage_path == "small" \
        else ("herm_kernel" if packed else "fused_kernel")
    # DRAM bytes of one stage: the stage kernel plus the up-term kernel (committed ncu summaries)
    traffic = profiled_traffic(args.config, kernel)
    traffic_files = [f"profiles/{kernel}_{args.config}_ncu.txt"]
    up_traffic = profiled_traffic(args.config, "upterm_kernel")
    if traffic is not None and up_traffic is not None and info_kernels_per_stage(ctx) == 2:
        traffic += up_traffic
        traffic_files.append(f"profiles/upterm_kernel_{args.config}_ncu.txt")
    slab_elems = p.dim * (p.dim + 1) // 2 if packed else p.dim * p.dim

    # ---- end to end through the C ABI with host buffers (e2e) --------------
    pinned = torch.empty(H * p.dim * p.dim * 2, dtype=torch.float64, pin_memory=True)
    host_state = pinned.numpy().view(np.complex128).reshape(H, p.dim, p.dim)
    host_state[:] = 0
    host_state[0] = S.initial_rho0(p.dim)
    rho_trace = torch.empty(args.steps * p.dim * p.dim * 2, dtype=torch.float64, pin_memory=True).numpy()
    en_trace = np.zeros(args.steps)
    # untimed pass: the library's pinned staging buffers are allocated on first use
    ctx.set_state(host_state)
    ctx.step_trace_into(1, rho_trace, en_trace)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.set_state(host_state)
    ctx.step_trace_into(args.steps, rho_trace, en_trace)
    final = ctx.rho0()
    e2e_sec = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_sec], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_sec = float(t.item())
    e2e_value = world * H * args.steps / e2e_sec
    assert np.isfinite(final).all() and np.isfinite(en_trace).all()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(cfg, args.cpu_steps)

    ctx.close()
    ref_cuda = None
    if rank == 0 and world == 1 and not args.no_ref_cuda:
        ref_cuda = reference_cuda(cfg, p, args.steps)
        if "value" in ref_cuda.get("fp64", {}):
            ref_cuda["value_over_fp64_reference"] = value / ref_cuda["fp64"]["value"]
            ref_cuda["e2e_over_fp64_reference"] = e2e_value / ref_cuda["fp64"]["value"]
    # the reference publishes one number: its compiled default (the legacy
    # workload, FP32, RTX 4070 SUPER): 85.718 ms per step of 10 ADOs
    published = LEGACY_PUBLISHED_ADO_STEPS if cfg.get("legacy") else None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": value / published if published else None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(cfg, p, world),
            "timing": {"windows": len(windows), "window_ms_min": min(windows), "window_ms_max": max(windows),
                       "statistic": "median device time of the --steps window"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                         else "fallback 6650 GB/s",
                         "algorithmic_bytes_per_launch": per_launch_bytes,
                         "kernel": stage_kernels_label(ctx, p, packed, info_kernels_per_stage(ctx)),
                         "traffic_source": (("dram bytes of one step launch from " if step_launch else
                                             "dram bytes of one stage from ") + " + ".join(traffic_files))
                         if traffic is not None else "no ncu summary of this workload under profiles/",
                         "launch_ms": launch_ms},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes / args.steps,
                    "d2h_bytes_per_step": slab_elems * 16 + 24,
                    "path": "hx_ctx_write_state (pinned host) + hx_ctx_step_trace (rho0, <H> per step) + hx_ctx_read_rho0"},
            "gpu_launches": launches,
            "clocks": clk,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if ref_cuda is not None:
            line["reference_cuda"] = ref_cuda
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_batch(args, cfg: dict) -> None:
    """Batched disorder average: instances sharded over ranks by state size
    (no data-path collective), one persistent graph-captured launch per stage
    on each rank, one all-reduce of the <sigma_z> sums at the end."""
    import torch
    import torch.distributed as dist

    from helix_b200 import capi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    problems = S.disorder_batch(cfg["count"], cfg["seed"], dt=cfg["dt"])
    parts = S.shard_instances([S.state_bytes(p) for p in problems], world)
    mine = [problems[i] for i in parts[rank]]
    ados = sum(p.hierarchy_size() for p in mine)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    stream = torch.cuda.Stream()
    b = capi.Batch(mine, tune=True)
    b.set_stream(stream.cuda_stream)
    st = b.info()
    state_bytes = int(st.state_bytes)
    b.step(args.warmup, trace=False)
    b.sync()
    l0 = int(b.info().kernel_launches)
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    b.step(args.steps, trace=False)
    ev1.record(stream)
    b.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    launches = int(b.info().kernel_launches) - l0
    total_ados = sum(p.hierarchy_size() for p in problems)
    value = total_ados * args.steps / (ms / 1000.0)
    stage_ms = ms / (args.steps * 4)
    per_stage_bytes = 11 * state_bytes / 4
    achieved = per_stage_bytes / (stage_ms / 1000.0) / 1e9
    peak, peak_kind = load_peaks()
    b.close()

    # end to end through the public API: create from host problems (tuned, as
    # for the device-timed run), step with
    # the per-step disorder-average trace copied to the host, all-reduce
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b = capi.Batch(mine, tune=True)
    sz = b.step(args.steps)
    b.close()
    tot = torch.tensor(np.concatenate([sz, [len(mine)]]), device="cuda")
    if world > 1:
        dist.all_reduce(tot)
    mean_sz = (tot[:-1] / tot[-1]).cpu().numpy()
    e2e_sec = max_over_ranks(time.perf_counter() - t0)
    e2e_value = total_ados * args.steps / e2e_sec
    h2d = sum(p.dim * (1 + len(p.baths)) * 8 + p.n_spins * 8 for p in mine)
    assert np.all(np.isfinite(mean_sz)) and np.all(np.abs(mean_sz) <= 1.0 + 1e-9)

    # plain FP64 form on the same GPU: every instance of this rank as its own
    # context on its own stream (all in flight together), against the batch,
    # both timed by the wall clock over the same steps
    plain = None
    if rank == 0 and not args.no_cpu_baseline:
        n_plain = 10
        ctxs = [capi.Context(p) for p in mine]
        for c in ctxs:
            c.step(2)
        for c in ctxs:
            c.sync()
        t0 = time.perf_counter()
        for c in ctxs:
            c.step(n_plain)
        for c in ctxs:
            c.sync()
        sec = time.perf_counter() - t0
        plain_value = sum(c.size for c in ctxs) * n_plain / sec
        for c in ctxs:
            c.close()
        bs = capi.Batch(mine, tune=True)
        bs.step(2, trace=False)
        bs.sync()
        t0 = time.perf_counter()
        bs.step(n_plain, trace=False)
        bs.sync()
        sec_b = time.perf_counter() - t0
        batched_wall = ados * n_plain / sec_b
        bs.close()
        plain = {"plain_fp64_contexts": plain_value, "batched": batched_wall, "ratio": batched_wall / plain_value,
                 "sample": f"all {len(mine)} instances of this rank, {n_plain} steps, wall clock after sync; "
                           "plain = one hx_ctx and stream per instance"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        sample = [p for p in problems if p.hierarchy_size() <= 1000][:16]
        ors = [O.Oracle(p) for p in sample]
        for o in ors:
            o.run(1)
        t0 = time.perf_counter()
        for o in ors:
            o.run(args.cpu_steps * 10)
        sec = time.perf_counter() - t0
        cpu = {"value": sum(o.size for o in ors) * args.cpu_steps * 10 / sec, "unit": UNIT, "cores": O.threads(),
               "kind": "port", "sample": f"{len(sample)} instances of the batch (<= 1000 ADOs each), "
                                         f"{args.cpu_steps * 10} steps each, FP64 oracle, OpenMP"}
        for o in ors:
            o.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": batch_config(cfg, problems, world),
            "batch_layout": {"ados_this_rank": ados, "state_bytes_this_rank": state_bytes,
                             "tile_elems": int(st.tile_elems), "threads": int(st.threads), "grid": int(st.grid)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None,
                         "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                         else "fallback 6650 GB/s",
                         "algorithmic_bytes_per_launch": per_stage_bytes, "kernel": "batch_stage_kernel",
                         "launch_ms": stage_ms},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d / args.steps,
                    "d2h_bytes_per_step": 8,
                    "path": "hx_batch_create (host problems, with the tile autotuner) + hx_batch_step "
                            "(<sigma_z> sum per step to host) + all-reduce"},
            "gpu_launches": launches,
            "clocks": clk,
            "disorder_average_sz_final": float(mean_sz[-1]),
        }
        if plain is not None:
            line["plain_fp64_same_gpu"] = plain
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_mixed(args, cfg: dict) -> None:
    """Mixed precision (complex64 hierarchy, rho_0 in FP64) against the plain
    FP64 propagator on the same GPU; error = trace distance of rho_0 against
    the FP64 run over the configuration's full step count."""
    import torch

    from helix_b200 import capi

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1 and rank != 0:
        return  # one hierarchy: the comparison runs on one GPU
    p = make_problem(cfg, 0)
    stream = torch.cuda.Stream()

    def timed(precision: str):
        ctx = capi.Context(p, precision=precision)
        ctx.set_stream(stream.cuda_stream)
        for _ in range(args.warmup):
            ctx.step(1)
        ctx.sync()
        c0 = ctx.counters()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        ctx.step(args.steps)
        ev1.record(stream)
        ctx.sync()
        torch.cuda.synchronize()
        launches = int(ctx.counters().kernel_launches - c0.kernel_launches)
        info = ctx.get_info()
        ctx.close()
        return ev0.elapsed_time(ev1), launches, info

    ms64, _, info64 = timed("double")
    clocks = ClockSampler(local)
    clocks.start()
    ms, launches, info = timed("mixed")
    clk = clocks.stop()
    H = int(info.hierarchy_size)
    value = H * args.steps / (ms / 1000.0)
    plain = H * args.steps / (ms64 / 1000.0)
    # complex64 bytes of one state: packed slabs hold d(d+1)/2 elements (state_bytes counts them at 16 B)
    state32 = int(info.state_bytes) // 2
    per_stage = 11 * state32 / 4
    stage_ms = ms / (args.steps * 4)
    achieved = per_stage / (stage_ms / 1000.0) / 1e9
    peak, peak_kind = load_peaks()

    # error against the FP64 propagator, every 10 steps over the full run
    def trace_distance(a, b):
        m = a - b
        return 0.5 * float(np.sum(np.abs(np.linalg.eigvalsh(0.5 * (m + m.conj().T)))))

    n_err = cfg["error_steps"]
    c64 = capi.Context(p)
    cm = capi.Context(p, precision="mixed")
    td, en_err = [], []
    for _ in range(n_err // 10):
        r64, e64 = c64.step_trace(10)
        rm, em = cm.step_trace(10)
        td.append(trace_distance(rm[-1], r64[-1]))
        en_err.append(float(np.max(np.abs(em - e64))))
    c64.close()
    cm.close()

    # end to end through the C ABI: state upload from host, steps with rho_0(t)
    # and <H>(t) to the host, final rho_0
    pinned = torch.empty(H * p.dim * p.dim * 2, dtype=torch.float64, pin_memory=True)
    host_state = pinned.numpy().view(np.complex128).reshape(H, p.dim, p.dim)
    host_state[:] = 0
    host_state[0] = S.initial_rho0(p.dim)
    rho_trace = torch.empty(args.steps * p.dim * p.dim * 2, dtype=torch.float64, pin_memory=True).numpy()
    en_trace = np.zeros(args.steps)
    ctx = capi.Context(p, precision="mixed")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.set_state(host_state)
    ctx.step_trace_into(args.steps, rho_trace, en_trace)
    ctx.rho0()
    e2e_sec = time.perf_counter() - t0
    ctx.close()
    e2e_value = H * args.steps / e2e_sec

    cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        o = O.Oracle(p)
        t0 = time.perf_counter()
        o.run(1)
        sec = time.perf_counter() - t0
        o.close()
        cpu = {"value": H / sec, "unit": UNIT, "cores": O.threads(), "kind": "port",
               "sample": f"1 full step of the {H}-ADO hierarchy, FP64 oracle, OpenMP"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64 (rho_0 f64)", "data": "synthetic",
        "config": {"workload": cfg["workload"], "ados": H, "dim": p.dim, "modes": p.modes, "depth_L": p.max_depth - 1,
                   "dt": p.dt, "integrator": "RK4 (4-term Taylor, Horner form)", "parallelism": "single",
                   "l2": f"inputs larger than L2 (state {state32 / 1e9:.3f} GB complex64)"},
        "plain_fp64_same_gpu": {"value": plain, "ms_per_step": ms64 / args.steps, "speedup": value / plain},
        "error_vs_fp64": {"trace_distance_max": max(td), "trace_distance_final": td[-1],
                          "energy_abs_max": max(en_err), "steps": n_err, "every": 10},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None,
                     "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                     else "fallback 6650 GB/s",
                     "algorithmic_bytes_per_launch": per_stage,
                     "kernel": ("herm_band_kernel<float,8>" if state32 < H * p.dim * p.dim * 8 else "large_kernel<float,8>")
                     + " + large_upterm_kernel + ado0_kernel",
                     "launch_ms": stage_ms},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": H * p.dim * p.dim * 16 / args.steps,
                "d2h_bytes_per_step": p.dim * p.dim * 16 + 24,
                "path": "hx_ctx_write_state + hx_ctx_step_trace (rho0, <H> per step) + hx_ctx_read_rho0"},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def load_tensor_peak() -> tuple[float, str]:
    """Dense TF32 tensor peak in TFLOP/s: half the measured BF16 GEMM rate (the
    TF32 tensor rate is half the BF16 rate on this part), else half the
    fallback BF16 figure."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return 0.5 * float(json.load(f)["bf16_tflops"]), "measured bf16_tflops / 2 (MEASURED_PEAKS.json)"
    except (OSError, KeyError, ValueError):
        return 0.5 * 1590.0, "fallback 1590 TFLOP/s bf16 / 2"


def run_dense(args, cfg: dict) -> None:
    """Dense H on the tensor cores (HX_FLAG_DENSE_H) against the plain FP64
    propagator for the same H (the CSR path, the only FP64 path for a dense
    H) on the same GPU.  The roofline is the tensor one: the GEMM kernel alone
    (hx_ctx_dense_product) timed with CUDA events, algorithmic FLOPs
    8 H d^3 per launch (the complex product X H_off of every ADO) and executed
    FLOPs 3x that (the TF32 split)."""
    import torch

    from helix_b200 import capi

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if rank != 0:
        return  # one hierarchy: the comparison runs on one GPU
    p = make_problem(cfg, 0)
    stream = torch.cuda.Stream()
    H, d = p.hierarchy_size(), p.dim

    def events_ms(fn) -> float:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1)

    ctx = capi.Context(p, precision="mixed", dense_h=True)
    ctx.set_stream(stream.cuda_stream)
    for _ in range(args.warmup):
        ctx.step(1)
    ctx.sync()
    c0 = ctx.counters()
    clocks = ClockSampler(local)
    clocks.start()
    ms = events_ms(lambda: ctx.step(args.steps))
    clk = clocks.stop()
    launches = int(ctx.counters().kernel_launches - c0.kernel_launches)
    info = ctx.get_info()
    # the GEMM alone (split of X in shared memory) on the current state
    reps = 20
    ctx.dense_product(2)
    gemm_ms = events_ms(lambda: ctx.dense_product(reps)) / reps
    ctx.close()
    value = H * args.steps / (ms / 1000.0)

    # cuBLAS TF32 on one of the three products of the same shape, for scale (not on the product path)
    torch.backends.cuda.matmul.allow_tf32 = True
    a = torch.randn(H * d, 2 * d, device="cuda")
    b = torch.randn(2 * d, 2 * d, device="cuda")
    c = torch.empty(H * d, 2 * d, device="cuda")
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for _ in range(3):
            torch.matmul(a, b, out=c)
        cublas_ms = events_ms(lambda: [torch.matmul(a, b, out=c) for _ in range(reps)]) / reps
    del a, b, c

    # plain FP64 propagator for the same dense H (CSR path) and the error against it
    c64 = capi.Context(p)
    c64.set_stream(stream.cuda_stream)
    c64.step(1)
    c64.sync()
    k64 = 2
    ms64 = events_ms(lambda: c64.step(k64)) / k64
    c64.close()

    def trace_distance(x, y):
        m = x - y
        return 0.5 * float(np.sum(np.abs(np.linalg.eigvalsh(0.5 * (m + m.conj().T)))))

    n_err = cfg["error_steps"]
    c64 = capi.Context(p)
    cm = capi.Context(p, precision="mixed", dense_h=True)
    td, en_err, tr_err = [], [], []
    for _ in range(n_err // 10):
        r64, e64 = c64.step_trace(10)
        rm, em = cm.step_trace(10)
        td.append(trace_distance(rm[-1], r64[-1]))
        en_err.append(float(np.max(np.abs(em - e64))))
        tr_err.append(abs(float(np.trace(rm[-1]).real) - 1.0))
    c64.close()
    cm.close()

    # end to end through the C ABI: state upload from host, steps with rho_0(t) and <H>(t), final rho_0
    pinned = torch.empty(H * d * d * 2, dtype=torch.float64, pin_memory=True)
    host_state = pinned.numpy().view(np.complex128).reshape(H, d, d)
    host_state[:] = 0
    host_state[0] = S.initial_rho0(d)
    rho_trace = torch.empty(args.steps * d * d * 2, dtype=torch.float64, pin_memory=True).numpy()
    en_trace = np.zeros(args.steps)
    ctx = capi.Context(p, precision="mixed", dense_h=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.set_state(host_state)
    ctx.step_trace_into(args.steps, rho_trace, en_trace)
    ctx.rho0()
    e2e_sec = time.perf_counter() - t0
    ctx.close()

    cpu = None
    if not args.no_cpu_baseline:
        # one full step of the same H and baths with a depth-1 hierarchy (17 ADOs), per ADO
        from oracle import oracle as O
        q = make_problem(dict(cfg, depth=1), 0)
        o = O.Oracle(q)
        t0 = time.perf_counter()
        o.run(1)
        sec = time.perf_counter() - t0
        o.close()
        cpu = {"value": q.hierarchy_size() / sec, "unit": UNIT, "cores": O.threads(), "kind": "port",
               "sample": f"1 full step of the same H and baths at depth 1 ({q.hierarchy_size()} ADOs), "
                         "FP64 oracle (CSR H), OpenMP; per-ADO cost does not depend on the depth"}
    alg = 8.0 * H * d ** 3
    tpeak, tpeak_src = load_tensor_peak()
    achieved = alg / (gemm_ms / 1000.0) / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64 state, tf32x3 products, f32 accumulate (rho_0 f64)", "data": "synthetic",
        "config": {"workload": cfg["workload"], "ados": H, "dim": d, "modes": p.modes, "depth_L": p.max_depth - 1,
                   "dt": p.dt, "h_nnz_per_row": d, "integrator": "RK4 (4-term Taylor, Horner form)",
                   "parallelism": "single", "l2": f"inputs larger than L2 (state {H * d * d * 8 / 1e9:.3f} GB complex64)"},
        "plain_fp64_same_gpu": {"value": H / (ms64 / 1000.0), "ms_per_step": ms64, "path": "csr (FP64)",
                                "speedup": value / (H / (ms64 / 1000.0))},
        "error_vs_fp64": {"trace_distance_max": max(td), "trace_distance_final": td[-1],
                          "energy_abs_max": max(en_err), "trace_abs_max": max(tr_err), "steps": n_err, "every": 10},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": tpeak, "unit": "TFLOP/s",
                     "frac": achieved / tpeak, "traffic": profiled_traffic(args.config, "tc_split_gemm_kernel"),
                     "peak_source": tpeak_src, "kernel": "tc_split_gemm_kernel",
                     "algorithmic_flops_per_launch": alg, "executed_flops_per_launch": 3 * alg,
                     "executed_tflops": 3 * achieved, "launch_ms": gemm_ms,
                     "cublas_tf32_one_product_ms": cublas_ms,
                     "cublas_tf32_tflops": alg / (cublas_ms / 1000.0) / 1e12},
        "e2e": {"value": H * args.steps / e2e_sec, "unit": UNIT, "h2d_bytes_per_step": H * d * d * 16 / args.steps,
                "d2h_bytes_per_step": d * d * 16 + 24,
                "path": "hx_ctx_write_state + hx_ctx_step_trace (rho0, <H> per step) + hx_ctx_read_rho0"},
        "gpu_launches": launches,
        "kernels_per_step": int(info.kernels_per_step),
        "clocks": clk,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def run_closure(args, cfg: dict) -> None:
    """Learned closure: L=2 hierarchy + MLP closure of tier 3 against the plain
    L=5 run (the reference solution) and the plain truncated L=2 run, on held-out seeds.
    value = closure ADO-steps/s of the coarse hierarchy; the line also gives
    the simulated-steps rate of closure and of plain L=5 and the trace
    distances of rho_0(t)."""
    import torch

    from helix_b200 import capi

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1 and rank != 0:
        return
    n, K, dt = cfg["n"], cfg["K"], cfg["dt"]
    steps, every = cfg["traj_steps"], cfg["every"]

    def problem(seed, depth):
        return S.spin_glass(n, seed=seed, depth=depth, K=K, h=cfg["h"], dt=dt)

    def td(a, b):
        m = a - b
        return 0.5 * float(np.sum(np.abs(np.linalg.eigvalsh(0.5 * (m + m.conj().T)))))

    train_seeds = [5000 + i for i in range(cfg["train_seeds"])]
    test_seeds = [9000 + i for i in range(cfg["test_seeds"])]
    t0 = time.perf_counter()
    cl = capi.Closure(problem(train_seeds[0], cfg["coarse_depth"]), fine_max_depth=cfg["fine_depth"] + 1,
                      hidden=cfg["hidden"], capacity=len(train_seeds) * steps // every, seed=1)
    for s in train_seeds:
        with capi.Context(problem(s, cfg["fine_depth"])) as ctx:
            for _ in range(steps // every):
                ctx.step(every)
                cl.harvest(ctx)
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    loss = cl.train(iters=cfg["iters"], batch=cfg["mlp_batch"], lr=cfg["lr"], seed=7)
    t_train = time.perf_counter() - t0
    info = cl.info()

    # held-out seeds: plain L=5 (the reference solution), plain L=2 and L=2 +
    # closure over the full trajectory (errors, untimed); then the step rate of
    # each form on the first seeds, timed step by step with L2 flushed in between
    stream = torch.cuda.Stream()
    flusher = L2Flush(stream, local)

    def trajectory(p, closure=None):
        with capi.Context(p) as ctx:
            if closure is not None:
                closure.attach(ctx)
            rho, _ = ctx.step_trace(steps, rho0=True, energy=False)
            return rho, ctx.size

    def step_rate(p, closure=None):
        with capi.Context(p) as ctx:
            ctx.set_stream(stream.cuda_stream)
            if closure is not None:
                closure.attach(ctx)
            for _ in range(args.warmup):
                ctx.step(1)
            ctx.sync()
            k0 = ctx.counters().kernel_launches
            ms = flusher.time_steps(lambda: ctx.step(1), time_steps)
            return ms, int(ctx.counters().kernel_launches - k0)

    e_plain, e_closed = [], []
    for s in test_seeds:
        ref, H_fine = trajectory(problem(s, cfg["fine_depth"]))
        plain, _ = trajectory(problem(s, cfg["coarse_depth"]))
        closed, H_coarse = trajectory(problem(s, cfg["coarse_depth"]), cl)
        e_plain.append(max(td(plain[t], ref[t]) for t in range(0, steps, 10)))
        e_closed.append(max(td(closed[t], ref[t]) for t in range(0, steps, 10)))
    time_seeds = test_seeds[:cfg["time_seeds"]]
    time_steps = cfg["time_steps"]
    ms_fine = ms_plain = ms_closed = 0.0
    launches = 0
    clocks = ClockSampler(local)
    clocks.start()
    for s in time_seeds:
        ms_fine += step_rate(problem(s, cfg["fine_depth"]))[0]
        ms_plain += step_rate(problem(s, cfg["coarse_depth"]))[0]
        mc, lc = step_rate(problem(s, cfg["coarse_depth"]), cl)
        ms_closed += mc
        launches += lc
    clk = clocks.stop()
    cl.close()
    del flusher
    nt = len(test_seeds)
    timed = len(time_seeds) * time_steps
    value = H_coarse * timed / (ms_closed / 1000.0)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": timed, "warmup": args.warmup,
        "ms_per_step": ms_closed / timed, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 hierarchy, bf16 MLP (f32 accumulation)", "data": "synthetic",
        "config": {"workload": cfg["workload"], "ados_coarse": H_coarse, "ados_fine": H_fine, "dim": 1 << n,
                   "modes": 3 * n, "coarse_depth_L": cfg["coarse_depth"], "fine_depth_L": cfg["fine_depth"],
                   "dt": dt, "train_seeds": len(train_seeds), "test_seeds": nt, "trajectory_steps": steps,
                   "snapshot_every": every, "timed": f"{time_steps} steps on each of {len(time_seeds)} held-out "
                                                  "seeds per form, after the warm-up",
                   "l2": "L2 flushed before every timed step (steps timed one by one with CUDA events)",
                   "mlp": f"features of (mode, n_k, r, c) {3 * n + 3 + cfg['coarse_depth'] + 1}-{cfg['hidden']}-"
                   f"{cfg['hidden']}-2 GELU -> complex coefficient of rho_n(r, c); table of "
                   f"{3 * n * (cfg['coarse_depth'] + 1) * (1 << n) ** 2} coefficients, elementwise closure kernel",
                   "parallelism": "single"},
        "closure": {"simulated_steps_per_s": timed / (ms_closed / 1000.0),
                    "plain_fine_steps_per_s": timed / (ms_fine / 1000.0),
                    "plain_coarse_steps_per_s": timed / (ms_plain / 1000.0),
                    "speedup_vs_plain_fine": ms_fine / ms_closed,
                    "trace_distance_vs_fine": {"closure_max": max(e_closed), "closure_mean": float(np.mean(e_closed)),
                                               "truncated_max": max(e_plain), "truncated_mean": float(np.mean(e_plain))},
                    "gain_over_truncation": float(np.mean(e_plain) / np.mean(e_closed)),
                    "train": {"snapshots": info["snapshots"], "data_s": t_data, "train_s": t_train,
                              "iters": cfg["iters"], "batch": cfg["mlp_batch"], "loss_first": float(loss[:20].mean()),
                              "loss_last": float(loss[-100:].mean())}},
        "gpu_launches": launches,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="c2")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--windows", type=int, default=0,
                    help="timed windows of --steps steps (default: repeat until ~1 s of device time, at least 5)")
    ap.add_argument("--no-ref-cuda", action="store_true",
                    help="skip timing the reference's own CUDA propagator at the workload's shape")
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    if args.impl == "reference":
        run_reference(args, cfg)
    elif cfg.get("batch"):
        run_batch(args, cfg)
    elif cfg.get("mixed"):
        run_mixed(args, cfg)
    elif cfg.get("dense"):
        run_dense(args, cfg)
    elif cfg.get("closure"):
        run_closure(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
