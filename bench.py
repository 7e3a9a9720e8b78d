"""Benchmark of the electrostatic PIC time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the MCC configuration): 513x513 nodes (512^2 cells, dx = 1e-4 m),
4M electrons + 4M ions, left wall 100 V, multigrid to a 1e-8 relative
residual, null-collision MCC against an argon-like gas (1e21 m^-3, 300 K,
elastic / excitation / ionisation / charge exchange), dt = 1e-11 s.  Inputs
are synthetic and seeded.  One step = kick + MCC + drift + absorb + deposit,
the Poisson solve and E.  The metric is particle-steps/s; `value` times K
steps with the state resident in HBM (particle arrays 8M x 20 B = 160 MB,
larger than the 126 MB L2).  `e2e` times the public API from pinned host
arrays: load, init, K steps, read back particles and phi.  `poisson` times
the large workload's solve (2049^2, 64M + 64M particles, Gaussian blob) to a
1e-10 relative residual, mixed precision against plain FP64.  On one GPU the
line also carries the reference's other configurations: `large_step` (that
workload as a PIC step for 200 steps, each multigrid), `ensemble` (64
independent members of 129^2-513^2 nodes, 500 steps, one graph launch, one
particle pass over all members per step) and `adjoint` (the differentiable
257^2 workload: forward and backward cost, central finite differences).

Multi-GPU (torchrun): independent replicas, one per GPU (the path does not
shard); the time is the max over ranks and `value` sums all ranks' work.
--impl reference runs the reference's own kernels (compiled for the CPU by
oracle/ref_build.py) on the host cores for the same workload.
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

METRIC = "particle-steps/s/GPU at 512², 8M ptcl; mixed vs FP64 multigrid at 1e-10 residual"
UNIT = "particle-steps/s"
FALLBACK_HBM_GBS = 6650.0
BYTES_PER_PARTICLE = 32.0  # x, y, vx, vy float32, read and written by the fused pass
BYTES_PER_NODE = 12.0      # E (float2) read, charge (float) written


def sort_passes(nodes, tile=16, digit_max=10):
    """Radix passes of the cell sort of an nodes x nodes grid: tile-major cell
    keys plus the dead key, in digits of at most digit_max bits."""
    tiles = -(-(nodes - 1) // tile)
    bits = (tiles * tiles * tile * tile).bit_length()
    return -(-bits // digit_max)


def sort_bytes_per_particle(passes):
    """Compulsory bytes of one cell sort per particle: keys from x, y (8 B
    read, key and slot 8 B written), each pass's histogram (4 B) and scatter
    (8 B read, 8 B written), the tile starts (4 B), and the gather of the five
    arrays through the permutation (4 B + 20 B read, 20 B written)."""
    return 16.0 + 20.0 * passes + 4.0 + 44.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # 80 timed steps after 5 warm-up steps hold exactly one cell sort (every 80 steps)
    ap.add_argument("--steps", type=int, default=80)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--sort-interval", type=int, default=80,
                    help="steps between cell sorts (80: the autotuner's choice for 513^2 shapes)")
    ap.add_argument("--particles", type=int, default=4_000_000, help="per species")
    ap.add_argument("--tile", type=int, default=16, help="cells per side of the push's work tiles")
    ap.add_argument("--push", default="ring", choices=["ring", "warp", "warp_agg", "pipe"],
                    help="particle-pass streaming: one ring of bulk copies per block (ring), per-warp pipelines "
                         "(warp), per-warp pipelines with warp-aggregated deposit atomics (warp_agg)")
    ap.add_argument("--no-poisson", action="store_true")
    ap.add_argument("--poisson-only", action="store_true",
                    help="run only the large Poisson comparison (its multigrid in the --mg-launch mode when that "
                         "is 'host', so that profilers see each kernel)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-collisionless", action="store_true")
    ap.add_argument("--no-dst", action="store_true", help="skip the step timed with the sine-transform solve")
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-graph", action="store_true", help="launch every kernel from the host (profilers)")
    ap.add_argument("--mg-sweeps", type=int, nargs=2, default=(2, 2), metavar=("PRE", "POST"),
                    help="red-black sweeps before and after each coarse-grid correction")
    ap.add_argument("--omega", type=float, default=1.15, help="smoother over-relaxation")
    ap.add_argument("--coarse-fp32", action="store_true",
                    help="the mixed multigrid's direct solve of its 33^2 level in FP32 (default FP64)")
    ap.add_argument("--mg-launch", default="graph", choices=["persistent", "host", "graph", "cluster", "dst", "hybrid"],
                    help="multigrid launch mode (host: one launch per kernel, for profilers; dst: the "
                         "sine-transform solve in place of the V-cycles; hybrid: the levels of at most 129^2 nodes "
                         "in one cluster launch per cycle)")
    ap.add_argument("--ensemble", type=int, default=-1,
                    help="also time an ensemble of this many independent collisionless members (0: off; default: "
                         "64 on one GPU, off on several)")
    ap.add_argument("--ensemble-steps", type=int, default=500)
    ap.add_argument("--ensemble-one-pass", action="store_true",
                    help="time the ensemble with one particle pass over all members first (default: a pass per "
                         "member in its branch; the other structure is timed second either way)")
    ap.add_argument("--no-large-step", action="store_true",
                    help="skip the large workload as a PIC step (2049^2 nodes, 64M + 64M particles, multigrid to "
                         "1e-10, mixed precision against plain FP64, 200 steps; run on one GPU by default)")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the differentiable workload (forward, adjoint, finite-difference check; run on one GPU "
                         "by default)")
    ap.add_argument("--tune-cache", default=os.path.join(ROOT, "pic_b200", "tuned_b200.json"),
                    help="autotuner results (read if present, written after tuning)")
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------

class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed
    region, read only: through NVML in this process every half millisecond
    (the timed windows last milliseconds), else nvidia-smi every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []       # nvidia-smi rows
        self.nvml_rows = []  # (sm MHz, max sm MHz, reason bits)
        self.bits = {}
        self._stop = threading.Event()
        self._ready = threading.Event()
        self._t = None

    def _run_nvml(self):
        import pynvml

        pynvml.nvmlInit()
        try:
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            self.bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                         "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                         "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                         "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
            while True:
                sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.nvml_rows.append((float(sm), float(mx), int(r)))
                self._ready.set()
                if self._stop.wait(0.0005):
                    break
        finally:
            pynvml.nvmlShutdown()

    def _run(self):
        try:
            self._run_nvml()
            return
        except Exception:
            pass
        self._ready.set()
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.rows.append([c.strip() for c in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        self._ready.wait(10)  # the first sample precedes the timed region
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if self.nvml_rows:
            sm = [r[0] for r in self.nvml_rows]
            reasons = sorted({n for n in self.REASONS for r in self.nvml_rows if r[2] & self.bits[n]})
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(r[1] for r in self.nvml_rows),
                    "sm_min_mhz": min(sm), "reasons": reasons, "samples": len(self.nvml_rows), "source": "nvml"}
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        reasons = sorted({self.REASONS[k] for r in self.rows for k in range(4) if len(r) > 4 + k and "Active" in r[4 + k]
                          and "Not" not in r[4 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows), "source": "nvidia-smi"}


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------

def peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic():
    """DRAM bytes per k_push launch from the committed ncu summary (profiles/), or None."""
    p = os.path.join(ROOT, "profiles", "k_push_mcc_513x513_8M.md")
    try:
        for line in open(p):
            if line.startswith("bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


GRAPH_OPTS = {"use_graph": True, "mg_launch": "graph"}


def make_sim(w, rank, sort_interval, mcc=True, **over):
    from pic_b200 import Consts, workloads
    from pic_b200.simulation import PICSimulation

    mask, phi_bc = workloads.dirichlet(w)
    species = [dict(name="e", charge=-Consts.qe, mass=Consts.me, np2c=w.np2c(w.n_e), capacity=int(w.n_e * 1.25)),
               dict(name="i", charge=Consts.qe, mass=workloads.ION_MASS, np2c=w.np2c(w.n_i),
                    capacity=int(w.n_i * 1.25))]
    tables = workloads.mcc_tables(w) if mcc else None
    opts = dict(GRAPH_OPTS, **over)
    return PICSimulation(w.nodes, w.nodes, w.dx, w.dx, w.dt, species, mask, phi_bc, tol=w.tol, max_cycles=50,
                         sort_interval=sort_interval, mcc=tables, seed=1000 + rank, **opts)


def gen_arrays(w, rank):
    from pic_b200 import workloads

    rng = np.random.Generator(np.random.Philox(w.seed + 17 * rank))
    return [workloads.species_arrays(w, "e", rng), workloads.species_arrays(w, "i", rng)]


def live_count(sim):
    return sum(sim.counters()["count"])


def reduce_replicas(ms, work, world, device):
    """Whole-job throughput of independent replicas: the work (particle-steps)
    summed over ranks divided by the slowest rank's time.  Returns
    (units per second, max ms)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], device=device, dtype=torch.float64)
    w = torch.tensor([work], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(w)
    ms_max = float(t.item())
    return float(w.item()) / (ms_max / 1e3), ms_max


def time_sort(sim, reps=3):
    """Device time of one cell sort of every species (pic_sim_sort, the sort a
    step runs every sort_interval steps), averaged over `reps` sorts."""
    import torch

    stream = torch.cuda.current_stream()
    sim.sort()  # warm
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        sim.sort()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def sorts_in(first_step, K, interval):
    """Cell sorts a run of K steps starting at step `first_step` performs."""
    return sum(1 for k in range(first_step, first_step + K) if interval > 0 and k % interval == 0)


def window_start(warmup, K, interval):
    """First step of the timed window: at least `warmup` steps in, and placed
    so that the particle order is as old, on average, as over a whole run.  A
    step's cost grows with the steps since the last cell sort (513^2, 8M
    particles, MCC: 0.243 ms a few steps after a sort, 0.251 ms averaged over
    the 80-step interval), so a window shorter than the interval is centred in
    one, and a longer one starts at a sort."""
    if interval <= 0:
        return warmup
    target = (interval - K) // 2 if K < interval else 0
    return warmup + (target - warmup) % interval


def sort_roofline(sort_ms, particles, nodes, peak):
    """HBM fraction of one cell sort of every species (sort_bytes_per_particle)."""
    passes = sort_passes(nodes)
    b = particles * sort_bytes_per_particle(passes)
    gbs = b / (sort_ms / 1e3) / 1e9
    return {"passes": passes, "bytes": b, "achieved": round(gbs, 1), "unit": "GB/s", "frac": round(gbs / peak, 4)}


def amortised_ms(ms_window, K, first_step, interval, sort_ms):
    """The window's time with the cell sort counted at its average rate: a
    sort every `interval` steps, whatever number of sorts the window held."""
    if interval <= 0:
        return ms_window
    return ms_window + (K / interval - sorts_in(first_step, K, interval)) * sort_ms


def time_steps(sim, K, world):
    """K steps timed with CUDA events on the launching stream (the captured-graph path),
    then K more steps with per-phase event timing (the same kernels launched one by one)."""
    import torch
    import torch.distributed as dist

    stream = torch.cuda.current_stream()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    n0 = live_count(sim)
    l0 = sim.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step(K)
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    launches = sim.kernel_launches() - l0
    n1 = live_count(sim)
    sim.set_profiling(True)
    sim.step(K)
    prof = sim.read_profile()
    sim.set_profiling(False)
    return ms, prof, launches, n0, n1


def run_ours(args, world, rank, local):
    import torch
    import torch.distributed as dist

    from pic_b200 import workloads

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    w = workloads.scaled(workloads.MCC, n=args.particles)
    arrays = gen_arrays(w, rank)
    sim = make_sim(w, rank, args.sort_interval, mcc=True)
    for s, a in enumerate(arrays):
        sim.load(s, *a)
    sim.init()
    first = window_start(args.warmup, args.steps, args.sort_interval)
    sim.step(first)
    with ClockSampler(local) as clk:
        ms_window, prof, launches, n0, n1 = time_steps(sim, args.steps, world)
    clocks = clk.summary()
    sort_ms = time_sort(sim)
    # the window's time with its cell sorts counted at the average rate (one
    # every sort_interval steps): a window that held none is charged its share
    ms = amortised_ms(ms_window, args.steps, first, args.sort_interval, sort_ms)
    value, ms_max = reduce_replicas(ms, 0.5 * (n0 + n1) * args.steps, world, "cuda")
    _, ms_window_max = reduce_replicas(ms_window, 0.0, world, "cuda")
    counters = sim.counters()

    # roofline of the fused particle kernel: x, y, vx, vy read and written
    # (32 B per particle; vz is touched only by the collision candidates,
    # a few per thousand, in their own pass) plus the E field read
    # (8 B per node) and the charge written (4 B per node) once per step.
    G = w.nodes * w.nodes
    push = prof["push"]
    push_ms = push["ms"] / max(1, push["count"])
    bytes_per_launch = 0.5 * (n0 + n1) * BYTES_PER_PARTICLE + G * BYTES_PER_NODE
    achieved = bytes_per_launch / (push_ms / 1e3) / 1e9
    peak, peak_kind = peak_hbm()
    traffic = ncu_traffic()
    roofline = {"bound": "hbm", "kernel": {"ring": "k_push", "pipe": "k_push_pipe"}.get(args.push, "k_push_warp"), "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_kind,
                "bytes_per_launch": bytes_per_launch, "ms_per_launch": round(push_ms, 5)}
    phases = {k: round(v["ms"] / args.steps, 4) for k, v in prof.items() if isinstance(v, dict)}
    phases["sort"] = round(sort_ms / args.sort_interval, 4) if args.sort_interval > 0 else 0.0
    phases["timing"] = ("per-phase CUDA events over K further steps launched kernel by kernel; sort: one measured "
                        "sort of every species divided by the sort interval")
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "ms_per_step_window": ms_window_max / args.steps, "sort_ms": round(sort_ms, 4),
        "sort_ms_amortised": round(sort_ms / args.sort_interval, 5) if args.sort_interval > 0 else 0.0,
        "sort_roofline": sort_roofline(sort_ms, 0.5 * (n0 + n1), w.nodes, peak),
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 particles / f64 Poisson residual", "data": "synthetic (seeded Philox)",
        "config": {"workload": "mcc: 513x513 nodes (512^2 cells), dx 1e-4 m, "
                               f"{w.n_e} e- + {w.n_i} ions (40 amu), Te 2 eV, Ti 0.03 eV, n0 1e14, left wall 100 V, "
                               "argon-like gas 1e21 m^-3 300 K, elastic/excitation/ionisation/charge exchange, "
                               "dt 1e-11 s, multigrid tol 1e-8",
                   "global_batch": int(0.5 * (n0 + n1)) * world, "parallelism": f"replicas{world}",
                   "sort_interval": args.sort_interval,
                   "sorts_in_timed_region": sorts_in(first, args.steps, args.sort_interval),
                   "timed_window": f"steps {first}-{first + args.steps} after init (a cell sort at every multiple of "
                                   f"{args.sort_interval}): the window's mean particle-order age is that of a whole "
                                   f"run; the {first} steps before it are untimed warm-up",
                   "sort_accounting": "ms_per_step and value count one measured cell sort every sort_interval "
                                      "steps; ms_per_step_window is the timed window as it ran",
                   "l2": "inputs larger than L2 (particle arrays 160 MB > 126 MB)"},
        "phase_ms_per_step": phases,
        "mg_cycles_per_step": prof["mg_cycles"] / args.steps,
        "counters": {k: counters[k] for k in ("absorbed", "collisions", "born", "count", "last_rel_res")},
        "roofline": roofline,
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    sim.close()
    del sim
    torch.cuda.empty_cache()

    if not args.no_collisionless:
        sim = make_sim(w, rank, args.sort_interval, mcc=False)
        for s, a in enumerate(arrays):
            sim.load(s, *a)
        sim.init()
        first2 = window_start(args.warmup, args.steps, args.sort_interval)
        sim.step(first2)
        ms2, prof2, _, m0, m1 = time_steps(sim, args.steps, world)
        ms2 = amortised_ms(ms2, args.steps, first2, args.sort_interval, time_sort(sim))
        t2 = torch.tensor([ms2], device="cuda", dtype=torch.float64)
        if world > 1:
            dist.all_reduce(t2, op=dist.ReduceOp.MAX)
        p2 = prof2["push"]["ms"] / max(1, prof2["push"]["count"])
        out["collisionless"] = {"value": world * 0.5 * (m0 + m1) * args.steps / (float(t2.item()) / 1e3),
                                "ms_per_step": float(t2.item()) / args.steps,
                                "push_ms": round(p2, 5),
                                "push_frac_of_peak": round((0.5 * (m0 + m1) * BYTES_PER_PARTICLE + G * BYTES_PER_NODE)
                                                           / (p2 / 1e3) / 1e9 / peak, 4),
                                "mg_cycles_per_step": prof2["mg_cycles"] / args.steps}
        sim.close()
        del sim
        torch.cuda.empty_cache()

    if not args.no_dst and args.mg_launch != "dst":
        # the same workload with the field solved by sine transforms (the
        # reference's FFT path, src/FFT.py:10-64): exact to FP64 round-off,
        # no V-cycles; the headline stays on the multigrid
        sim = make_sim(w, rank, args.sort_interval, mcc=True, mg_launch="dst")
        for s, a in enumerate(arrays):
            sim.load(s, *a)
        sim.init()
        first3 = window_start(args.warmup, args.steps, args.sort_interval)
        sim.step(first3)
        ms3, prof3, _, m0, m1 = time_steps(sim, args.steps, world)
        ms3 = amortised_ms(ms3, args.steps, first3, args.sort_interval, time_sort(sim))
        t3 = torch.tensor([ms3], device="cuda", dtype=torch.float64)
        if world > 1:
            dist.all_reduce(t3, op=dist.ReduceOp.MAX)
        out["dst_solve"] = {"value": world * 0.5 * (m0 + m1) * args.steps / (float(t3.item()) / 1e3),
                            "ms_per_step": float(t3.item()) / args.steps,
                            "solve_ms_per_step": round(prof3["solve"]["ms"] / args.steps, 4),
                            "rel_res": sim.counters()["last_rel_res"],
                            "solver": sim.mg_effective_launch()}
        sim.close()
        del sim
        torch.cuda.empty_cache()

    if not args.no_e2e:
        out["e2e"] = run_e2e(w, arrays, args, world, rank)
    if not args.no_poisson and rank == 0:
        out["poisson"] = run_poisson()
    # the other workloads of the reference's configuration list, on one GPU
    # (a multi-GPU run times the replicated step only)
    members = args.ensemble if args.ensemble >= 0 else (64 if world == 1 else 0)
    if members > 0 and rank == 0:
        out["ensemble"] = run_ensemble(args, members)
    if not args.no_large_step and rank == 0 and world == 1:
        out["large_step"] = run_large_step()
    if not args.no_adjoint and rank == 0 and world == 1:
        out["adjoint"] = run_adjoint()
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        out["cpu_baseline"] = run_cpu_baseline(w, arrays, args.cpu_steps)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_ensemble(args, members):
    """Ensemble workload: members with grid sides from {129, 257, 513}, 1e5-2e6
    particles per species, Te 1-5 eV, left wall 0-200 V, collisionless; each
    member shape tuned by the autotuner; all members stepped by one graph
    launch per call (pic_ens_step)."""
    import torch

    from pic_b200 import autotune, ensemble

    ws = ensemble.ensemble_workloads(members)
    tuner = autotune.Autotuner(cache_path=args.tune_cache)
    t0 = time.time()
    choices = tuner.tune_ensemble(ws)
    tune_s = time.time() - t0
    sims = []
    for w, ch in zip(ws, choices):
        sims.append(ensemble.member_simulation(w, **ch.config()))

    def start():
        # every member from its initial particles (both step structures are
        # timed from the same state)
        for w, sim in zip(ws, sims):
            for s, a in enumerate(ensemble.member_arrays(w)):
                sim.load(s, *a)
            sim.init()

    start()
    ens = ensemble.Ensemble(sims)
    if args.ensemble_one_pass:
        ens.fused_pass = True
    ens.step(3)
    torch.cuda.synchronize()
    n0 = ens.particle_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ens.step(args.ensemble_steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    n1 = ens.particle_count()
    fused = ens.fused_pass
    # the other step structure on the same members, for comparison: every
    # member's pass in its own branch (or back to the one pass)
    ens.fused_pass = not fused
    other = None
    if ens.fused_pass != fused:
        start()
        ens.step(3)
        torch.cuda.synchronize()
        m0 = ens.particle_count()
        e0.record()
        ens.step(args.ensemble_steps)
        e1.record()
        torch.cuda.synchronize()
        ms2 = e0.elapsed_time(e1)
        m1 = ens.particle_count()
        other = {"one_particle_pass_over_all_members": ens.fused_pass, "ms_per_step": ms2 / args.ensemble_steps,
                 "value": 0.5 * (m0 + m1) * args.ensemble_steps / (ms2 / 1e3)}
    ens.close()
    for sim in sims:
        sim.close()
    # the particle arrays' compulsory bytes (32 B per particle-step) and the
    # grids' (12 B per node) over the whole ensemble step: a lower bound of the
    # step's traffic, whose time also holds every member's field solve
    nodes = sum(w.nodes * w.nodes for w in ws)
    step_bytes = 0.5 * (n0 + n1) * BYTES_PER_PARTICLE + nodes * BYTES_PER_NODE
    peak, kind = peak_hbm()
    gbs = step_bytes / (ms / args.ensemble_steps / 1e3) / 1e9
    picked = {}
    for ch in choices:
        k = (f"tile {ch.tile}, sort every {ch.sort_interval}, coarsest {ch.coarsest_max}, omega {ch.omega}, "
             f"{ch.mg_launch} multigrid")
        picked[k] = picked.get(k, 0) + 1
    sides = [w.nodes for w in ws]
    return {"members": len(ws), "particles": n0, "steps": args.ensemble_steps, "ms_per_step": ms / args.ensemble_steps,
            "value": 0.5 * (n0 + n1) * args.ensemble_steps / (ms / 1e3), "unit": UNIT,
            "sides": {str(k): sides.count(k) for k in ensemble.SIDES}, "tuned": picked,
            "tune_s": round(tune_s, 1), "tune_measurements": tuner.measurements,
            "one_particle_pass_over_all_members": fused, "other_structure": other,
            "hbm": {"bytes_per_step": step_bytes, "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                    "frac": round(gbs / peak, 4), "peak_source": kind,
                    "counts": "particle and grid bytes over the whole ensemble step (field solves included)"}}


def large_species_on_device(w, which, gen):
    """The large workload's particles, drawn on the device (seeded): ions
    uniform; electrons half in a Gaussian blob (sigma 0.2 L, re-drawn until
    inside the domain) and half uniform; Maxwellian velocities."""
    import torch

    from pic_b200 import Consts, workloads

    n = w.n_e if which == "e" else w.n_i
    top = float(w.nodes - 1)
    hi = float(np.nextafter(np.float32(top), np.float32(0)))
    x = torch.rand(n, generator=gen, device="cuda") * top
    y = torch.rand(n, generator=gen, device="cuda") * top
    if which == "e":
        h = n // 2
        c, sig = 0.5 * top, 0.2 * top
        bx = torch.randn(h, generator=gen, device="cuda") * sig + c
        by = torch.randn(h, generator=gen, device="cuda") * sig + c
        for _ in range(64):
            bad = (bx < 0) | (bx >= top) | (by < 0) | (by >= top)
            k = int(bad.sum())
            if k == 0:
                break
            bx[bad] = torch.randn(k, generator=gen, device="cuda") * sig + c
            by[bad] = torch.randn(k, generator=gen, device="cuda") * sig + c
        x[:h], y[:h] = bx, by
    x.clamp_(0.0, hi)
    y.clamp_(0.0, hi)
    mass = Consts.me if which == "e" else workloads.ION_MASS
    vth = float(np.sqrt((w.Te if which == "e" else w.Ti) * Consts.qe / mass))
    v = [torch.randn(n, generator=gen, device="cuda") * vth for _ in range(3)]
    return x, y, v[0], v[1], v[2]


def run_large_step(steps=200):
    """The large workload as a fused PIC step: 2049^2 nodes, 64M + 64M
    particles, collisionless, multigrid to a 1e-10 relative residual every
    step, the cell sort every 80 steps; once with the mixed-precision
    multigrid and once with the plain FP64 one, on the same inputs."""
    import torch

    from pic_b200 import Consts, workloads
    from pic_b200.simulation import PICSimulation

    w = workloads.LARGE
    mask, phi_bc = workloads.dirichlet(w)
    species = [dict(name="e", charge=-Consts.qe, mass=Consts.me, np2c=w.np2c(w.n_e), capacity=int(w.n_e * 1.05)),
               dict(name="i", charge=Consts.qe, mass=workloads.ION_MASS, np2c=w.np2c(w.n_i),
                    capacity=int(w.n_i * 1.05))]
    res = {"workload": "large: 2049x2049 nodes, 64M e- (half in a sigma=0.2L blob) + 64M ions, collisionless, "
                       f"multigrid tol 1e-10 every step, sort every 80 steps, {steps} timed steps after 3"}
    for prec in ("mixed", "fp64"):
        gen = torch.Generator(device="cuda")
        gen.manual_seed(7)
        sim = PICSimulation(w.nodes, w.nodes, w.dx, w.dx, w.dt, species, mask, phi_bc, tol=w.tol, max_cycles=60,
                            precision=prec, sort_interval=80, use_graph=True)
        for s, which in enumerate(("e", "i")):
            sim.load(s, *large_species_on_device(w, which, gen))
        torch.cuda.empty_cache()
        sim.init()
        sim.step(3)
        torch.cuda.synchronize()
        n0 = sum(sim.counters()["count"])
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sim.step(steps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        c = sim.counters()
        res[prec] = {"ms_per_step": ms / steps, "value": 0.5 * (n0 + sum(c["count"])) * steps / (ms / 1e3),
                     "unit": UNIT, "last_cycles": c["last_cycles"], "last_rel_res": c["last_rel_res"],
                     "absorbed": c["absorbed"]}
        sim.close()
        del sim
        torch.cuda.empty_cache()
    res["speedup_mixed_vs_fp64"] = round(res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"], 3)
    return res


def run_adjoint():
    """Differentiable workload: 257^2 nodes, 1e6 + 1e6 particles, 200 FP64
    collisionless steps, checkpoints every 20; gradients of the final
    electron-density loss with respect to four wall potentials and a velocity
    perturbation amplitude, against central finite differences."""
    import torch

    from pic_b200 import adjoint

    w = adjoint.AdjWorkload()
    prob, V0, A0, _ = adjoint.build(w)
    prob.forward(V0, A0)
    prob.backward()  # graphs captured
    t0 = time.perf_counter()
    loss = prob.forward(V0, A0)
    t1 = time.perf_counter()
    dV, dA = prob.backward()
    t2 = time.perf_counter()
    fd = {}
    # absorption as computed (wall crossings flip between runs), then frozen at
    # the base run's steps (the fixed mask the adjoint differentiates with)
    for frozen, h, hA in ((False, 1e-3, 1.0), (True, 1e-3, 1.0), (True, 1e-5, 0.1)):
        prob.forward(V0, A0)
        prob.freeze_absorption(frozen)
        g = []
        for q in range(4):
            e = np.zeros(4)
            e[q] = h
            g.append((prob.forward(V0 + e, A0) - prob.forward(V0 - e, A0)) / (2 * h))
        gA = (prob.forward(V0, A0 + hA) - prob.forward(V0, A0 - hA)) / (2 * hA)
        prob.freeze_absorption(False)
        err = max(abs(a - b) for a, b in zip(dV, g)) / max(abs(b) for b in g)
        fd[f"h={h:g} V{', absorption frozen' if frozen else ''}"] = {
            "dV_fd": g, "dA_fd": gA, "max_rel_err_dV": err, "rel_err_dA": abs(dA - gA) / abs(gA)}
    prob.close()
    # every solve a fixed 10 V-cycles and the absorption frozen: the map the
    # adjoint differentiates (a smooth solve map, a fixed absorption mask);
    # what is left between it and central differences is the CIC weights'
    # kinks: particles that sit in different cells in the +h and -h runs
    fixed = adjoint.AdjWorkload(tol=0.0, max_cycles=10)
    prob, V0, A0, _ = adjoint.build(fixed)
    prob.forward(V0, A0)
    fdV, fdA = prob.backward()
    prob.freeze_absorption(True)

    def cells(pr):
        x, y = pr.state()[:2]
        return torch.floor(x).to(torch.int64) * 100000 + torch.floor(y).to(torch.int64)

    for h, hA in ((1e-3, 1.0), (1e-4, 0.1), (1e-6, 0.01)):
        g, kinks = [], []
        for q in range(4):
            e = np.zeros(4)
            e[q] = h
            lp = prob.forward(V0 + e, A0)
            cp = cells(prob).clone()
            lm = prob.forward(V0 - e, A0)
            kinks.append(int((cells(prob) != cp).sum()))
            g.append((lp - lm) / (2 * h))
        gA = (prob.forward(V0, A0 + hA) - prob.forward(V0, A0 - hA)) / (2 * hA)
        err = max(abs(a - b) for a, b in zip(fdV, g)) / max(abs(b) for b in g)
        fd[f"h={h:g} V, absorption frozen, 10 V-cycles per solve"] = {
            "dV_adjoint": list(fdV), "dV_fd": g, "dA_fd": gA, "max_rel_err_dV": err, "rel_err_dA": abs(fdA - gA) / abs(gA),
            "particles_in_other_cells_at_the_end": kinks, "within_1e-4": bool(err <= 1e-4 and abs(fdA - gA) <= 1e-4 * abs(gA))}
    prob.close()
    return {"workload": "257x257 nodes, 1e6 e- + 1e6 ions, 200 FP64 steps, checkpoints every 20, 4 wall electrodes",
            "loss": loss, "dV": list(dV), "dA": dA, "forward_ms": 1e3 * (t1 - t0), "backward_ms": 1e3 * (t2 - t1),
            "backward_over_forward": (t2 - t1) / (t1 - t0), "finite_differences": fd}


def run_e2e(w, arrays, args, world, rank):
    """Public API from pinned host arrays: load, init, K steps, read back particles and phi."""
    import torch
    import torch.distributed as dist

    pinned = [[torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in sp] for sp in arrays]
    sim = make_sim(w, rank, args.sort_interval, mcc=True)
    # read-back buffers (pinned, allocated before the timed region like the
    # inputs): rows x, y, vx, vy, vz of each species, one copy per array
    cap = [int(len(sp[0]) * 1.25) for sp in arrays]
    host_out = [torch.empty(5 * c, dtype=torch.float32).pin_memory() for c in cap]
    host_phi = torch.empty(w.nodes * w.nodes, dtype=torch.float64).pin_memory()
    stream = torch.cuda.current_stream()
    # one untimed pass of the same calls first (args.warmup steps): the first
    # copies into freshly pinned pages, the field views and the step's graph
    # capture are one-time costs of a process, not of a run
    for s, a in enumerate(pinned):
        sim.load(s, *a)
    sim.init()
    sim.step(max(1, args.warmup))
    sim.sync()
    for s in range(2):
        sim.read_particles(s, host_out[s])
    host_phi.copy_(sim.fields()[0], non_blocking=True)
    outs = None
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    ev[0].record(stream)
    for s, a in enumerate(pinned):
        sim.load(s, *a)
    ev[1].record(stream)
    sim.init()
    ev[2].record(stream)
    sim.step(args.steps)
    sim.sync()
    ev[3].record(stream)
    outs = [sim.read_particles(s, host_out[s]) for s in range(2)]
    phi = host_phi.copy_(sim.fields()[0], non_blocking=True)
    ev[4].record(stream)
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[4])
    phases = {k: round(ev[i].elapsed_time(ev[i + 1]), 3) for i, k in enumerate(("load", "init", "steps", "read"))}
    t = torch.tensor([ms], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    n = sum(len(a[0]) for a in arrays)
    h2d = sum(a.numel() * 4 for sp in pinned for a in sp)
    d2h = sum(o.numel() * 4 for o in outs) + phi.numel() * 8
    sim.close()
    return {"value": world * n * args.steps / (float(t.item()) / 1e3), "unit": UNIT,
            "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps, "phase_ms": phases,
            "ms_total": float(t.item()),
            "read_gbs": round(d2h / (phases["read"] / 1e3) / 1e9, 1) if phases["read"] > 0 else None,
            "load_gbs": round(h2d / (phases["load"] / 1e3) / 1e9, 1) if phases["load"] > 0 else None,
            "includes": "H2D of all particles from pinned host memory, init, "
                        f"{args.steps} steps, D2H of particles (one copy per array) and phi into pinned host memory; "
                        "after one untimed pass of the same calls"}


def mg_levels(n, coarse_max=33):
    """Node sides of the multigrid hierarchy of an n x n grid: tile levels, then
    the first level of at most coarse_max nodes, which the direct solve owns."""
    sides = [n]
    while sides[-1] > coarse_max:
        sides.append((sides[-1] - 1) // 2 + 1)
    return sides


def mg_bytes_per_solve(n, precision, cycles):
    """Compulsory HBM bytes of one solve: each kernel's distinct inputs read
    once and outputs written once, at their stored precision (e, g in FP32 for
    the mixed solve, FP64 for the plain one; phi, f and the residual r in FP64;
    the mask 1 B).  Per V-cycle:
      finest down   r (8) + mask (1) read; e, g (2T) and the coarse g (T/4) written
      finest up     e, g (2T) + coarse e (T/4) + mask (1) + phi, r (16) read; phi, r (16) written
      level l >= 1  down: g + mask read, e + coarse g written; up: coarse e + e + g + mask read, e written
                    = (6.5 T + 2) bytes per node of level l
      direct solve  the inverse of the coarse level's free nodes (T each) and its g
    and once per solve the first residual: phi, f (16) + mask (1) read, r (8) + g (T) written."""
    T = 4 if precision == "mixed" else 8
    sides = mg_levels(n)
    G = [k * k for k in sides]
    fine = G[0] * ((9 + 2 * T + T / 4) + (2 * T + T / 4 + 1 + 16 + 16))
    mid = sum(g * (6.5 * T + 2) for g in G[1:-1])
    free = (sides[-1] - 2) ** 2
    direct = free * free * T + 2 * G[-1] * T
    r0 = G[0] * (17 + 8 + T)
    return r0 + cycles * (fine + mid + direct)


def run_poisson(launch="graph"):
    """Large workload: deposit 64M + 64M particles on 2049^2 nodes, solve to 1e-10 from phi = 0."""
    import torch

    from pic_b200 import Consts, _lib, workloads
    from pic_b200.multigrid import MultigridSolver

    w = workloads.LARGE
    n = w.nodes
    G = n * n
    g = torch.Generator(device="cuda")
    g.manual_seed(2)
    rho = torch.zeros(G, dtype=torch.float32, device="cuda")
    top = float(n - 1)
    chunk = 16_000_000
    for which, count in (("e", w.n_e), ("i", w.n_i)):
        q = -Consts.qe if which == "e" else Consts.qe
        scale = q * w.np2c(count) / (w.dx * w.dx)
        done = 0
        while done < count:
            k = min(chunk, count - done)
            if which == "e" and done < count // 2:
                k = min(k, count // 2 - done)
                c = 0.5 * top
                x = torch.randn(k, generator=g, device="cuda") * (0.2 * top) + c
                y = torch.randn(k, generator=g, device="cuda") * (0.2 * top) + c
                x = x.clamp(0, top - 1e-3)
                y = y.clamp(0, top - 1e-3)
            else:
                x = torch.rand(k, generator=g, device="cuda") * (top - 1e-3)
                y = torch.rand(k, generator=g, device="cuda") * (top - 1e-3)
            _lib.call("pic_deposit", _lib.ptr(x), _lib.ptr(y), k, float(scale), _lib.ptr(rho), n, n,
                      _lib.stream_ptr())
            done += k
    mask, _ = workloads.dirichlet(w)
    mask_t = torch.as_tensor(mask, device="cuda")
    f = torch.zeros(G, dtype=torch.float64, device="cuda")
    _lib.call("pic_form_rhs", _lib.ptr(rho), _lib.ptr(mask_t), Consts.eps0, _lib.ptr(f), n, n, _lib.stream_ptr())
    res = {"workload": "large: 2049x2049 nodes, 64M e- (half in a sigma=0.2L blob) + 64M ions, tol 1e-10, phi0 = 0"}
    for prec in ("mixed", "fp64"):
        mg = MultigridSolver(mask, n, n, w.dx, precision=prec, launch=launch)
        phi = torch.zeros(G, dtype=torch.float64, device="cuda")
        mg.solve(phi, f, tol=1e-10, max_cycles=60)  # warm-up (allocations, caches)
        best = None
        for _ in range(3):
            phi.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _, (cycles, rel) = mg.solve(phi, f, tol=1e-10, max_cycles=60)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None or ms < best else best
        nbytes = mg_bytes_per_solve(n, prec, cycles)
        peak, kind = peak_hbm()
        gbs = nbytes / (best / 1e3) / 1e9
        res[prec] = {"ms": round(best, 3), "cycles": cycles, "rel_res": rel,
                     "roofline": {"bound": "hbm", "bytes": nbytes, "achieved": round(gbs, 1), "peak": peak,
                                  "unit": "GB/s", "frac": round(gbs / peak, 4), "peak_source": kind}}
        del mg
    res["speedup_mixed_vs_fp64"] = round(res["fp64"]["ms"] / res["mixed"]["ms"], 3)
    return res


def run_cpu_baseline(w, arrays, steps):
    from oracle import oracle as O
    from oracle import refstep
    from pic_b200 import workloads

    if not O.ref_available():
        return {"value": None, "unavailable": "oracle/_ref/libpicref.so not built"}
    E, el, *_ = workloads.cross_sections()
    ref = refstep.ReferenceCPU(w.nodes, w.dx, w.dt, arrays[0], arrays[1], w.np2c(w.n_e), workloads.ION_MASS,
                               left_V=w.left_V, tol=w.tol, mcc_table=(E, el), gas_density=w.gas_density)
    dt, cycles = refstep.time_steps(ref, steps, warmup=1)
    n = ref.N
    ref.close()
    return {"value": n * steps / dt, "unit": UNIT, "cores": ref.threads, "kind": "reference",
            "sample": f"{steps} full steps of the same workload ({n} particles, 513^2) after 1 warm-up step; "
                      f"multigrid cycles {cycles}", "cpu": refstep.cpu_model()}


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------

def run_reference(args, world, rank):
    if rank != 0:
        return
    from oracle import oracle as O
    from oracle import refstep
    from pic_b200 import workloads

    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libpicref.so not built"}))
        return
    w = workloads.scaled(workloads.MCC, n=args.particles)
    arrays = gen_arrays(w, 0)
    E, el, *_ = workloads.cross_sections()
    ref = refstep.ReferenceCPU(w.nodes, w.dx, w.dt, arrays[0], arrays[1], w.np2c(w.n_e), workloads.ION_MASS,
                               left_V=w.left_V, tol=w.tol, mcc_table=(E, el), gas_density=w.gas_density)
    steps = max(1, args.steps)
    dt, cycles = refstep.time_steps(ref, steps, warmup=max(0, args.warmup))
    value = ref.N * steps / dt
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Philox)",
        "config": {"workload": "mcc: 513x513 nodes, "
                               f"{w.n_e} e- + {w.n_i} ions, left wall 100 V, multigrid tol 1e-8, MCC (elastic table)",
                   "global_batch": ref.N, "parallelism": "host cores"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref.threads, "kind": "reference",
                         "sample": f"{steps} full steps after {args.warmup} warm-up steps; multigrid cycles {cycles}",
                         "cpu": refstep.cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    ref.close()
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    GRAPH_OPTS["use_graph"] = not args.no_graph
    GRAPH_OPTS["mg_launch"] = args.mg_launch
    GRAPH_OPTS["pre_sweeps"], GRAPH_OPTS["post_sweeps"] = args.mg_sweeps
    GRAPH_OPTS["omega"] = args.omega
    GRAPH_OPTS["coarse_fp32"] = args.coarse_fp32
    GRAPH_OPTS["tile"] = args.tile
    GRAPH_OPTS["push_kernel"] = args.push
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.poisson_only:
        import torch

        torch.cuda.set_device(local)
        if rank == 0:
            print(json.dumps({"poisson": run_poisson("host" if args.mg_launch == "host" else "graph")}), flush=True)
        return
    run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
