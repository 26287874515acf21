"""Benchmark of the Barnes-Hut step: steps/s at N=2^20, theta=0.5.

Workload: Plummer sphere (G=1, total mass 1, a=1, r<10a, AHW velocities,
centre of mass removed), N = 2^20, theta = 0.5, eps = 0.01, dt = 1e-3,
synthetic and seeded.  One step = leapfrog KD + full spatial rebuild + force
evaluation + K, replayed from a CUDA graph.  ``value`` is the steps/s of the
mixed-precision form summed over all GPUs; the FP64 plain form is measured
on the same GPU in the same run (``plain_fp64``), and the mixed form's force
error against FP64 direct summation on 4096 seeded targets is reported
(``force_error``): the headline is valid when its RMS relative error is
<= 1e-3.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl nbb|reference]
  python bench.py --workload disk|blobs|ensemble|adjoint   (secondary workloads of
                                                             nbb.workloads, one GPU)

With N > 1 (launched by torch.distributed.run) every rank steps an
independent replica on its own GPU ("replicas only": the path has no
exchange step); the elapsed time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "amsc-nbody_b200"))

METRIC = "steps/s at N=2^20 θ=0.5: mixed vs FP64 path, same B200, rms force err ≤1e-3"
N_DEFAULT = 1 << 20
THETA, EPS, DT, G = 0.5, 0.01, 1e-3, 1.0
L2_FLUSH_BYTES = 256 << 20
HBM_FALLBACK_GBS = 6650.0  # measured copy bandwidth when MEASURED_PEAKS.json is absent
ERROR_TARGETS = 4096


def workload_name(n):
    exp = int(round(math.log2(n))) if n > 0 else 0
    size = f"2^{exp}" if (1 << exp) == n else str(n)
    return f"plummer N={size} theta={THETA} eps={EPS} dt={DT} G={G} (seed 0)"


# ------------------------------------------------------------ clocks ---

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons, each stamped with
    its arrival time on this host, so that a summary can cover exactly the
    timed regions (the sampler starts well before them: nvidia-smi takes a
    moment to produce its first line)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 20

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []  # (arrival time, csv line)
        self.thread = None
        self.windows = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", str(self.PERIOD_MS)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 10.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def __exit__(self, *exc):
        time.sleep(2.5 * self.PERIOD_MS / 1000.0)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)

    def window(self):
        """Context manager marking one timed region."""
        sampler = self

        class _W:
            def __enter__(self):
                self.t0 = time.time()
                return self

            def __exit__(self, *exc):
                sampler.windows.append((self.t0, time.time()))
                return False

        return _W()

    def summary(self):
        """Median SM clock, max clock and throttle reasons of the samples that
        arrived inside a timed region (one sampler period of slack after it)."""
        slack = self.PERIOD_MS / 1000.0
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for t, line in self.lines:
            if self.windows and not any(a <= t <= b + slack for a, b in self.windows):
                continue
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        timed_s = sum(b - a for a, b in self.windows)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0, "timed_s": timed_s}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "timed_s": timed_s, "period_ms": self.PERIOD_MS}


# ------------------------------------------------------- distributed ---

def dist_setup():
    """Rank bookkeeping for torchrun launches; returns (rank, world, local)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(value: float, world: int) -> float:
    """Max of a per-rank scalar over all ranks (identity on one rank)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, world: int) -> float:
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def dist_teardown(world):
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# --------------------------------------------------------- measuring ---

def nominal_fp32_tflops(sm_mhz: float, sms: int = 148) -> float:
    """FP32 SIMT FMA peak: SMs x 128 lanes x 2 flops x clock."""
    return sms * 128 * 2 * sm_mhz * 1e6 / 1e12


def time_steps(nbb, sim, torch, stream, flush, steps):
    """Per-step CUDA-event times (ms) of `steps` graph-replayed steps; L2 is
    flushed between steps, outside the timed events."""
    times = []
    launches0 = nbb.kernel_launch_count()
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        sim.step()
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return times, nbb.kernel_launch_count() - launches0


def force_error(nbb, p, precision, targets):
    exact = np.stack(nbb.compute_direct_accelerations(p.mass, p.x, p.y, p.z, G, EPS, targets=targets))
    ax, ay, az = nbb.compute_accelerations(p, THETA, EPS, G, precision=precision)
    a = np.stack([ax, ay, az])[:, targets]
    rel = np.linalg.norm(a - exact, axis=0) / np.linalg.norm(exact, axis=0)
    return {"rms_rel": float(np.sqrt(np.mean(rel ** 2))), "max_rel": float(rel.max()),
            "rel_l2": float(np.linalg.norm(a - exact) / np.linalg.norm(exact)),
            "targets": int(targets.size), "reference": "FP64 direct summation (GPU kernel)"}


def cpu_baseline(p, samples=3):
    """The oracle (CPU restatement of the reference pipeline) on this host,
    every core via OpenMP: `samples` full steps -- kick-drift, rebuild, force
    evaluation of every target, kick -- on a copy of the state; the value is
    the median step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    cores = os.cpu_count() or 1
    m = np.ascontiguousarray(p.mass)
    x, y, z, vx, vy, vz = (np.array(a, dtype=np.float64) for a in (p.x, p.y, p.z, p.vx, p.vy, p.vz))
    a = pyoracle.pipeline(m, x, y, z, theta=THETA, soft=EPS, g=G, n_threads=cores)
    ax, ay, az = a["ax"], a["ay"], a["az"]
    times = []
    for _ in range(samples):
        t0 = time.perf_counter()
        x, y, z, vx, vy, vz = pyoracle.kick_drift(x, y, z, vx, vy, vz, ax, ay, az, DT)
        a = pyoracle.pipeline(m, x, y, z, theta=THETA, soft=EPS, g=G, n_threads=cores)
        ax, ay, az = a["ax"], a["ay"], a["az"]
        vx, vy, vz = pyoracle.kick(vx, vy, vz, ax, ay, az, DT)
        times.append(time.perf_counter() - t0)
    dt = statistics.median(times)
    return {"value": 1.0 / dt, "unit": "steps/s", "cores": cores, "kind": "port",
            "sample": f"median of {samples} full KDK steps of all {len(p)} particles (kick-drift, "
                      f"rebuild, force evaluation of every target, kick; "
                      f"{', '.join(f'{t:.2f}' for t in times)} s; OpenMP over targets)"}


def run_nbb(args, rank, world, local):
    import torch

    import nbb
    from nbb import ics

    torch.cuda.set_device(local)
    n = args.n
    p = ics.plummer(n, seed=0)
    stream = torch.cuda.Stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    results = {}
    sims = {}
    for name, prec in (("mixed", nbb.PRECISION_MIXED), ("fp64", nbb.PRECISION_FP64)):
        sim = nbb.Simulation(p, nbb.SimulationConfig(DT, THETA, EPS, G, precision=prec, device=local))
        sim.set_stream(stream.cuda_stream)
        sim.initialize()
        sims[name] = sim
    with ClockSampler(local) as sampler:
        for name, sim in sims.items():
            for _ in range(args.warmup):
                sim.step()
            torch.cuda.synchronize()
            barrier(world)
            torch.cuda.synchronize()
            with sampler.window():
                times, launches = time_steps(nbb, sim, torch, stream, flush, args.steps)
                torch.cuda.synchronize()
            barrier(world)
            total_ms = max_over_ranks(sum(times), world)
            stage_ms, st = sim.profile()
            results[name] = {"ms_per_step": total_ms / args.steps, "step_ms": times, "launches": launches,
                             "stages_ms": stage_ms, "interactions": st.interactions,
                             "mac_tests": st.mac_tests, "stack_overflow": st.stack_overflow,
                             "n_groups": st.n_groups, "n_octree_nodes": st.n_octree_nodes,
                             "group_size": st.group_size, "cache_depth": st.cache_depth}
        # end to end through the public API: pinned host state in, step, state out
        sim = sims["mixed"]
        pin = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in p.arrays()]
        hst = [t.numpy() for t in pin]
        sim.upload(mass=hst[0], x=hst[1], y=hst[2], z=hst[3], vx=hst[4], vy=hst[5], vz=hst[6])
        torch.cuda.synchronize()
        e2e_times = []
        for k in range(args.warmup + args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                flush.zero_()
                e0.record(stream)
            # upload, step and download in one call; the positions' copy back
            # overlaps the rebuild and the walk
            sim.step_host(mass=hst[0], x=hst[1], y=hst[2], z=hst[3], vx=hst[4], vy=hst[5], vz=hst[6],
                          out=hst[1:])
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            if k >= args.warmup:
                e2e_times.append(e0.elapsed_time(e1))
    e2e_ms = max_over_ranks(sum(e2e_times), world) / args.steps
    return p, results, e2e_ms, sampler.summary()


# Algorithmic bytes of the step's rebuild (the level-order build of a mixed
# step): per particle, per unique-key group (= occupied leaf), per octree node
# and per internal node, each term the sum of the arrays that kernel must read
# once and write once.
BUILD_BYTES_PER_PARTICLE = (152 + 32 + 4 * 16     # kick-drift + box (+ position records), encode, 4 sort passes
                            + 20 + 76 + 32 + 1)   # groups, Morton gather, leaf mass, target-group scan
BUILD_BYTES_PER_GROUP = 16 + 24 + 20 + 124        # group arrays, level spans, cell ranks, leaf records
BUILD_BYTES_PER_OCTREE_NODE = 32 + 48 + 12        # cell entries, read once as a child, arrival counter
BUILD_BYTES_PER_INTERNAL_NODE = 160               # level pass: entries, LevelNode, MixedNode, child list


def build_algorithmic_bytes(n, groups, nodes):
    return (BUILD_BYTES_PER_PARTICLE * n + BUILD_BYTES_PER_GROUP * groups + BUILD_BYTES_PER_OCTREE_NODE * nodes
            + BUILD_BYTES_PER_INTERNAL_NODE * max(nodes - groups, 0))


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f)
    except OSError:
        return {}


PROFILE_CASES = ("step", "adjoint", "direct", "frozen", "diagnostics", "frame", "ensemble")


def profile_run(args):
    """One small, self-contained run of the kernels of one case, for ncu
    captures (no timing, no JSON line).  Workload: the benchmark's Plummer
    sphere at --n (theta 0.5, eps 0.01, dt 1e-3, G 1).

      step         --steps graph-replayed steps of the --precision form (optional
                   --group-size pins the mixed walk's target group size), then
                   one diagnostic force evaluation with per-stage events
      adjoint      a rollout of --adjoint steps (checkpoints every 32) and its
                   backward pass for the loss sum(x_T) / n
      direct       FP64 direct summation for 4096 seeded targets
      frozen       frozen-structure replay of 4 perturbed copies over --steps steps
      diagnostics  conserved quantities with the tree and all-pairs potentials
      frame        one quantized frame of 100000 sampled particles
      ensemble     --steps steps of 64 Plummer systems, N log-uniform in
                   [1024, 131072], one segmented launch per stage
    """
    import nbb
    from nbb import ics

    prec = nbb.PRECISION_MIXED if args.precision == "mixed" else nbb.PRECISION_FP64
    cfg = nbb.SimulationConfig(DT, THETA, EPS, G, precision=prec, group_size=args.group_size)
    if args.profile == "ensemble":
        ens = ics.plummer_ensemble(64, seed=3)
        sim = nbb.EnsembleSimulation(ens, cfg)
        sim.initialize()
        sim.run(args.steps)
        print("ensemble steps", args.steps, "particles", len(ens.particles))
        return
    p = ics.plummer(args.n, seed=0)
    if args.profile == "direct":
        rng = np.random.Generator(np.random.Philox(12345))
        tg = np.sort(rng.choice(args.n, min(ERROR_TARGETS, args.n), replace=False)).astype(np.int32)
        ax = nbb.compute_direct_accelerations(p.mass, p.x, p.y, p.z, G, EPS, targets=tg)[0]
        print("direct", float(ax[0]))
        return
    if args.profile == "frozen":
        rng = np.random.Generator(np.random.Philox(7))
        copies = []
        for _ in range(4):
            q = ics.ParticleData(*(np.array(a) for a in p.arrays()))
            q.x[rng.integers(0, args.n)] += 1e-6
            copies.append(q)
        out = nbb.frozen_rollout(p, cfg, copies, args.steps)
        print("frozen copies", out.shape[0], float(out[0, 0, 0]))
        return
    sim = nbb.Simulation(p, cfg)
    sim.initialize()
    if args.profile == "adjoint":
        sim.rollout(args.adjoint, 32)
        gm, gx, gv = sim.backward(np.full((3, args.n), 1.0 / args.n))
        print("backward done", float(gx[0, 0]))
        return
    if args.profile == "diagnostics":
        d0 = sim.diagnostics(nbb.POTENTIAL_TREE)
        d1 = sim.diagnostics(nbb.POTENTIAL_DIRECT) if args.n <= (1 << 17) else d0
        print("energies", d0["total_energy"], d1["total_energy"])
        return
    if args.profile == "frame":
        frame = sim.capture_frame(100000, sequence=1)
        print("frame bytes", len(frame))
        return
    sim.run(args.steps)
    stages, st = sim.profile()
    print({k: round(v, 4) for k, v in stages.items()}, "interactions", st.interactions,
          "mac_tests", st.mac_tests, "groups", st.n_groups, "nodes", st.n_octree_nodes)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["nbb", "reference"], default="nbb")
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-error", action="store_true")
    ap.add_argument("--workload", choices=["plummer", "disk", "blobs", "ensemble", "adjoint"],
                    default="plummer")
    ap.add_argument("--profile", choices=PROFILE_CASES, default=None,
                    help="run one small case of the kernels for an ncu capture (no timing)")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed", help="--profile step form")
    ap.add_argument("--group-size", type=int, default=0, help="--profile: mixed walk group size (0 = tuned)")
    ap.add_argument("--adjoint", type=int, default=4, help="--profile adjoint: rollout steps")
    args = ap.parse_args()
    if args.profile:
        profile_run(args)
        return
    args.warmup = max(args.warmup, 3)
    if args.workload != "plummer":
        from nbb import workloads

        print(json.dumps(workloads.WORKLOADS[args.workload]()), flush=True)
        return
    rank, world, local = dist_setup()
    try:
        if args.impl == "reference":
            line = run_reference(args, rank, world, local)
        else:
            line = bench_nbb(args, rank, world, local)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        dist_teardown(world)


def bench_nbb(args, rank, world, local):
    import nbb

    p, res, e2e_ms, clocks = run_nbb(args, rank, world, local)
    mixed, plain = res["mixed"], res["fp64"]
    steps_s = world * 1000.0 / mixed["ms_per_step"]
    plain_s = world * 1000.0 / plain["ms_per_step"]
    line = {
        "metric": METRIC, "value": steps_s, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mixed["ms_per_step"],
        # median of the per-step CUDA-event times (this rank), beside the mean the value uses
        "ms_per_step_median": statistics.median(mixed["step_ms"]), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 interactions / f64 state",
        "data": "synthetic (seeded Plummer sphere)",
        "config": {"workload": workload_name(args.n), "n": args.n, "theta": THETA, "softening": EPS,
                   "dt": DT, "G": G, "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "flushed between timed steps (256 MiB write, outside the step events)",
                   "step": "CUDA-graph replay of KD + rebuild + traversal + K"},
        "plain_fp64": {"value": plain_s, "unit": "steps/s", "ms_per_step": plain["ms_per_step"],
                       "ms_per_step_median": statistics.median(plain["step_ms"]),
                       "dtype": "f64", "stages_ms": plain["stages_ms"],
                       "interactions": plain["interactions"]},
        "speedup_mixed_vs_fp64": plain["ms_per_step"] / mixed["ms_per_step"],
        "stages_ms": mixed["stages_ms"],
        "interactions": mixed["interactions"], "mac_tests": mixed["mac_tests"],
        # nodes accepted for lack of stack space (0: the test ran everywhere)
        "stack_overflow": mixed["stack_overflow"],
        "octree": {"groups": mixed["n_groups"], "nodes": mixed["n_octree_nodes"]},
        "gpu_launches": int(mixed["launches"]),
        "clocks": clocks,
    }
    # e2e: the same metric through the public API with host buffers
    bi = 7 * args.n * 8
    bo = 6 * args.n * 8
    line["e2e"] = {"value": world * 1000.0 / e2e_ms, "unit": "steps/s", "h2d_bytes_per_step": bi,
                   "d2h_bytes_per_step": bo}
    # roofline of the dominant kernel (mixed traversal): 20 flops/interaction
    trav_ms = mixed["stages_ms"]["traversal"]
    achieved = 20.0 * mixed["interactions"] / (trav_ms * 1e-3) / 1e12
    peak32_scalar = nbb.measure_fma_tflops(nbb.PRECISION_MIXED)
    peak32_packed = nbb.measure_fma_tflops(2)
    peak32 = max(peak32_scalar, peak32_packed)  # the walk issues packed FFMA2
    peak64 = nbb.measure_fma_tflops(nbb.PRECISION_FP64)
    sm_mhz = clocks.get("sm_max_mhz") or 1965.0
    line["roofline"] = {"bound": "fp32", "achieved": achieved, "peak": peak32, "unit": "TFLOP/s",
                        "frac": achieved / peak32,
                        # DRAM bytes per launch come from an ncu capture, which this timed run
                        # does not take
                        "traffic": None,
                        "kernel": "traverse_mixed_kernel",
                        "peak_source": "measured in this run: the larger of scalar FFMA "
                                       f"({peak32_scalar:.1f}) and packed FFMA2 ({peak32_packed:.1f}) "
                                       "SIMT FP32 throughput kernels (MEASURED_PEAKS.json has HBM and "
                                       f"bf16-tensor figures only; nominal {nominal_fp32_tflops(sm_mhz):.1f})",
                        "flops_per_interaction": 20,
                        "interactions_per_s": mixed["interactions"] / (trav_ms * 1e-3)}
    ptrav = plain["stages_ms"]["traversal"]
    p_ach = 20.0 * plain["interactions"] / (ptrav * 1e-3) / 1e12
    line["plain_fp64"]["roofline"] = {"bound": "fp64", "achieved": p_ach, "peak": peak64,
                                      "unit": "TFLOP/s", "frac": p_ach / peak64,
                                      "traffic": None,
                                      "kernel": "traverse_fp64_kernel",
                                      "interactions_per_s": plain["interactions"] / (ptrav * 1e-3)}
    peaks = load_peaks()
    hbm = peaks.get("hbm_gbs")
    hbm_source = "MEASURED_PEAKS.json hbm_gbs (of measured)"
    if not hbm:
        hbm, hbm_source = HBM_FALLBACK_GBS, "fallback 6650 GB/s, an earlier measurement on this pool (of fallback)"
    st = mixed["stages_ms"]
    build_ms = st["bbox"] + st["morton_sort_groups"] + st["tree"]
    build_bytes = build_algorithmic_bytes(args.n, mixed["n_groups"], mixed["n_octree_nodes"])
    build_gbs = build_bytes / (build_ms * 1e-3) / 1e9
    line["build_roofline"] = {"bound": "hbm", "achieved": build_gbs, "peak": hbm, "unit": "GB/s",
                              "frac": (build_gbs / hbm) if hbm else None,
                              "algorithmic_bytes": build_bytes, "ms": build_ms,
                              "peak_source": hbm_source}
    line["group_size"] = mixed["group_size"]
    line["cache_depth"] = mixed["cache_depth"]
    if rank == 0 and not args.no_error:
        rng = np.random.Generator(np.random.Philox(12345))
        tg = np.sort(rng.choice(args.n, min(ERROR_TARGETS, args.n), replace=False)).astype(np.int32)
        line["force_error"] = {"mixed": force_error(nbb, p, nbb.PRECISION_MIXED, tg),
                               "fp64": force_error(nbb, p, nbb.PRECISION_FP64, tg)}
        line["valid_rms_le_1e-3"] = line["force_error"]["mixed"]["rms_rel"] <= 1e-3
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(p)
    return line if rank == 0 else None


def run_reference(args, rank, world, local):
    """The reference's own implementation of the step: its CUDA sources,
    unmodified, built into oracle/_ref/libnbody_ref.so and driven through its
    function-level API in Simulation::step order (G=1), on this GPU.  Rank 0
    alone runs it."""
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    from nbb import ics

    p = ics.plummer(args.n, seed=0)
    if not pyoracle.ref_available():
        # no reference build travelled with the snapshot: time the oracle
        # port on the host cores instead
        base = cpu_baseline(p)
        return {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": "steps/s",
                "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": 1000.0 / base["value"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded Plummer sphere)",
                "config": {"workload": workload_name(args.n), "n": args.n},
                "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": "steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
    steps = args.steps
    ms = np.zeros(args.warmup + steps, np.float32)
    with ClockSampler(local) as sampler:
        pyoracle.ref_simulate(p, args.warmup + steps, DT, THETA, EPS, G, step_ms=ms)
    timed = ms[args.warmup:]
    ms_per_step = float(timed.mean())
    value = 1000.0 / ms_per_step
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": 1,
            "steps": steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Plummer sphere)",
            "config": {"workload": workload_name(args.n), "n": args.n, "theta": THETA,
                       "softening": EPS, "dt": DT, "G": G,
                       "implementation": "reference CUDA sources (unmodified) built for sm_100a, "
                                         "Simulation::step order, per-step allocation and host "
                                         "syncs as in the reference"},
            "cpu_baseline": {"value": value, "unit": "steps/s", "cores": 1, "kind": "reference",
                             "sample": f"{steps} reference steps on the GPU, driven by one host "
                                       "thread (the reference has no CPU implementation of the path)"},
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "clocks": sampler.summary()}


if __name__ == "__main__":
    main()
