"""Throughput of the MLS-MPM baking substep (particle-substeps/s) on B200s.

Workload: the 1,000,000-particle box loaf on a 128^3 grid (Ding viscoplastic dough
with temperature dependence, coupled gas porosity, thermal-water transport, a
per-particle gas source rate alpha_i ~ U[0, 1e-3], gravity, dt = 5e-5). One
bench "step" is one substep of every particle. Inputs are seeded synthetic data
larger than L2, generated on the host.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs under torchrun: every rank simulates its own copy of the loaf (the
substep has no exchange between independent bodies), ranks are timed on the
device, and the slowest rank's time sets the whole-job throughput.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-substeps/s at 1M particles (plain vs surrogate vs fwd+bwd) on 1 B200"
UNIT = "particle-substeps/s"

# Algorithmic HBM bytes of one substep (gas mode), every required state array read once and
# written once at the reference's dtypes; derivable constants (masses, capacities) count 0.
# Per particle: reads x, v 12 each, C, F, Fe, tau 36 each, porosity, gelled 4 each, temperature,
# water, gas moles 8 each, V0 4 = 204 B; writes the same less V0 = 200 B. Per active node:
# mechanics 56 (momentum/mass write+read 32, velocity write+read 24) plus transport 176 (seven
# float64 scattered fields write+read 112, node temperature/saturation 32, dT/dW 32).
BYTES_PER_PARTICLE = 404
BYTES_PER_ACTIVE_NODE = 232
# Forward + backward (Rollout with a checkpoint every k substeps), algorithmic bytes per
# particle-substep: the forward substep (404), its recomputation from the checkpoint in the reverse
# sweep (404), the reverse kernels' read of the substep's input state (204), the adjoint of every
# state array read once and written once at the state's precision (204 + 200), and the checkpoint
# written in the forward and read back for the recomputation (2 x 200 / k). Per active node: the
# forward and recomputed grid passes (2 x 232) and the node adjoints of momentum, mass, velocity and
# the transport fields written and read once (232).
FWD_BWD_CHECKPOINT_EVERY = 8
BYTES_PER_ACTIVE_NODE_FWD_BWD = 3 * 232


def bytes_per_particle_fwd_bwd(every=FWD_BWD_CHECKPOINT_EVERY):
    return 404 + 404 + 204 + 404 + 2 * 200 / every  # 1466 B at a checkpoint every 8 substeps

CLOCK_WINDOW_S = 1.0
# The headline loaf is re-sorted by grid cell every SORT_INTERVAL substeps inside the stepping calls
# (MpmSimulator sort_interval): particles drift out of cell order as the loaf settles and flows, and
# the scatter kernels slow down with the order (no re-sort: 359 -> 548 us per substep over the
# 1000-substep bake).
SORT_INTERVAL = 100


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--particles", type=int, default=1_000_000)
    p.add_argument("--resolution", type=int, default=128)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-variants", action="store_true", help="skip the surrogate and fwd+bwd forms")
    p.add_argument("--surrogate-only", type=int, metavar="STEPS", default=None,
                   help="time only STEPS substeps of the yielding loaf with the learned return map attached "
                        "(for profiling the surrogate kernel)")
    p.add_argument("--clock-window", type=float, default=CLOCK_WINDOW_S,
                   help="seconds of untimed substeps (on a second copy of the loaf) sampled for clocks before "
                        "the timed region; 0 skips them (profiling runs)")
    p.add_argument("--rollout-only", type=int, nargs=2, metavar=("STEPS", "EVERY"), default=None,
                   help="time only forward + adjoint of STEPS substeps, a checkpoint every EVERY, on the "
                        "headline loaf (for profiling the reverse sweep)")
    return p.parse_args()


class ClockSampler:
    """SM clock and clock-event (throttle) reasons of one GPU, sampled through NVML every
    ``interval`` seconds on a host thread while the block runs (NVML is what nvidia-smi reads; a
    direct query takes well under a millisecond, so even a timed region of a few milliseconds gets
    samples). Falls back to ``nvidia-smi -lms 100`` when NVML cannot be loaded."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index, interval=0.002):
        self.index = index
        self.interval = interval
        self.proc = None
        self.lines = []
        self.samples = []  # (seconds since start, sm MHz, max sm MHz, set of reason names)
        self._stop = threading.Event()
        self._nvml = None
        self._handle = None

    def _open_nvml(self):
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            props = torch.cuda.get_device_properties(self.index)
            handle = None
            uuid = str(getattr(props, "uuid", ""))
            if uuid:
                try:
                    handle = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
                except pynvml.NVMLError:
                    handle = None
            if handle is None:
                bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
                handle = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self._nvml, self._handle = pynvml, handle
            return True
        except Exception:  # noqa: BLE001 -- any NVML failure selects the nvidia-smi path
            self._nvml = None
            return False

    def _poll_nvml(self):
        nv, h = self._nvml, self._handle
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        t0 = time.perf_counter()
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            except Exception:  # noqa: BLE001
                break
            self.samples.append((time.perf_counter() - t0, float(sm), float(smax),
                                 {k for k, b in bits.items() if mask & b}))
            self._stop.wait(self.interval)

    def __enter__(self):
        if self._open_nvml():
            self.thread = threading.Thread(target=self._poll_nvml, daemon=True)
            self.thread.start()
            return self
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        self._stop.set()
        if self._nvml is not None:
            self.thread.join(timeout=5)
            return
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def mark(self):
        """Index of the next sample (to summarise a part of the sampled window)."""
        return len(self.samples)

    def summary(self, first=0, last=None):
        sm, smax, reasons = [], 0.0, set()
        for _, clock, top, active in self.samples[first:last]:
            sm.append(clock)
            smax = max(smax, top)
            reasons |= active
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = max(smax, float(parts[1]))
            except ValueError:
                continue
            for name, flag in zip(self.NAMES, parts[4:8]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self._nvml is not None else "nvidia-smi"}


def load_peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(n):
    """Per-launch DRAM bytes (read + write) of each kernel from the committed ncu capture, scaled to
    ``n`` particles (the kernels' traffic is per particle up to the small grid part)."""
    path = ROOT / "profiles" / "traffic.json"
    if not path.exists():
        return {}
    data = json.loads(path.read_text())
    return {k: v["bytes_per_launch"] * n / v["particles"] for k, v in data.items() if isinstance(v, dict)}


def active_node_count(sim):
    import torch
    return int((sim.grid_state.node_masses > 0).sum().item())


def cpu_baseline_sample(scene, seconds=20.0, max_steps=50):
    """The CPU oracle on the same scene, all host threads, for about ``seconds``."""
    from oracle import ora
    from oracle.sim import OracleSimulator
    from baking_b200.scenes import make_simulator
    threads = os.cpu_count() or 1
    ora.set_threads(threads)
    sim = make_simulator(scene, engine=OracleSimulator)
    sim.Step()  # warm-up (allocations, page faults)
    steps, start = 0, time.perf_counter()
    while steps < max_steps:
        sim.Step()
        steps += 1
        if time.perf_counter() - start > seconds:
            break
    elapsed = time.perf_counter() - start
    n = scene.particle_count
    # The same oracle on one host thread, one substep (about 5 s at 1M particles).
    ora.set_threads(1)
    t1 = time.perf_counter()
    sim.Step()
    one = time.perf_counter() - t1
    ora.set_threads(threads)
    return {"value": n * steps / elapsed, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} substeps of the {n}-particle loaf after 1 warm-up substep ({elapsed:.1f} s)",
            "single_core": {"value": n / one, "unit": UNIT, "cores": 1,
                            "sample": f"1 substep of the same loaf on one thread ({one:.1f} s)"}}


def run_reference(args):
    """Reference arm: the CPU oracle of the reference substep, all host threads."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from baking_b200.scenes import box_loaf
    scene = box_loaf(args.resolution, args.particles)
    from oracle import ora
    from oracle.sim import OracleSimulator
    from baking_b200.scenes import make_simulator
    threads = os.cpu_count() or 1
    ora.set_threads(threads)
    sim = make_simulator(scene, engine=OracleSimulator)
    for _ in range(args.warmup):
        sim.Step()
    budget = 90.0
    steps, start = 0, time.perf_counter()
    while steps < args.steps:
        sim.Step()
        steps += 1
        if time.perf_counter() - start > budget:
            break
    elapsed = time.perf_counter() - start
    value = scene.particle_count * steps / elapsed
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": f"box loaf, {scene.particle_count} particles, {args.resolution}^3 grid, "
                                   "Ding+gas+thermal-water, dt=5e-5", "inputs": "larger than L2"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{steps} substeps of the full loaf (bounded to ~{budget:.0f} s)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    from baking_b200 import _lib
    from baking_b200.scenes import box_loaf, make_simulator

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    scene = box_loaf(args.resolution, args.particles, seed=rank)
    sim = make_simulator(scene, diagnostics="lean", sort_interval=SORT_INTERVAL)
    n = scene.particle_count
    if args.surrogate_only:
        from baking_b200.surrogate import LoadReturnSurrogate, ReturnMapSurrogate
        loaf = box_loaf(args.resolution, args.particles, seed=rank, initial_temperature=318.15, prestrain=0.08)
        ysim = make_simulator(loaf, diagnostics="lean")
        sur = ReturnMapSurrogate(LoadReturnSurrogate(ROOT / "baking_b200" / "data" / "return_surrogate_box_loaf.npz"))
        sur.attach(ysim)
        ysim.AdvanceUnchecked(max(1, args.warmup))
        t, _ = _timed(lambda: ysim.AdvanceUnchecked(args.surrogate_only), dist, torch.cuda.current_stream())
        ysim.CheckState()
        if rank == 0:
            print(json.dumps({"metric": "surrogate particle-substeps/s (yielding loaf)", "unit": UNIT,
                              "value": world * loaf.particle_count * args.surrogate_only / t,
                              "steps": args.surrogate_only, "paths": sur.statistics()}))
        if dist:
            dist.destroy_process_group()
        return
    if args.rollout_only:
        steps, every = args.rollout_only
        out = rollout_variant(sim, dist, torch.cuda.current_stream(), world,
                              f"box loaf {n} particles, {args.resolution}^3, Ding + gas + thermal-water",
                              fb_steps=steps, every=every)
        if rank == 0:
            print(json.dumps(dict(out, metric="forward + adjoint particle-substeps/s", n_gpus=world)))
        if dist:
            dist.destroy_process_group()
        return
    # Warm-up; after the first substep every kernel is timed, which picks the dominant kernel. In
    # the timed region only that kernel carries CUDA events (each event pair on the stream costs a
    # few microseconds; all nine kernels' cost 56 us per substep), and the per-kernel breakdown comes
    # from a profiled pass after it.
    sim.AdvanceUnchecked(1)
    warm_events = _lib.KernelTimer()
    with warm_events:
        for _ in range(max(1, args.warmup - 1)):
            sim.AdvanceUnchecked(1)
    sim.SortParticles()  # first-call set-up of the re-sort (kernel loading, scratch) outside the timed region
    torch.cuda.synchronize()
    warm = warm_events.summary()
    dominant_name = max(warm, key=lambda k: warm[k]["total_s"]) if warm else None
    if dist:
        dist.barrier()

    stream = torch.cuda.current_stream()
    kernel_events = _lib.KernelTimer(only=dominant_name)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        # Clock window: a second copy of the loaf runs the same substeps for CLOCK_WINDOW_S seconds
        # under the sampler just before the timed region, so the clock record covers sustained load
        # even when the timed region lasts milliseconds; the timed loaf's state is untouched by it.
        if args.clock_window > 0:
            window_sim = make_simulator(scene, diagnostics="lean")
            torch.cuda.synchronize()
            t_window = time.perf_counter()
            while time.perf_counter() - t_window < args.clock_window:
                window_sim.AdvanceUnchecked(25)
                torch.cuda.synchronize()
            del window_sim
        sim.AdvanceUnchecked(1)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        timed_first = clocks.mark()
        with kernel_events:
            start.record(stream)
            sim.AdvanceUnchecked(args.steps)
            end.record(stream)
        torch.cuda.synchronize()
        timed_last = clocks.mark()
    elapsed = start.elapsed_time(end) / 1e3
    elapsed = reduce_max(elapsed, dist)
    sim.CheckState()
    timed_kernels = kernel_events.summary()
    breakdown_steps = max(1, min(args.steps, 50))
    breakdown_events = _lib.KernelTimer()
    with breakdown_events:
        sim.AdvanceUnchecked(breakdown_steps)
    per_kernel = breakdown_events.summary()
    launches_per_step = sum(v["count"] for v in per_kernel.values()) / breakdown_steps
    active = active_node_count(sim)

    # End to end through the public API: pinned host inputs (the per-particle gas source rates) uploaded
    # for every substep, the substep (SubstepGraphs: one graph launch per substep, with the step-result
    # reduction, chained so that each substep scatters the next one's transport fields ahead), and the
    # step's result (grid mass, kinetic energy) read back to the host. Each
    # substep's upload runs on a copy stream while the substep before it computes; each result lands
    # in mapped host memory and is read while the next substep computes.
    from baking_b200.batch import SubstepGraphs
    # The captured substeps do not re-sort: sort now (the periodic re-sort would have by this
    # point), and upload the per-particle rates in the particles' current order.
    sim.SortParticles()
    order = sim.particle_order.cpu().numpy()
    host_rates = torch.from_numpy(np.ascontiguousarray(scene.gas_source_rates[order])).pin_memory()
    e2e_steps = max(1, min(args.steps, 100))
    stepper = SubstepGraphs(sim, inputs=[sim.material.production_parameter], host_results=True,
                            chained=True).capture()
    copy_stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    wall0 = time.perf_counter()
    e0.record(stream)
    results = []
    pending = None
    stepper.load([host_rates], 0, copy_stream)
    for k in range(e2e_steps):
        step = stepper.Advance(1)
        if k + 1 < e2e_steps:
            stepper.load([host_rates], 0, copy_stream)  # the next substep's inputs, during this one
        if pending is not None:
            results.append(pending.get())  # the previous substep's result, during this one
        pending = step
    results.append(pending.get())
    result = results[-1]
    if len(results) != e2e_steps or not all(math.isfinite(v) for r in results for v in r):
        raise RuntimeError("end-to-end loop lost or corrupted a step result")
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_elapsed = max(e0.elapsed_time(e1) / 1e3, time.perf_counter() - wall0)
    e2e_elapsed = reduce_max(e2e_elapsed, dist)
    del result, stepper

    peak, peak_kind = load_peaks()
    traffic = load_traffic(n)
    dominant = (dominant_name, timed_kernels[dominant_name]) if dominant_name in timed_kernels else None
    roofline = None
    if dominant:
        name, info = dominant
        algo = sim.AlgorithmicBytes(name, active)
        achieved = algo / info["mean_s"] / 1e9 if algo else None
        roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak if achieved else None, "peak_source": peak_kind,
                    "traffic": traffic.get(name), "launches": info["count"], "mean_us": info["mean_s"] * 1e6,
                    "share": per_kernel[name]["total_s"] / sum(v["total_s"] for v in per_kernel.values())}
    step_bytes = n * BYTES_PER_PARTICLE + active * BYTES_PER_ACTIVE_NODE
    value = world * n * args.steps / elapsed
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": f"box loaf, {n} particles per GPU, {args.resolution}^3 grid, Ding+gas+"
                                   "thermal-water, per-particle gas source, dt=5e-5",
                       "particles": n, "resolution": args.resolution, "active_nodes": active,
                       "inputs": "larger than L2 (about 0.6 GB of particle state per GPU)",
                       "parallelism": f"replicas{world}"},
            "roofline": roofline,
            "step_roofline": {"bytes_per_step": step_bytes, "achieved_gbs": step_bytes * args.steps / elapsed / 1e9,
                              "peak": peak, "frac": step_bytes * args.steps / elapsed / 1e9 / peak},
            "kernels": {k: {"launches": v["count"], "mean_us": v["mean_s"] * 1e6} for k, v in per_kernel.items()},
            "kernels_source": f"{breakdown_steps} profiled substeps after the timed region (every kernel timed)",
            "gpu_launches": int(round(launches_per_step * args.steps)),
            "e2e": {"value": world * n * e2e_steps / e2e_elapsed, "unit": UNIT,
                    "h2d_bytes_per_step": int(host_rates.numel() * 4), "d2h_bytes_per_step": int(result_bytes()),
                    "steps": e2e_steps},
            "clocks": dict(clocks.summary(), timed_region=clocks.summary(timed_first, timed_last),
                           window=f"{args.clock_window:.1f} s of the same substeps on a second copy of the "
                                  "loaf, one untimed substep, then the timed region")}
    if not args.no_variants:
        del sim
        line["variants"] = variants(args, rank, dist)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(scene)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def position_error(xs, xe):
    """Relative final-position error of the surrogate run: the largest particle distance between the
    two runs over the largest particle position of the exact run (positions measured from the grid
    origin, as the simulator stores them)."""
    return float((xs - xe).norm(dim=1).max() / xe.norm(dim=1).max())


def result_bytes():
    return 2 * 8


def step_roofline(particles, active_nodes, steps, seconds, per_particle=BYTES_PER_PARTICLE,
                  per_node=BYTES_PER_ACTIVE_NODE):
    """Whole-substep roofline: algorithmic bytes (per particle and per active node) moved per second
    against the HBM peak."""
    peak, kind = load_peaks()
    step_bytes = particles * per_particle + active_nodes * per_node
    achieved = step_bytes * steps / seconds / 1e9
    return {"bound": "hbm", "bytes_per_step": int(step_bytes), "bytes_per_particle": per_particle,
            "bytes_per_active_node": per_node, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": kind}


def reduce_max(value, dist):
    """The maximum of ``value`` over the ranks of the process group (``dist``, or None for one
    process): on the GPU under NCCL, on the host under gloo."""
    if not dist:
        return value
    import torch
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _timed(fn, dist, stream):
    """Device time of fn() between CUDA events on the launching stream, max over ranks."""
    import torch
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    out = fn()
    b.record(stream)
    torch.cuda.synchronize()
    return reduce_max(a.elapsed_time(b) / 1e3, dist), out


def batched(args, rank, dist, net, count=64, steps=200):
    """64 independent dough balls (particles ~ U[5k, 200k], grids from {32, 48, 64, 96}^3, oven
    ~ U[150, 220] C, prestrain ~ U[0.04, 0.1] so that they yield), advanced together under one
    captured CUDA graph (BatchedSimulators' default: bodies under 50k particles through instance
    tables, one launch per stage for all of them, larger bodies with their own launches on 8
    streams): exact return map, then the surrogate from the same initial states; also the exact
    map with every body in a table and with every body on its own launches, the default launched
    without the graph, and 128 small bodies (4-6k particles, 32-48^3) through tables against
    their own launches."""
    import torch
    from baking_b200.batch import BatchedSimulators, RestoreStates, SnapshotStates
    from baking_b200.scenes import dough_batch, make_simulator
    from baking_b200.surrogate import ReturnMapSurrogate
    world = int(os.environ.get("WORLD_SIZE", "1"))
    stream = torch.cuda.current_stream()
    bodies = dough_batch(count, seed=rank, prestrain=(0.04, 0.1))
    sims = [make_simulator(b, diagnostics="lean") for b in bodies]
    n = sum(s.particle_data.particle_count for s in sims)
    saved = SnapshotStates(sims)
    exact = BatchedSimulators(sims).capture()
    RestoreStates(sims, saved)
    t_exact, _ = _timed(lambda: exact.Advance(steps), dist, stream)
    active = sum(active_node_count(s) for s in sims)
    t_launch, _ = _timed(lambda: exact.Advance(20, graph=False), dist, stream)
    exact.CheckState()
    del exact
    RestoreStates(sims, saved)
    alt = {}
    for launch in ("streams", "table"):
        other = BatchedSimulators(sims, launch=launch).capture()
        RestoreStates(sims, saved)
        alt[launch], _ = _timed(lambda: other.Advance(steps), dist, stream)
        del other
        RestoreStates(sims, saved)
    surs = [ReturnMapSurrogate(net).attach(s) for s in sims]
    fast = BatchedSimulators(sims).capture()
    RestoreStates(sims, saved)
    for s in surs:
        s.reset_statistics()
    t_sur, _ = _timed(lambda: fast.Advance(steps), dist, stream)
    fast.CheckState()
    paths = [sum(s.statistics()[k] for s in surs) for k in ("elastic", "surrogate", "exact_yielding")]
    return {"value": world * n * steps / t_exact, "unit": UNIT, "surrogate": world * n * steps / t_sur,
            "without_graph": world * n * 20 / t_launch,
            "all_own_launches": world * n * steps / alt["streams"], "all_tables": world * n * steps / alt["table"],
            "small_bodies": small_bodies(dist, stream, world, rank),
            "instances": count, "particles": n, "steps": steps,
            "surrogate_paths": dict(zip(("elastic", "surrogate", "exact_yielding"), paths)),
            "roofline": step_roofline(n, active, steps, t_exact),
            "surrogate_roofline": step_roofline(n, active, steps, t_sur),
            "scene": "dough balls (loaf dough: Ding + gas + thermal-water), dt 5e-5, one CUDA graph per 2 substeps",
            "launch": "bodies under 50k particles: one launch per stage per instance table; larger: own launches"}


def small_bodies(dist, stream, world, rank, count=128, steps=40):
    """128 dough balls of 4-6k particles on 32^3-48^3 grids: launch-bound bodies, through instance
    tables (BatchedSimulators' default for them) against their own launches on 8 streams."""
    from baking_b200.batch import BatchedSimulators, RestoreStates, SnapshotStates
    from baking_b200.scenes import dough_batch, make_simulator
    bodies = dough_batch(count, seed=rank + 1, particles=(4000, 6000), resolutions=(32, 48), prestrain=(0.04, 0.1))
    sims = [make_simulator(b, diagnostics="lean") for b in bodies]
    n = sum(s.particle_data.particle_count for s in sims)
    saved = SnapshotStates(sims)
    out = {"instances": count, "particles": n, "steps": steps, "unit": UNIT}
    for name, launch in (("tables", "auto"), ("own_launches", "streams")):
        batch = BatchedSimulators(sims, launch=launch).capture()
        RestoreStates(sims, saved)
        t, _ = _timed(lambda: batch.Advance(steps), dist, stream)
        out[name] = world * n * steps / t
        del batch
        RestoreStates(sims, saved)
    return out


def rollout_variant(sim, dist, stream, world, scene, fb_steps=64, every=FWD_BWD_CHECKPOINT_EVERY):
    """Forward + hand-written adjoint of ``fb_steps`` substeps with a checkpoint every ``every``
    (Rollout): loss = mean squared distance of the final positions to the initial cloud scaled by
    1.2 about its centre; gradients with respect to the per-particle initial temperatures and gas
    source rates and Young's modulus."""
    import torch
    from baking_b200.physics.adjoint import Rollout
    n = sim.particle_data.particle_count
    sim.AdvanceUnchecked(2)
    st = sim.current_state
    x0 = st.particle_positions.clone()
    center = x0.mean(0)
    target = 1.2 * (x0 - center) + center
    T0 = st.transport_state.temperatures.clone().requires_grad_(True)
    rates = sim.material.production_parameter.clone().requires_grad_(True)
    E0 = torch.tensor([sim.material.material_config.young_modulus], device="cuda", requires_grad=True)

    def fwd_bwd():
        res = Rollout(sim, fb_steps, checkpoint_every=every, transport_temperatures=T0, gas_source_rates=rates,
                      young_modulus=E0)
        loss = ((res["positions"] - target) ** 2).sum(1).mean()
        loss.backward()
        return loss

    fwd_bwd()  # warm-up: first-call set-up of the reverse-mode buffers and kernels
    for t in (T0, rates, E0):
        t.grad = None
    repeats = 3  # forward + backward rollouts timed back to back (one alone varies by ~20% between runs)

    def rollouts():
        for _ in range(repeats):
            for t in (T0, rates, E0):
                t.grad = None
            fwd_bwd()

    t_fb, _ = _timed(rollouts, dist, stream)
    t_fb /= repeats
    t_f, _ = _timed(lambda: sim.AdvanceUnchecked(fb_steps), dist, stream)
    active = active_node_count(sim)
    finite = all(bool(torch.isfinite(t.grad).all()) for t in (T0, rates, E0))
    out = {"value": world * n * fb_steps / t_fb, "unit": UNIT, "forward_only": world * n * fb_steps / t_f,
           "forward_over_fwd_bwd": t_fb / t_f,
           "roofline": step_roofline(n, active, fb_steps, t_fb, bytes_per_particle_fwd_bwd(every),
                                     BYTES_PER_ACTIVE_NODE_FWD_BWD),
           "ms_per_substep": 1e3 * t_fb / fb_steps, "steps": fb_steps, "checkpoint_every": every,
           "rollouts_timed": repeats,
           "gradients": ["transport_temperatures", "gas_source_rates", "young_modulus"],
           "finite_gradients": finite, "scene": scene}
    del sim
    return out


def variants(args, rank, dist):
    """The metric's other two forms at the same particle count and grid.

    surrogate: the learned return map (committed weights) against the exact map on a loaf that yields
    from its first substep (part-baked at 318 K, isochoric elastic prestrain 0.08), both timed over
    the same substeps from the same state; the plain loaf of the headline never yields in the timed
    window, so the surrogate has nothing to replace there.
    fwd_bwd: forward + hand-written adjoint of 64 substeps with a checkpoint every 8 (Rollout) on the
    headline loaf (Ding + gas + thermal-water), loss = mean squared distance of the final positions
    to the initial cloud scaled by 1.2 about its centre, gradients with respect to the per-particle
    initial temperatures and gas source rates and Young's modulus; also on a 100k-particle dough
    sphere on a 64^3 grid."""
    import torch
    from baking_b200.scenes import box_loaf, dough_ball, make_simulator
    from baking_b200.surrogate import LoadReturnSurrogate, ReturnMapSurrogate
    world = int(os.environ.get("WORLD_SIZE", "1"))
    stream = torch.cuda.current_stream()
    out = {}
    steps = max(1, min(args.steps, 100))
    loaf = box_loaf(args.resolution, args.particles, seed=rank, initial_temperature=318.15, prestrain=0.08)
    n = loaf.particle_count
    net = LoadReturnSurrogate(ROOT / "baking_b200" / "data" / "return_surrogate_box_loaf.npz")
    results = {}
    for mode in ("exact", "surrogate"):
        sim = make_simulator(loaf, diagnostics="lean")
        sur = ReturnMapSurrogate(net).attach(sim) if mode == "surrogate" else None
        sim.AdvanceUnchecked(max(3, min(args.warmup, 10)))
        if sur:
            sur.reset_statistics()
        t, _ = _timed(lambda: sim.AdvanceUnchecked(steps), dist, stream)
        sim.CheckState()
        results[mode] = (t, sim.current_state.particle_positions.double().clone(), sur.statistics() if sur else None,
                         active_node_count(sim))
        del sim
    (te, xe, _, ae), (ts, xs, stats, asur) = results["exact"], results["surrogate"]
    x0 = torch.as_tensor(loaf.samples.particle_positions, device=xe.device)
    moved = float((xe - x0).norm(dim=1).max())
    dev = float((xs - xe).norm(dim=1).max())
    out["surrogate"] = {"value": world * n * steps / ts, "unit": UNIT, "exact_same_scene": world * n * steps / te,
                        "speedup": te / ts, "steps": steps, "paths": stats,
                        "max_position_deviation_m": dev,
                        "relative_final_position_error": position_error(xs, xe),
                        "deviation_over_max_displacement": dev / moved,
                        "roofline": step_roofline(n, asur, steps, ts),
                        "exact_roofline": step_roofline(n, ae, steps, te),
                        "scene": f"box loaf {n} particles, {args.resolution}^3, 318 K, prestrain 0.08, gas + transport"}
    del results, xe, xs
    # forward + backward
    out["fwd_bwd"] = rollout_variant(make_simulator(box_loaf(args.resolution, args.particles, seed=rank),
                                                    diagnostics="lean"), dist, stream, world,
                                     f"box loaf {n} particles, {args.resolution}^3, Ding + gas + thermal-water")
    sphere = dough_ball(64, 100_000, seed=rank, initial_temperature=298.15)
    out["fwd_bwd"]["sphere_64"] = rollout_variant(
        make_simulator(sphere, diagnostics="lean"), dist, stream, world,
        f"dough sphere {sphere.particle_count} particles, 64^3, Ding + gas + thermal-water")
    out["batched"] = batched(args, rank, dist, net)
    out["config4"] = config4_variant(args, rank, dist, stream, world, net)
    out["bake_1000"] = bake_variant(args, rank, dist, stream, world)
    out["cell_order"] = cell_order_variant(args, rank, dist, stream, world)
    return out


def config4_variant(args, rank, dist, stream, world, net, particles=4_000_000, resolution=256, steps=500):
    """The learned return map deployed at scale: a 4M-particle box loaf on a 256^3 grid for 500
    substeps, part-baked (318 K) and pre-stressed (prestrain 0.08) so that the return map yields
    everywhere, with the surrogate attached (out-of-range particles take the exact map) and the exact
    map on the same substeps from the same state; path counts and the final position deviation. The
    judge (the exact map re-run on one warp in 64 to record the network's largest log-strain error)
    checks a further 20 substeps after the timed region: inside it, its inline exact solves cost
    about a tenth of the surrogate substep."""
    import torch
    from baking_b200.scenes import box_loaf, make_simulator
    from baking_b200.surrogate import ReturnMapSurrogate
    loaf = box_loaf(resolution, particles, seed=rank, initial_temperature=318.15, prestrain=0.08)
    n = loaf.particle_count
    results = {}
    for mode in ("exact", "surrogate"):
        sim = make_simulator(loaf, diagnostics="lean")
        sur = ReturnMapSurrogate(net).attach(sim) if mode == "surrogate" else None
        sim.AdvanceUnchecked(3)
        if sur:
            sur.reset_statistics()
        t, _ = _timed(lambda: sim.AdvanceUnchecked(steps), dist, stream)
        sim.CheckState()
        stats = sur.statistics() if sur else None
        results[mode] = (t, sim.current_state.particle_positions.double().clone(), stats, active_node_count(sim))
        if sur:
            judge = ReturnMapSurrogate(net, judge_stride=64).attach(sim)
            sim.AdvanceUnchecked(20)
            stats["judge_max_log_strain_error"] = judge.statistics()["judge_max_log_strain_error"]
            stats["judged_substeps"] = 20
        del sim, sur
        torch.cuda.empty_cache()
    (te, xe, _, ae), (ts, xs, stats, asur) = results["exact"], results["surrogate"]
    x0 = torch.as_tensor(loaf.samples.particle_positions, device=xe.device)
    moved = float((xe - x0).norm(dim=1).max())
    dev = float((xs - xe).norm(dim=1).max())
    return {"value": world * n * steps / ts, "unit": UNIT, "exact": world * n * steps / te, "speedup": te / ts,
            "steps": steps, "particles": n, "resolution": resolution, "paths": stats,
            "max_position_deviation_m": dev, "relative_final_position_error": position_error(xs, xe),
            "deviation_over_max_displacement": dev / moved,
            "roofline": step_roofline(n, asur, steps, ts), "exact_roofline": step_roofline(n, ae, steps, te),
            "scene": f"box loaf {n} particles, {resolution}^3, 318 K, prestrain 0.08, gas + transport, "
                     f"{steps} substeps after 3 warm-up substeps"}


def bake_variant(args, rank, dist, stream, world, steps=1000):
    """The plain workload over its whole stated length: the headline loaf advanced 1000 substeps
    from its initial state in one timed region, with the periodic re-sort by cell (every
    SORT_INTERVAL substeps, its cost inside the region) and without it; the throughput of each
    100-substep window shows how the cost changes as the loaf settles."""
    import torch
    from baking_b200.scenes import box_loaf, make_simulator
    scene = box_loaf(args.resolution, args.particles, seed=rank)
    n = scene.particle_count
    out = {"unit": UNIT, "steps": steps, "sort_interval": SORT_INTERVAL,
           "scene": f"box loaf {n} particles, {args.resolution}^3, substeps 0-{steps} from the initial state"}
    for name, interval in (("sorted", SORT_INTERVAL), ("unsorted", 0)):
        sim = make_simulator(scene, diagnostics="lean", sort_interval=interval)
        marks = [torch.cuda.Event(enable_timing=True) for _ in range(steps // 100 + 1)]
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        marks[0].record(stream)
        for k in range(steps // 100):
            sim.AdvanceUnchecked(100)
            marks[k + 1].record(stream)
        torch.cuda.synchronize()
        sim.CheckState()
        total = reduce_max(marks[0].elapsed_time(marks[-1]) / 1e3, dist)
        out[name] = world * n * (steps // 100 * 100) / total
        out[name + "_per_100_us"] = [round(1e3 * a.elapsed_time(b) / 100, 1) for a, b in zip(marks, marks[1:])]
        del sim
        torch.cuda.empty_cache()
    out["value"] = out["sorted"]
    return out


def cell_order_variant(args, rank, dist, stream, world, steps=20):
    """The headline loaf with its particles listed in a random order, timed before and after
    MpmSimulator.SortParticles (device radix sort by stencil base, every per-particle array
    permuted in place), and the cost of the sort itself."""
    import torch
    from baking_b200.scenes import box_loaf, make_simulator, permuted
    scene = box_loaf(args.resolution, args.particles, seed=rank)
    n = scene.particle_count
    shuffled = permuted(scene, np.random.default_rng(rank).permutation(n))
    sim = make_simulator(shuffled, diagnostics="lean")
    sim.AdvanceUnchecked(3)
    t_shuffled, _ = _timed(lambda: sim.AdvanceUnchecked(steps), dist, stream)
    sim.CellOrder()  # loads the sort kernels
    t_keys, _ = _timed(sim.CellOrder, dist, stream)
    torch.cuda.synchronize()
    wall = time.perf_counter()
    t_first, _ = _timed(sim.SortParticles, dist, stream)  # includes loading the permutation kernels
    wall = reduce_max(time.perf_counter() - wall, dist)
    sim.AdvanceUnchecked(3)
    t_sort, _ = _timed(sim.SortParticles, dist, stream)  # the same work again, order already near sorted
    t_sorted, _ = _timed(lambda: sim.AdvanceUnchecked(steps), dist, stream)
    sim.CheckState()
    return {"unit": UNIT, "shuffled": world * n * steps / t_shuffled, "sorted": world * n * steps / t_sorted,
            "speedup": t_shuffled / t_sorted, "cell_order_ms": 1e3 * t_keys, "sort_particles_ms": 1e3 * t_sort,
            "sort_particles_first_call_ms": 1e3 * t_first, "sort_particles_first_call_wall_ms": 1e3 * wall,
            "steps": steps,
            "scene": f"box loaf {n} particles, {args.resolution}^3, particles in random order"}


if __name__ == "__main__":
    main()
