#!/usr/bin/env python3
"""Benchmark of the explicit step on the 20^3 BCC elastoplastic impact lattice.

Workload (one "step" = one explicit time step over the whole lattice):
  20x20x20 BCC unit cells of 10 mm, 64,000 corner-to-centre struts at 2
  elements each (128,000 elements, 81,261 nodes), strut radius
  0.5 mm x (1 + U[-0.05, 0.05]) per strut (seed 0), aluminium E=70 GPa,
  nu=0.33, rho=2700, yield 300 MPa with 1 GPa linear isotropic hardening
  (stress-resultant yield surface, 2 Gauss points), bottom face fixed, top
  face driven down at 10 m/s, dt = 5e-8 s.  Synthetic, seeded data.

Headline ``value``: element-steps/s of the mixed-precision engine (FP32
element force and return map, FP64 state) with the L2 cache flushed before
every timed step (the lattice's working set is smaller than L2), timed with
CUDA events around each step's launch on the engine's stream.  The state
error of the mixed path against the plain FP64 path over the same steps is
reported beside it (``mixed_vs_fp64``).

``--impl reference`` times the CPU restatement of the reference algorithm
(the oracle; the reference binary cannot be built) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "element-steps/s at ≤1e-5 rel. state error: mixed vs FP64; adjoint/forward time"
UNIT = "element-steps/s"
# canonical algorithmic bytes per node / per element and step (mixed precision,
# elastoplastic, 2 Gauss points; plain FP64: 360 / 864)
BYTES_NODE = {"mixed": 288, "fp64": 360}
BYTES_ELEM = {"mixed": 500, "fp64": 864}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2000)
    p.add_argument("--warmup", type=int, default=20)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--cells", type=int, default=20)
    p.add_argument("--err-steps", type=int, default=20000)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--workload", default="bcc20", choices=["bcc20", "batch256", "fibre20k", "rod32", "adjoint8"],
                   help="bcc20: the 20^3 BCC impact (default line); batch256: 256 uneven lattices; "
                        "fibre20k: 20 000-rod fibre network with rod--rod contact and plates; "
                        "rod32: the 32-element clamped rod (FP64); adjoint8: gradient of the 8^3 BCC impact")
    p.add_argument("--rods", type=int, default=20000, help="rods of --workload fibre20k")
    p.add_argument("--no-fd", action="store_true", help="--workload adjoint8 without the finite-difference checks")
    p.add_argument("--block", type=int, default=100, help="steps per launch for --workload batch256")
    p.add_argument("--profile", action="store_true",
                   help="for ncu captures: --warmup launches of --steps steps each, then one more, and nothing "
                        "else (mixed precision, or FP64 with --fp64); prints no JSON line")
    p.add_argument("--fp64", action="store_true", help="with --profile: the plain FP64 path")
    p.add_argument("--exec-mode", type=int, default=0, help="with --profile: 0 persistent, 1 two launches per step")
    return p.parse_args()


def workload(cells):
    from dynlattice_b200 import lattices
    spec = lattices.lattice_impact("bcc", n=cells, cell=10e-3, elems_per_strut=2, radius=0.5e-3,
                                   radius_jitter=0.05, seed=0, velocity=10.0, dt=5e-8, plastic=True,
                                   n_gauss=2)
    return spec


def peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed region.

    A thread polls NVML every millisecond from __enter__ to __exit__, so even a
    timed region of a few milliseconds gets samples; if the region ends before
    the first poll, one sample is taken at its end (clocks lag the load by far
    more than that).  Without NVML the sampler falls back to `nvidia-smi -lms`."""

    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int, period_s: float = 1e-3):
        self.index = index
        self.period = period_s
        self.samples = []            # (sm_mhz, sm_max_mhz, set of reasons)
        self.proc = None
        self.t = None
        self.nvml = None
        self.stop = threading.Event()

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            idx = torch.cuda._get_nvml_device_index(self.index)
        except Exception:
            idx = self.index
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(idx)

    def _nvml_sample(self):
        nv, h = self.nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        flags = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                 nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
        self.samples.append((float(sm), float(mx), {n for n, f in zip(self.NAMES, flags) if bits & f}))

    def _poll(self):
        while not self.stop.is_set():
            try:
                self._nvml_sample()
            except Exception:
                return
            self.stop.wait(self.period)

    def __enter__(self):
        try:
            self.nvml = self._handle()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm, mx = float(parts[0]), float(parts[1])
            except ValueError:
                continue
            self.samples.append((sm, mx, {n for n, v in zip(self.NAMES, parts[3:7])
                                          if v.lower().startswith("active")}))

    def __exit__(self, *a):
        self.stop.set()
        if self.nvml is not None:
            self.t.join(timeout=5)
            if not self.samples:
                try:
                    self._nvml_sample()
                except Exception:
                    pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [x[0] for x in self.samples]
        reasons = set().union(*(x[2] for x in self.samples))
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(x[1] for x in self.samples)),
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self.nvml is not None else "nvidia-smi"}


def traffic_per_step():
    """DRAM bytes per step of the persistent kernel from the committed ncu summary."""
    f = ROOT / "profiles" / "traffic.json"
    if f.exists():
        try:
            return float(json.loads(f.read_text())["dram_bytes_per_step"])
        except Exception:
            return None
    return None


def cpu_baseline_run(spec, seconds, threads, steps_cap=None):
    """Time the oracle (CPU restatement, FP64) on this host; returns (value, steps, secs)."""
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_ffi import Oracle
    o = Oracle(spec, threads=threads)
    o.run(2)  # warm-up
    t0 = time.perf_counter()
    o.run(1)
    one = max(time.perf_counter() - t0, 1e-6)
    n = max(1, int(seconds / one))
    if steps_cap is not None:
        n = max(1, min(n, steps_cap))
    t0 = time.perf_counter()
    o.run(n)
    dt = time.perf_counter() - t0
    o.close()
    return spec.n_elems * n / dt, n, dt


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload == "fibre20k":
        return run_reference_fibre(args)
    spec = workload(args.cells)
    threads = os.cpu_count() or 1
    # bounded sample: warm-up and timed steps capped so the run ends within minutes
    value, n, dt = cpu_baseline_run(spec, seconds=max(10.0, min(90.0, args.cpu_seconds * 4)), threads=threads,
                                    steps_cap=args.steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / n * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"bcc{args.cells}^3 elastoplastic impact ({spec.n_elems} elements, "
                               f"{spec.n_nodes} nodes), CPU restatement of the reference (FP64)",
                   "parallelism": "openmp"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{n} explicit steps of the full lattice after 3 warm-up steps "
                                   f"(reference binary unbuildable: JEM/JIVE absent)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def measure_batch(args):
    """256 independent lattices of uneven size (BCC/SC/octet, n^3 cells with
    n ~ U{4..12}, strut radius U(0.3, 0.7) mm, impact 1-50 m/s log-uniform, dt
    per lattice from its critical step) in one launch per block of 100 steps;
    L2 flushed before every block.  Reports lattices*steps/s and p50/p99 per block."""
    import torch
    from dynlattice_b200 import lattices
    from dynlattice_b200.abi import DL_MIXED
    from dynlattice_b200.engine import Batch
    from dynlattice_b200.shard import max_over_ranks, shard_for_rank
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    all_specs = lattices.batch_lattices(256, seed=0)
    E = sum(s.n_elems for s in all_specs)
    N = sum(s.n_nodes for s in all_specs)
    # lattices shared out by element count; no collective in the data path
    _, specs = shard_for_rank(all_specs, rank, world)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    b = Batch(specs, DL_MIXED, stream=stream.cuda_stream)
    tune = b.autotune(args.block)   # launch shape for this batch (engine autotuner)
    nblocks = max(3, args.steps // args.block)
    for _ in range(max(1, args.warmup // args.block)):
        b.run(args.block)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nblocks)]
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for a, e in ev:
            flush.zero_()
            a.record(stream)
            b.run(args.block)
            e.record(stream)
        torch.cuda.synchronize()
    b.synchronize()
    t = np.array([a.elapsed_time(e) / 1e3 for a, e in ev])
    steps = nblocks * args.block
    t_total = max_over_ranks(float(t.sum()))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({
                "metric": "lattices*steps/s (batched uneven lattices)", "value": 256 * steps / t_total,
                "unit": "lattice-steps/s", "element_steps_per_s": E * steps / t_total, "n_gpus": world,
                "steps": steps, "warmup": args.warmup, "ms_per_step": t_total / steps * 1e3,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32/f64",
                "data": "synthetic", "config": {"workload": f"256 lattices sharded by element count over "
                                                            f"{world} GPUs, {E} elements, {N} nodes",
                                                "block": args.block, "l2": "flushed before every block"},
                "gpu_launches": nblocks, "clocks": clk.summary()}), flush=True)
        return None
    # the same blocks replayed from a CUDA graph (exec mode 2), and the autotuner's pick
    bg = Batch(specs, DL_MIXED, stream=stream.cuda_stream)
    bg.autotune(args.block)
    bg.set_exec_mode(2)
    bg.run(args.block)
    torch.cuda.synchronize()
    evg = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nblocks)]
    for a, e in evg:
        flush.zero_()
        a.record(stream)
        bg.run(args.block)
        e.record(stream)
    torch.cuda.synchronize()
    bg.synchronize()
    tg = np.array([a.elapsed_time(e) / 1e3 for a, e in evg])
    del bg
    peak, peak_kind = peaks()
    bytes_step = N * BYTES_NODE["mixed"] + E * BYTES_ELEM["mixed"]
    achieved = bytes_step * args.block / t.mean() / 1e9
    line = {"metric": "lattices*steps/s (batched uneven lattices)", "value": 256 * steps / t.sum(),
            "unit": "lattice-steps/s", "element_steps_per_s": E * steps / t.sum(), "n_gpus": 1,
            "steps": steps, "warmup": args.warmup, "ms_per_step": t.sum() / steps * 1e3,
            "block_ms_p50": float(np.percentile(t, 50) * 1e3), "block_ms_p99": float(np.percentile(t, 99) * 1e3),
            "higher_is_better": True, "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": f"256 lattices (bcc/sc/octet, n^3 cells n in 4..12), {E} elements, {N} nodes",
                       "block": args.block, "l2": "flushed before every block"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "bytes_per_step": bytes_step, "peak_kind": peak_kind},
            "gpu_launches": nblocks, "clocks": clk.summary(), "jit": b.info()["jit"],
            "graph": {"block_ms_p50": float(np.percentile(tg, 50) * 1e3),
                      "block_ms_p99": float(np.percentile(tg, 99) * 1e3),
                      "note": "exec mode 2: each block one CUDA graph replay"},
            "autotune": {"mode": tune[0], "threads_per_block": tune[1], "ms_per_block": tune[2]}}
    return line


# elastic rods drop the 224 B of history per element (2 Gauss points) of the
# canonical elastoplastic figure; a candidate pair reads its 8-byte index pair
BYTES_ELEM_ELASTIC = BYTES_ELEM["mixed"] - 224
BYTES_PAIR = 8


def fibre_spec(args):
    from dynlattice_b200 import lattices
    return lattices.fibre_network(n_rods=args.rods, seed=0, plate_velocity=5.0, penalty=1e4, dt=1e-8)


def fibre_desc(spec):
    return (f"{spec.n_elems // 4} rods x 4 elements ({spec.n_elems} elements, {spec.n_nodes} nodes), L=10 mm, "
            f"r=0.1 mm, E=3 GPa, rod-rod penalty contact 1e4 N/m, plates at 5 m/s, dt=1e-8 s")


def run_reference_fibre(args):
    spec = fibre_spec(args)
    threads = os.cpu_count() or 1
    value, n, dt = cpu_baseline_run(spec, seconds=max(10.0, min(60.0, args.cpu_seconds * 2)), threads=threads,
                                    steps_cap=args.steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / n * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "fibre network: " + fibre_desc(spec) +
                               "; CPU restatement of the reference (FP64, O(R^2) contact search every step)",
                   "parallelism": "openmp"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{n} explicit steps of the full network after 3 warm-up steps"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def measure_fibre(args):
    """20 000 straight rods (4 elements each) compressed between two rigid
    plates with rod--rod penalty contact; mixed precision.  Timed in blocks of
    --block steps with the L2 flushed before every block; the candidate-list
    rebuilds that fall inside a block are part of its time."""
    import torch
    from dynlattice_b200.abi import DL_MIXED
    from dynlattice_b200.engine import Lattice
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    spec = fibre_spec(args)
    E, N = spec.n_elems, spec.n_nodes
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    eng = Lattice(spec, DL_MIXED, stream=stream.cuda_stream)
    eng.run(max(3, args.warmup))
    torch.cuda.synchronize()
    nblocks = max(3, args.steps // args.block)
    _, builds0 = eng.contact_stats()
    launches0 = eng.launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nblocks)]
    cand = []
    with ClockSampler(local) as clk:
        for a, b in ev:
            flush.zero_()
            a.record(stream)
            eng.run(args.block)
            b.record(stream)
            cand.append(eng.contact_stats()[0])
        torch.cuda.synchronize()
    eng.synchronize()
    t = np.array([a.elapsed_time(b) / 1e3 for a, b in ev])
    steps = nblocks * args.block
    n_cand, builds1 = eng.contact_stats()
    launches = eng.launch_count() - launches0
    closed, _ = eng.contact_pairs()
    energies = eng.energies()
    reaction = eng.plate_reaction()
    # end to end through the C ABI: state pushed from pinned host memory before
    # every block (which also forces a candidate-list rebuild), energies read
    # back after it, state pulled back at the end
    u0 = torch.zeros((N, 3), dtype=torch.float64).pin_memory()
    th0 = torch.zeros((N, 3), dtype=torch.float64).pin_memory()
    v0 = torch.zeros((N, 6), dtype=torch.float64).pin_memory()
    e2e_eng = Lattice(spec, DL_MIXED, stream=stream.cuda_stream)
    e2e_blocks = max(2, min(nblocks, 10))
    for _ in range(3):  # warm-up of the same calls (first launches of each kernel load it)
        e2e_eng.set_state_ptrs(u0.data_ptr(), th0.data_ptr(), v0.data_ptr())
        e2e_eng.run(args.block)
        e2e_eng.energies()
    e2e_eng.get_state_ptrs(u0.data_ptr(), th0.data_ptr(), v0.data_ptr())
    u0.zero_(); th0.zero_(); v0.zero_()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_blocks):
        e2e_eng.set_state_ptrs(u0.data_ptr(), th0.data_ptr(), v0.data_ptr())
        e2e_eng.run(args.block)
        e2e_eng.energies()
    e2e_eng.get_state_ptrs(u0.data_ptr(), th0.data_ptr(), v0.data_ptr())
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t0
    del e2e_eng
    state_bytes = N * 12 * 8
    peak, peak_kind = peaks()
    mean_cand = float(np.mean(cand))
    bytes_step = N * BYTES_NODE["mixed"] + E * BYTES_ELEM_ELASTIC + mean_cand * BYTES_PAIR
    achieved = bytes_step * steps / t.sum() / 1e9
    line = {
        "metric": METRIC, "value": E * steps / t.sum(), "unit": UNIT, "n_gpus": 1, "steps": steps,
        "warmup": args.warmup, "ms_per_step": t.sum() / steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
        "config": {"workload": "fibre network: " + fibre_desc(spec), "block": args.block,
                   "l2": "flushed (256 MiB write) before every block"},
        "contact": {"candidates_mean": mean_cand, "list_builds": builds1 - builds0,
                    "closed_pairs_last_step": int(closed.shape[0]), "contact_energy": energies["contact"],
                    "plate_reaction_z": [float(reaction[0, 2]), float(reaction[1, 2])]},
        "block_ms_p50": float(np.percentile(t, 50) * 1e3), "block_ms_p99": float(np.percentile(t, 99) * 1e3),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "bytes_per_step": bytes_step, "peak_kind": peak_kind},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "e2e": {"value": E * e2e_blocks * args.block / t_e2e, "unit": UNIT,
                "h2d_bytes_per_step": state_bytes / args.block, "d2h_bytes_per_step": 40 + state_bytes / (
                    e2e_blocks * args.block),
                "protocol": f"{e2e_blocks} x (dl_set_state from pinned host, dl_run({args.block}), "
                            f"dl_get_energies), dl_get_state"},
    }
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cv, cn, cdt = cpu_baseline_run(spec, args.cpu_seconds, threads)
        line["cpu_baseline"] = {"value": cv, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{cn} explicit steps of the full network (FP64 oracle, reference "
                                          f"O(R^2) contact search every step), {cdt:.1f} s"}
    return line


def measure_rod(args):
    """32-element clamped elastic rod, tip load ramped over 500 steps, dt 2e-6,
    plain FP64 (launch/latency bound: the whole model is 18 KB).  Timed as
    blocks of --block steps, one persistent launch each, L2 flushed before
    every block; the 5000-step horizon of the workload is one run of 50 blocks."""
    import torch
    from dynlattice_b200 import lattices
    from dynlattice_b200.abi import DL_PLAIN_FP64
    from dynlattice_b200.engine import Lattice
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    spec = lattices.straight_rod()
    E, N = spec.n_elems, spec.n_nodes
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    eng = Lattice(spec, DL_PLAIN_FP64, stream=stream.cuda_stream)
    tip = spec.groups["free"]
    eng.set_sampling(10, tip, capacity=(args.steps + args.warmup) // 10 + 2)
    eng.run(max(3, args.warmup))
    torch.cuda.synchronize()
    nblocks = max(3, args.steps // args.block)
    launches0 = eng.launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nblocks)]
    with ClockSampler(local) as clk:
        for a, b in ev:
            flush.zero_()
            a.record(stream)
            eng.run(args.block)
            b.record(stream)
        torch.cuda.synchronize()
    eng.synchronize()
    launches = eng.launch_count() - launches0
    t = np.array([a.elapsed_time(b) / 1e3 for a, b in ev])
    steps = nblocks * args.block
    # end to end: a fresh rod from pinned host state, the 5000-step horizon in
    # blocks with the tip samples read back after each block
    u0 = torch.zeros((N, 3), dtype=torch.float64).pin_memory()
    th0 = torch.zeros((N, 3), dtype=torch.float64).pin_memory()
    v0 = torch.zeros((N, 6), dtype=torch.float64).pin_memory()
    warm = Lattice(spec, DL_PLAIN_FP64, stream=stream.cuda_stream)  # warm-up of the same calls
    warm.set_sampling(10, tip, capacity=3 * args.block // 10 + 2)
    for _ in range(3):
        warm.set_state_ptrs(u0.data_ptr(), th0.data_ptr(), v0.data_ptr())
        warm.run(args.block)
    warm.samples()
    del warm
    e2e_eng = Lattice(spec, DL_PLAIN_FP64, stream=stream.cuda_stream)
    e2e_eng.set_sampling(10, tip, capacity=5000 // 10 + 2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_eng.set_state_ptrs(u0.data_ptr(), th0.data_ptr(), v0.data_ptr())
    for _ in range(5000 // args.block):
        e2e_eng.run(args.block)
    steps_s, rows, en = e2e_eng.samples()
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t0
    peak, peak_kind = peaks()
    bytes_step = N * BYTES_NODE["fp64"] + E * (BYTES_ELEM["fp64"] - 2 * 224)
    achieved = bytes_step * steps / t.sum() / 1e9
    line = {
        "metric": METRIC, "value": E * steps / t.sum(), "unit": UNIT, "n_gpus": 1, "steps": steps,
        "warmup": args.warmup, "ms_per_step": t.sum() / steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "straight elastic rod: 32 elements, 33 nodes, clamped, tip load ramp, dt=2e-6 s, "
                               "plain FP64, tip sampled every 10 steps",
                   "block": args.block, "l2": "flushed (256 MiB write) before every block"},
        "roofline": {"bound": "latency", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "bytes_per_step": bytes_step,
                     "peak_kind": peak_kind,
                     "note": "18 KB model: one block of 256 threads, grid-barrier latency per phase"},
        "gpu_launches": launches, "clocks": clk.summary(),
        "e2e": {"value": E * 5000 / t_e2e, "unit": UNIT,
                "h2d_bytes_per_step": N * 12 * 8 / 5000,
                "d2h_bytes_per_step": int(steps_s.size) * (8 + 12 * 8 + 40) / 5000,
                "protocol": f"dl_set_state from pinned host, 5000 steps in blocks of {args.block}, "
                            "tip samples and energies read back"},
    }
    if not args.no_cpu_baseline:
        cv, cn, cdt = cpu_baseline_run(spec, min(args.cpu_seconds, 10.0), 1, steps_cap=200000)
        line["cpu_baseline"] = {"value": cv, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": f"{cn} explicit steps (FP64 oracle, 1 thread), {cdt:.1f} s"}
    return line


def run_batch(args):
    line = measure_batch(args)
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def run_fibre(args):
    print(json.dumps(measure_fibre(args)), flush=True)
    return 0


def run_rod(args):
    print(json.dumps(measure_rod(args)), flush=True)
    return 0


def other_workloads():
    """Short runs of the other configurations for the default line: the
    32-element rod (its whole 5000-step horizon), the 20 000-rod fibre
    network (10 blocks of 100 steps) and the 256-lattice batch (3 blocks of
    100 steps); no CPU baselines here (each has its own --workload line)."""
    import argparse as ap
    out = {}
    a = ap.Namespace(steps=5000, warmup=100, block=100, no_cpu_baseline=True, cpu_seconds=0.0, rods=20000)
    r = measure_rod(a)
    out["rod32"] = {"us_per_step": r["ms_per_step"] * 1e3, "value": r["value"], "unit": r["unit"],
                    "e2e_us_per_step": 1e9 / r["e2e"]["value"] * 32 / 1e3 if r["e2e"]["value"] else None,
                    "config": r["config"]["workload"], "l2": r["config"]["l2"]}
    a = ap.Namespace(steps=1000, warmup=100, block=100, no_cpu_baseline=True, cpu_seconds=0.0, rods=20000)
    f = measure_fibre(a)
    out["fibre20k"] = {"value": f["value"], "unit": f["unit"], "us_per_step": f["ms_per_step"] * 1e3,
                       "roofline_frac": f["roofline"]["frac"], "contact": f["contact"],
                       "e2e": f["e2e"]["value"], "config": f["config"]["workload"], "l2": f["config"]["l2"]}
    a = ap.Namespace(steps=300, warmup=100, block=100)
    b = measure_batch(a)
    out["batch256"] = {"value": b["value"], "unit": b["unit"], "element_steps_per_s": b["element_steps_per_s"],
                       "block_ms_p50": b["block_ms_p50"], "block_ms_p99": b["block_ms_p99"],
                       "roofline_frac": b["roofline"]["frac"], "graph_block_ms_p50": b["graph"]["block_ms_p50"],
                       "config": b["config"]["workload"], "l2": b["config"]["l2"]}
    return out


def adjoint_case():
    """8^3 BCC elastoplastic impact at 20 m/s (4096 struts, 8192 elements), 2000
    steps at dt 5e-8; J = E_diss(T) - 0.1 max_k R_top(k) w.r.t. the strut radii
    (0.5 mm +- 5 %)."""
    from dynlattice_b200 import lattices
    return lattices.lattice_impact("bcc", n=8, cell=10e-3, elems_per_strut=2, radius=0.5e-3, radius_jitter=0.05,
                                   seed=0, velocity=20.0, dt=5e-8, plastic=True, n_gauss=2)


def measure_adjoint(steps=2000, K=100, n_dirs=16, fd="full"):
    """Forward time, adjoint time (checkpointed forward + recomputation +
    reverse sweep) and the finite-difference check of the mixed-precision
    gradient against the FP64 path along n_dirs seeded directions."""
    import copy

    import torch
    from dynlattice_b200.abi import DL_MIXED, DL_PLAIN_FP64
    from dynlattice_b200.engine import Lattice
    spec = adjoint_case()
    r0 = spec.strut_radius.copy()
    top = spec.groups["top"]

    def with_r(r):
        s2 = copy.copy(spec)
        s2.elem_radius = np.repeat(r, 2)
        return s2

    stream = torch.cuda.current_stream()
    ev = lambda: torch.cuda.Event(enable_timing=True)
    # warm-up (runtime compilation of both kernel sets)
    w = Lattice(with_r(r0), DL_MIXED, stream=stream.cuda_stream)
    w.adjoint_radius(200, K, elem_param=spec.elem_rod, react_nodes=top, react_dof=2, react_weight=-0.1)
    w.synchronize()
    del w
    a, b = ev(), ev()
    t_fwds = []
    for _ in range(3):  # median of 3, as the gradient times below
        fw = Lattice(with_r(r0), DL_MIXED, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        a.record(stream)
        fw.run(steps)
        b.record(stream)
        torch.cuda.synchronize()
        t_fwds.append(a.elapsed_time(b) / 1e3)
        fw.synchronize()
        del fw
    t_fwd = float(np.median(t_fwds))
    def timed_adjoint(budget):
        ad = Lattice(with_r(r0), DL_MIXED, stream=stream.cuda_stream)
        ad.set_tape_budget(budget)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        a.record(stream)
        J, g = ad.adjoint_radius(steps, K, elem_param=spec.elem_rod, react_nodes=top, react_dof=2,
                                 react_weight=-0.1)
        b.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        ad.synchronize()
        del ad
        return J, g, a.elapsed_time(b) / 1e3, wall

    # first full-length gradient of the process: maps the engine's retained
    # tape pool (about 3 GB for the whole-run tape); later gradients, each
    # on a new handle as an optimisation loop over radii makes them, reuse it
    _, _, t_first, _ = timed_adjoint(-1)
    # each mode timed three times, the median reported (single gradients of
    # this size vary by up to a quarter from box to box)
    # checkpoints every K steps, every segment recomputed (the workload's memory plan)
    runs = [timed_adjoint(0) for _ in range(3)]
    J, g = runs[0][0], runs[0][1]
    t_adj = float(np.median([r[2] for r in runs]))
    t_adj_wall = float(np.median([r[3] for r in runs]))
    # the whole state tape kept in HBM (2000 steps of this lattice: about 3 GB)
    runs_full = [timed_adjoint(-1) for _ in range(3)]
    g_full = runs_full[0][1]
    t_full = float(np.median([r[2] for r in runs_full]))
    out = {"workload": "8^3 BCC elastoplastic impact at 20 m/s, 8192 elements, 4096 strut radii, 2000 steps "
                       "dt=5e-8, checkpoint every 100 steps, mixed precision (FP32 forces, FP64 state/adjoint); "
                       "forward and gradient times: median of 3",
           "J": J, "forward_s": t_fwd, "adjoint_s": t_adj, "adjoint_wall_s": t_adj_wall,
           "adjoint_over_forward": t_adj / t_fwd, "grad_norm": float(np.linalg.norm(g)),
           "full_tape": {"adjoint_s": t_full, "adjoint_over_forward": t_full / t_fwd,
                         "first_call_s": t_first,
                         "grad_rel_diff_vs_checkpointed": float(np.abs(g_full - g).max() / np.abs(g).max())}}
    if fd:
        out["fd_check"] = fd_checks(spec, r0, g, steps, K, n_dirs, tight=(fd == "full"))
    return out


def fd_checks(spec, r0, g_mixed, steps, K, n_dirs, tight=False):
    """Central differences of J (FP64 forward, relative step 1e-6 of the
    mean radius, n_dirs seeded directions) against the adjoint gradients.

    J is piecewise smooth: a Gauss point that starts or stops yielding, a
    change of the cutting plane's iteration count or of the peak step
    switches branches, and a difference quotient that straddles a switch
    measures a secant across it.  The adjoint differentiates the branch its
    forward run takes; "branch_imposed" takes the differences along that
    branch (the FP64 run's recorded iteration counts and peak step imposed on
    the perturbed runs), "free" lets every perturbed run take its own."""
    import copy

    from dynlattice_b200.abi import DL_PLAIN_FP64
    from dynlattice_b200.engine import Lattice
    top = spec.groups["top"]

    def with_r(r):
        s2 = copy.copy(spec)
        s2.elem_radius = np.repeat(r, 2)
        return s2

    def objective(r, tape=None):
        L = Lattice(with_r(r), DL_PLAIN_FP64)
        if tape is not None:
            L.set_branch_mode(2)
            L.set_branch_tape(*tape)
        Jx, _ = L.adjoint_radius(steps, 0, elem_param=spec.elem_rod, react_nodes=top, react_dof=2,
                                 react_weight=-0.1)
        L.close()
        return Jx

    L64 = Lattice(with_r(r0), DL_PLAIN_FP64)
    L64.set_branch_mode(1)
    J64, g64 = L64.adjoint_radius(steps, K, elem_param=spec.elem_rod, react_nodes=top, react_dof=2,
                                  react_weight=-0.1)
    tape = L64.branch_tape()
    L64.close()
    rng = np.random.default_rng(0)
    dirs = [rng.normal(size=r0.size) for _ in range(n_dirs)]

    def check(tape_or_none, h_rel=1e-6):
        h = h_rel * np.abs(r0).mean()
        e64, emx = [], []
        for d in dirs:
            fdv = (objective(r0 + h * d, tape_or_none) - objective(r0 - h * d, tape_or_none)) / (2 * h)
            e64.append(abs(g64 @ d - fdv) / abs(fdv))
            emx.append(abs(g_mixed @ d - fdv) / abs(fdv))
        summ = lambda e: {"max_rel_err": float(max(e)), "median_rel_err": float(np.median(e))}
        return {"fp64_adjoint": summ(e64), "mixed_adjoint": summ(emx)}

    res = {"directions": n_dirs, "h_rel": 1e-6, "reference": "FP64 central differences of J",
           "yielding_gauss_point_steps": int((tape[0] > 0).sum()), "peak_step": int(tape[1]),
           "branch_imposed": check(tape), "free": check(None),
           "mixed_vs_fp64_adjoint_rel": float(np.abs(g_mixed - g64).max() / np.abs(g64).max())}
    res["fd_max_rel"] = res["branch_imposed"]["fp64_adjoint"]["max_rel_err"]
    if tight:
        # free differences converge to the adjoint as the step shrinks (the
        # branch switches inside the step's interval become rarer): h = 1e-7
        res["free_h1e-7"] = check(None, 1e-7)["fp64_adjoint"]
    return res


def run_adjoint(args):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    spec = adjoint_case()
    E = spec.n_elems
    with ClockSampler(local) as clk:
        res = measure_adjoint(steps=2000, fd=False if args.no_fd else "full")
    peak, peak_kind = peaks()
    line = {
        "metric": METRIC, "value": E * 2000 / res["adjoint_s"], "unit": "element-steps/s (gradient)",
        "n_gpus": 1, "steps": 2000, "warmup": 200, "ms_per_step": res["adjoint_s"] / 2000 * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
        "config": {"workload": res["workload"], "l2": "working set 6 MB, L2 resident (not flushed)"},
        "adjoint_over_forward": res["full_tape"]["adjoint_over_forward"],
        "checkpointed_over_forward": res["adjoint_over_forward"], "adjoint": res,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


def run_profile(args):
    """Launches of the default workload for an ncu capture."""
    import torch
    from dynlattice_b200.abi import DL_MIXED, DL_PLAIN_FP64
    from dynlattice_b200.engine import Lattice
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    eng = Lattice(workload(args.cells), DL_PLAIN_FP64 if args.fp64 else DL_MIXED)
    eng.set_exec_mode(args.exec_mode)
    for _ in range(args.warmup + 1):
        eng.run(args.steps)
    eng.synchronize()
    return 0


def main():
    args = parse()
    if args.profile:
        return run_profile(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch256":
        return run_batch(args)
    if args.workload == "fibre20k":
        return run_fibre(args)
    if args.workload == "rod32":
        return run_rod(args)
    if args.workload == "adjoint8":
        return run_adjoint(args)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from dynlattice_b200.abi import DL_MIXED, DL_PLAIN_FP64
    from dynlattice_b200.engine import Lattice

    spec = workload(args.cells)
    E, N = spec.n_elems, spec.n_nodes
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed_steps(eng, k, w):
        """w untimed + k timed single-step launches, L2 flushed before each."""
        for _ in range(w):
            flush.zero_()
            eng.run(1)
        barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        for a, b in ev:
            flush.zero_()
            a.record(stream)
            eng.run(1)
            b.record(stream)
        barrier()
        return sum(a.elapsed_time(b) for a, b in ev) / 1e3  # seconds

    # ---- headline: mixed precision, L2 flushed before every step
    mixed = Lattice(spec, DL_MIXED, stream=stream.cuda_stream)
    launches0 = mixed.launch_count()
    with ClockSampler(local) as clk:
        t_mixed = timed_steps(mixed, args.steps, args.warmup)
    step_launches = (mixed.launch_count() - launches0) * args.steps // (args.steps + args.warmup)
    mixed.synchronize()
    t_max = t_mixed
    if dist is not None:
        tt = torch.tensor([t_mixed], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    value = world * E * args.steps / t_max
    ms_per_step = t_max / args.steps * 1e3

    # ---- steady state: one persistent launch over many steps (L2-resident lattice)
    steady = Lattice(spec, DL_MIXED, stream=stream.cuda_stream)
    steady.run(args.warmup)
    barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    steady.run(args.steps)
    b.record(stream)
    barrier()
    t_steady = a.elapsed_time(b) / 1e3
    # ---- blocks of 100 steps, one launch each, L2 flushed before every block
    # (how a 20 000-step run of this lattice executes)
    nblk = 5
    evb = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nblk)]
    for a2, b2 in evb:
        flush.zero_()
        a2.record(stream)
        steady.run(100)
        b2.record(stream)
    barrier()
    t_blocks = sum(a2.elapsed_time(b2) for a2, b2 in evb) / 1e3
    steady.synchronize()
    del steady

    # ---- plain FP64 path, same protocol
    k64 = max(3, args.steps // 4)
    plain = Lattice(spec, DL_PLAIN_FP64, stream=stream.cuda_stream)
    t_plain = timed_steps(plain, k64, max(3, args.warmup // 4))
    plain.synchronize()
    del plain

    # ---- state error of the mixed path against FP64 over err_steps steps
    ref = Lattice(spec, DL_PLAIN_FP64, stream=stream.cuda_stream)
    mix = Lattice(spec, DL_MIXED, stream=stream.cuda_stream)
    ref.run(args.err_steps)
    mix.run(args.err_steps)
    ur, tr, vr = ref.state()
    um, tm, vm = mix.state()
    er = ref.energies()
    em = mix.energies()
    ref.synchronize()
    mix.synchronize()
    dmax = np.abs(ur).max()
    from scipy.spatial.transform import Rotation as Rot
    ang = (Rot.from_rotvec(tr).inv() * Rot.from_rotvec(tm)).magnitude()
    err = {
        "steps": args.err_steps,
        "disp_rel": float(np.abs(um - ur).max() / dmax),
        "rot_geodesic_rel": float(ang.max() / max(np.abs(tr).max(), 1e-300)),
        "E_kin_rel": abs(em["kinetic"] - er["kinetic"]) / abs(er["kinetic"]),
        "E_pot_rel": abs(em["potential"] - er["potential"]) / abs(er["potential"]),
        "E_diss_rel": abs(em["dissipated"] - er["dissipated"]) / max(abs(er["dissipated"]), 1e-300),
    }
    del ref, mix

    # ---- end to end through the C ABI: state from pinned host memory, one
    # dl_run(1) + energy read-back per step, state back to pinned host memory
    e2e_eng = Lattice(spec, DL_MIXED, stream=stream.cuda_stream)
    u0 = torch.zeros((N, 3), dtype=torch.float64).pin_memory()
    th0 = torch.zeros((N, 3), dtype=torch.float64).pin_memory()
    v_init = np.zeros((N, 6))
    v_init[spec.groups["top"], 2] = -10.0
    v0 = torch.from_numpy(v_init).pin_memory()
    uo = torch.empty((N, 3), dtype=torch.float64).pin_memory()
    tho = torch.empty((N, 3), dtype=torch.float64).pin_memory()
    vo = torch.empty((N, 6), dtype=torch.float64).pin_memory()
    # a fixed horizon of 500 steps, whatever --steps is: the state upload and
    # download are paid once per 500 steps
    e2e_steps = 500
    for _ in range(3):  # warm-up of the same calls (first launches of each kernel load it)
        e2e_eng.set_state_ptrs(u0.data_ptr(), th0.data_ptr(), v0.data_ptr())
        e2e_eng.run(1)
        e2e_eng.energies()
        e2e_eng.get_state_ptrs(uo.data_ptr(), tho.data_ptr(), vo.data_ptr())
    barrier()
    t0 = time.perf_counter()
    e2e_eng.set_state_ptrs(u0.data_ptr(), th0.data_ptr(), v0.data_ptr())
    for _ in range(e2e_steps):
        e2e_eng.run(1)
        e2e_eng.energies()
    e2e_eng.get_state_ptrs(uo.data_ptr(), tho.data_ptr(), vo.data_ptr())
    barrier()
    t_e2e = time.perf_counter() - t0
    state_bytes = N * 12 * 8
    e2e = {"value": world * E * e2e_steps / t_e2e, "unit": UNIT,
           "h2d_bytes_per_step": state_bytes / e2e_steps,
           "d2h_bytes_per_step": 5 * 8 + state_bytes / e2e_steps,
           "protocol": f"dl_set_state from pinned host, {e2e_steps} x (dl_run(1) + dl_get_energies), "
                       f"dl_get_state to pinned host"}
    del e2e_eng

    peak, peak_kind = peaks()
    bytes_step = N * BYTES_NODE["mixed"] + E * BYTES_ELEM["mixed"]
    achieved = bytes_step / (t_mixed / args.steps) / 1e9
    traffic = traffic_per_step()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
        "config": {"workload": f"bcc{args.cells}^3 elastoplastic impact: {E} elements, {N} nodes, "
                               f"2 Gauss points, dt=5e-8 s, mixed precision (FP32 element force, FP64 state)",
                   "l2": "flushed (256 MiB write) before every timed step",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "bytes_per_step": bytes_step, "peak_kind": peak_kind,
                     "kernel": "k_persistent<float> (one launch per timed step)"},
        "gpu_launches": step_launches,
        "clocks": clk.summary(),
        "e2e": e2e,
        "mixed_vs_fp64": err,
        "fp64": {"value": world * E * k64 / t_plain, "ms_per_step": t_plain / k64 * 1e3},
        "steady_state_l2_resident": {"value": E * args.steps / t_steady,
                                     "ms_per_step": t_steady / args.steps * 1e3,
                                     "note": "one persistent launch over all steps, no flush"},
        "blocks_of_100_flushed": {"value": E * 100 * nblk / t_blocks,
                                  "ms_per_step": t_blocks / (100 * nblk) * 1e3,
                                  "roofline_frac": bytes_step * 100 * nblk / t_blocks / 1e9 / peak,
                                  "note": f"{nblk} launches of 100 steps, L2 flushed (256 MiB write) before each"},
        "adjoint_over_forward": None,
    }
    if world == 1:
        # configs 1, 3 and 4 (each also has its own --workload line)
        line["workloads"] = other_workloads()
    if world == 1:
        # the differentiation workload's ratio (8^3 BCC, 2000 steps; full
        # report with the finite-difference check: --workload adjoint8)
        adj = measure_adjoint(fd="default")
        # the engine's default: the whole state tape in HBM (no recomputation)
        line["adjoint_over_forward"] = adj["full_tape"]["adjoint_over_forward"]
        fdc = adj["fd_check"]
        line["adjoint"] = {"workload": adj["workload"], "forward_s": adj["forward_s"],
                           "adjoint_s_full_tape": adj["full_tape"]["adjoint_s"],
                           "adjoint_s_checkpoint_every_100": adj["adjoint_s"],
                           "checkpointed_over_forward": adj["adjoint_over_forward"],
                           "fd_max_rel": fdc["fd_max_rel"],
                           "fd_check": fdc}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cv, cn, cdt = cpu_baseline_run(spec, args.cpu_seconds, threads)
        line["cpu_baseline"] = {"value": cv, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{cn} explicit steps of the full lattice (FP64 oracle, "
                                          f"OpenMP over elements), {cdt:.1f} s"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
