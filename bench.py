"""Benchmark of the per-step transport path (bulk -> cells -> LOD_3D diffusion).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): 256^3 voxels x 10 substrates FP64, 100k agents, central
bulk sphere (biofvm_b200.workloads.lod_256), seeded synthetic inputs.  A step
is one full transport step; the metric is voxel-substrate updates per second
(N voxels x S substrates per step).  The 1.34 GB field is larger than L2
(126 MB), so no L2 flush is needed between steps.

N > 1 (torchrun, one process per GPU): every rank advances its own
independent microenvironment of the same size (instances shard across GPUs
with no data-path collective), so per-GPU work is fixed: weak scaling.  Time
is the max over ranks of the device time.

--impl reference times the unmodified BioFVM reference (compiled from its
sources into oracle/_ref/) on this host's cores, on the same workload with the
same --steps and --warmup, and prints the same metric.  The reference's
layout of the 256^3 x 10 case takes about 26 GB of host memory; a host with
less runs the 128^3 x 10 sample instead and says so in the line.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "voxel-substrate updates/s per LOD step"
UNIT = "voxel-substrate updates/s"
BYTES_PER_VS_SWEEP = 16  # one FP64 read + one FP64 write per element per sweep
BYTES_PER_VS_STEP = 3 * BYTES_PER_VS_SWEEP


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons of this process's GPU,
    sampled through NVML every 5 ms while the timed region runs (read only;
    nothing is set).  Falls back to `nvidia-smi -lms 50` without NVML."""

    REASONS = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
               "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
               "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
               "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.samples: list[tuple[float, float, set]] = []
        self.stop = threading.Event()
        self.t = None
        self.proc = None

    def _nvml_handle(self):
        import pynvml

        pynvml.nvmlInit()
        try:
            import torch

            pr = torch.cuda.get_device_properties(self.gpu)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def _nvml_loop(self, nv, h):
        mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        masks = {k: getattr(nv, v) for k, v in self.REASONS.items()}
        while not self.stop.is_set():
            sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            self.samples.append((sm, mx, {k for k, m in masks.items() if r & m}))
            self.stop.wait(0.005)

    def _smi_loop(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        self.proc = subprocess.Popen(
            ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits",
             "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            try:
                sm, mx = float(f[0]), float(f[1])
            except (ValueError, IndexError):
                continue
            act = {k for k, v in zip(self.REASONS, f[2:6]) if v.lower() == "active"}
            self.samples.append((sm, mx, act))

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.t = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
        except Exception:
            self.t = threading.Thread(target=self._smi_loop, daemon=True)
        self.t.start()
        time.sleep(0.01)
        return self

    def __exit__(self, *exc):
        self.stop.set()
        if self.proc is not None:
            self.proc.terminate()
        if self.t is not None:
            self.t.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        reasons = set().union(*(r for _, _, r in self.samples))
        return {"sm_mhz": statistics.median(s for s, _, _ in self.samples),
                "sm_max_mhz": max(m for _, m, _ in self.samples),
                "reasons": sorted(reasons), "samples": len(self.samples)}


TRAFFIC_PROFILE = os.path.join(ROOT, "profiles", "sweeps_traffic_lod256.json")


def ncu_traffic(axis_key: str, kernel_kind: int, chunk: int, row_build: int):
    """DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch
    of the sweep kernel of an axis at the full 256^3 x 10 size, from the
    one-pass ncu capture recorded in profiles/sweeps_traffic_lod256.json
    (the capture's command is in the file).  None when the file lacks the
    axis or the capture ran another kernel than the one timed here: another
    kernel kind (kernel_kind: the tuner's choice, a BFVM_PATH_* value, 0 =
    the default, which the capture ran), chunk length or x row-kernel
    build."""
    if not os.path.exists(TRAFFIC_PROFILE):
        return None, None
    with open(TRAFFIC_PROFILE) as f:
        d = json.load(f)
    k = d.get("launches", {}).get(axis_key)
    if not k or (kernel_kind != 0 and kernel_kind != k.get("path")):
        return None, None
    if k.get("chunk") != chunk or (axis_key == "x_sweep" and k.get("row_build") != row_build):
        return None, None
    return float(k["dram_bytes_read"]) + float(k["dram_bytes_write"]), k["kernel"]


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------

def host_memory_gb():
    """(MemTotal, MemAvailable) of this host in GB, and the cgroup memory
    limit that applies to this process (None when unlimited)."""
    total = avail = None
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                k, v = line.split(":", 1)
                if k == "MemTotal":
                    total = int(v.split()[0]) / 1e6
                elif k == "MemAvailable":
                    avail = int(v.split()[0]) / 1e6
    except OSError:
        pass
    limit = None
    for path in ("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory/memory.limit_in_bytes"):
        try:
            with open(path) as f:
                v = f.read().strip()
            if v.isdigit() and int(v) < (1 << 60):
                limit = int(v) / 1e9
            break
        except OSError:
            continue
    return total, avail, limit


# Host memory the reference's layout takes at 256^3 x 10 with 100k agents
# (a heap vector per voxel for the density, its double buffer and the three
# bulk-rate temporaries, plus the mesh's voxels): 26.4 GB peak resident,
# measured; with headroom for the rest of the process.
REFERENCE_256_GB = 32.0


def reference_scenario(sample: bool):
    """The headline workload (256^3 x 10 FP64, 100k agents, the bulk sphere)
    for the CPU reference; sample=True takes the 128^3 x 10 cube with agents
    at the same density (12.5k), for hosts without the memory for the full
    case."""
    from biofvm_b200 import workloads as W

    if sample:
        return W.lod_cube(128, 10, 12_500, steps=1, name="lod_128_sample")
    return W.lod_256(steps=1)


def time_reference(steps: int, warmup: int, threads: int, sample: bool = False):
    """The reference (compiled from its sources) on this host's cores: setup,
    `warmup` untimed steps (the first allocates the bulk temporaries), then
    `steps` timed steps (steady_clock around the loop)."""
    from oracle import oracle as O

    variant = "v3" if (O.reference_available("v3") and _host_has_avx2()) else "core2"
    scn = reference_scenario(sample)
    t0 = time.perf_counter()
    ref = O.Reference(scn, variant, threads=threads, cells_single_thread=False)
    setup = time.perf_counter() - t0
    if warmup > 0:
        ref.run(warmup)
    secs = ref.run(steps)
    ref.close()
    vs = scn.num_voxels * scn.S * steps / secs
    return vs, secs, setup, variant, scn


def reference_fits():
    """Whether this host can hold the reference's layout of the full
    headline case, and the memory figures that decided it."""
    total, avail, limit = host_memory_gb()
    known = [x for x in (avail, limit, total) if x is not None]
    room = min(known) if known else 0.0
    return room >= REFERENCE_256_GB, {"mem_total_gb": total, "mem_available_gb": avail,
                                      "cgroup_limit_gb": limit}


def _host_has_avx2() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
        return " avx2" in flags and " fma" in flags
    except OSError:
        return False


def reference_baseline(steps: int, warmup: int):
    """cpu_baseline entry: the reference on every host core, on the full
    headline workload when the host has the memory, else on the 128^3 sample
    (said in `sample`)."""
    threads = os.cpu_count() or 1
    fits, mem = reference_fits()
    vs, secs, setup, variant, scn = time_reference(steps, warmup, threads, sample=not fits)
    what = (f"{scn.shape[0]}^3 x {scn.S} substrates, {scn.num_agents} agents, bulk sphere "
            f"r=500um: " + ("the whole headline workload" if fits else
                            "1/8 of the headline workload's voxels (host memory "
                            f"{mem} below the {REFERENCE_256_GB} GB the full case needs)"))
    return {"value": vs, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{what}; {steps} timed steps after {warmup} warm-up; reference build "
                      f"{variant} (OpenMP threads {threads})",
            "ms_per_step": 1e3 * secs / steps, "setup_s": setup, "host_memory": mem,
            "same_config": fits}, scn


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    cpu, scn = reference_baseline(args.steps, args.warmup)
    full = cpu["same_config"]
    line = {
        "impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": cpu["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": ("lod_256: 256^3 voxels x 10 substrates FP64, 100000 agents, "
                                "bulk sphere r=500um, dt=0.01") if full else
                   "lod_256 sample: lod_128 (256^3 x 10 FP64 workload at 1/8 the voxels)",
                   "voxels": scn.num_voxels, "substrates": scn.S, "agents": scn.num_agents,
                   "threads": cpu["cores"], "parallelism": "host cores (OpenMP)"},
        "cpu_baseline": cpu,
        "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "setup_s": cpu["setup_s"],
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------

def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    from biofvm_b200 import STEP_ALL, Solver, load_scenario
    from biofvm_b200 import workloads as W

    if args.size == 256 and args.substrates == 10 and args.agents == 100_000:
        scn = W.lod_256(steps=args.steps)
    else:
        scn = W.lod_cube(args.size, args.substrates, args.agents, steps=args.steps,
                         name=f"lod_{args.size}")
    N, S = scn.num_voxels, scn.S
    sv = Solver(local)
    load_scenario(sv, scn)
    dt = scn.dt
    stream = torch.cuda.ExternalStream(sv.stream, device=torch.device("cuda", local))

    # warm-up (also builds the Thomas coefficients and the device lists), then
    # the per-axis kernel choice timed on this field (which is restored)
    sv.step(dt, args.warmup, STEP_ALL)
    tuned = sv.tune_sweeps(dt, 3) if not args.no_tune else [(0, 0, 0, 0, 0)] * 3
    if args.sweep_chunks:
        # only where the chunk length changes: a set configuration also
        # returns the axis to its default kernel kind
        for ax, ch in enumerate(int(c) for c in args.sweep_chunks.split(",")):
            if sv.get_sweep_config(ax)[0] != ch:
                sv.set_sweep_config(ax, ch, 16, 1)
    if args.row_build is not None:
        sv.set_row_build(args.row_build)
    row_build = sv.get_row_build()
    sv.synchronize()

    launches0 = sv.launch_count
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        barrier(world)
        torch.cuda.synchronize(local)
        sv.synchronize()
        ev0.record(stream)
        sv.step(dt, args.steps, STEP_ALL)
        ev1.record(stream)
        ev1.synchronize()
        sv.synchronize()
        barrier(world)
    launches = sv.launch_count - launches0
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms, world)
    value = N * S * args.steps * world / (ms / 1e3)
    ms_step = ms / args.steps

    # per-kernel device times on the solver's stream (CUDA events between sweeps)
    ks, kx, ky, kz = sv.profile_step(dt, max(3, min(args.steps, 10)), STEP_ALL)
    if sv.get_slab_planes() > 0:
        # x and y by slabs: their events bracket both sweeps together
        per = {"xy_sweeps_by_slabs": kx, "z_sweep": kz}
        sweeps_in = {"xy_sweeps_by_slabs": 2, "z_sweep": 1}
    else:
        per = {"x_sweep": kx, "y_sweep": ky, "z_sweep": kz}
        sweeps_in = {"x_sweep": 1, "y_sweep": 1, "z_sweep": 1}
    dom = max(per, key=per.get)
    per["sources"] = ks
    hbm, peak_kind = peaks()
    achieved = sweeps_in[dom] * BYTES_PER_VS_SWEEP * N * S / (per[dom] / 1e3) / 1e9
    dom_axis = {"x_sweep": 0, "y_sweep": 1, "z_sweep": 2}.get(dom)
    traffic, traffic_kernel = (ncu_traffic(dom, tuned[dom_axis][0],
                                           sv.get_sweep_config(dom_axis)[0], row_build[1])
                               if dom_axis is not None else (None, None))

    # end to end through the C ABI with host buffers: every step uploads the
    # agents' voxels and secretion/uptake constants (as when agents move and
    # change rates each step) and reads back the densities at the agents.
    e2e = None
    if not args.no_e2e:
        # host buffers in page-locked memory, as a host loop that exchanges
        # agent data with the solver every step would keep them
        import torch

        keep = []

        def pinned(a):
            t = torch.empty(a.shape, dtype=torch.from_numpy(a[:0]).dtype, pin_memory=True)
            keep.append(t)
            v = t.numpy()
            v[...] = a
            return v

        vox, t1, t2 = (pinned(np.ascontiguousarray(a)) for a in scn.agent_arrays())
        out = pinned(np.empty((scn.num_agents, S)))
        e_steps = max(1, min(args.steps, 20))

        def exchange_loop(asynchronous):
            sv.synchronize()
            barrier(world)
            t0 = time.perf_counter()
            for _ in range(e_steps):
                if asynchronous:
                    # the copies run on the solver's upload/download streams,
                    # overlapping the neighbouring steps' sweeps
                    sv.set_agents_async(vox, t1, t2)
                    sv.step(dt, 1, STEP_ALL)
                    sv.get_agent_densities_async(out)
                else:
                    sv.set_agents(vox, t1, t2)
                    sv.step(dt, 1, STEP_ALL)
                    sv.get_agent_densities(out)
            sv.synchronize()
            return max_over_ranks(time.perf_counter() - t0, world)

        exchange_loop(True)  # creates the transfer streams and events
        e_secs = exchange_loop(True)
        sync_secs = exchange_loop(False)
        e2e = {"value": N * S * e_steps * world / e_secs, "unit": UNIT,
               "h2d_bytes_per_step": int(vox.nbytes + t1.nbytes + t2.nbytes),
               "d2h_bytes_per_step": int(out.nbytes), "steps": e_steps,
               "what": "per step: bfvm_set_agents_async (pinned host voxel+temp1+temp2), "
                       "bfvm_step, bfvm_get_agent_densities_async (pinned host [A][S]); "
                       "wall clock to the last copy's end",
               "synchronous_calls_value": N * S * e_steps * world / sync_secs}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference on this host's cores, on the same workload with the
        # same steps and warm-up (after the device work, which it does not
        # overlap)
        try:
            sv.synchronize()
            cpu, _ = reference_baseline(args.steps, args.warmup)
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": f"{scn.name}: {args.size}^3 voxels x {S} substrates FP64, "
                                   f"{scn.num_agents} agents, bulk sphere r=500um, dt=0.01",
                       "voxels": N, "substrates": S, "agents": scn.num_agents,
                       "l2": (f"inputs ({N * S * 8 / 1e9:.2f} GB field) larger than L2; no flush"
                              if N * S * 8 > 126e6 else
                              f"field ({N * S * 8 / 1e6:.0f} MB) fits in L2; no flush"),
                       "parallelism": f"instances x{world}" if world > 1 else "1 GPU"},
            "hbm_gbs_step": BYTES_PER_VS_STEP * N * S / (ms_step / 1e3) / 1e9,
            "hbm_frac_step": BYTES_PER_VS_STEP * N * S / (ms_step / 1e3) / 1e9 / hbm,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic, "traffic_kernel": traffic_kernel,
                         "traffic_source": "profiles/sweeps_traffic_lod256.json (ncu, one "
                                           "launch at 256^3 x 10)" if traffic else None,
                         "algorithmic_bytes_per_launch": sweeps_in[dom] * BYTES_PER_VS_SWEEP * N * S},
            "kernel_ms": per,
            "tuned_sweeps": [{"axis": "xyz"[i], "kernel": ["default", "register", "tma", "direct"][k],
                              "chunk": ch, "columns": tw, "min_blocks": mb, "row_stages": st}
                             for i, (k, ch, tw, mb, st) in enumerate(tuned)],
            "row_build": dict(zip(("requested", "effective"), row_build)),
            "slab_planes": sv.get_slab_planes(), "fuse_sources": sv.get_fuse_sources(),
            "gpu_launches": int(launches),
            "e2e": e2e,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
        }
        if world == 1 and not args.no_configs:
            try:
                line["other_configs"] = other_configs(local)
            except Exception as exc:  # reported, not fatal
                line["other_configs"] = {"error": f"{type(exc).__name__}: {exc}"}
        print(json.dumps(line), flush=True)
    sv.close()


def other_configs(local):
    """The two other single-GPU configurations of the path, measured briefly
    beside the headline line so that every run records them:
      plain_50  50^3 x 1 FP64, all-boundary Dirichlet, 1000 agents, 100 steps:
                microseconds per step of one bfvm_step call (all steps in one
                cooperative launch) and of 100 one-step calls; the reference
                on the host cores for the same 100 steps;
      batched   the 64 instances (grids 32^3..128^3, 1-8 substrates, 0-20k
                agents), 200 steps: the batch in branch mode and in the
                persistent mode (default group budget, no tuning) against the
                same instances solved one by one, wall clock around each,
                results compared within 1e-10."""
    import torch

    from biofvm_b200 import STEP_ALL, Batch, Solver, load_scenario
    from biofvm_b200 import workloads as W
    from biofvm_b200._abi import BATCH_BRANCHES, BATCH_PERSISTENT, BATCH_PLANES
    from oracle import oracle as O

    out = {}
    # ---- plain_50
    scn = W.plain_50(steps=100)
    with Solver(local) as sv:
        load_scenario(sv, scn)
        stream = torch.cuda.ExternalStream(sv.stream, device=torch.device("cuda", local))
        p0 = scn.initial_field()

        def timed(fn):
            sv.set_densities(p0)
            sv.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1)

        def one_step_calls():
            for _ in range(100):
                sv.step(scn.dt, 1, STEP_ALL)

        sv.step(scn.dt, 3, STEP_ALL)
        ms_one = timed(one_step_calls)
        ms_all = timed(lambda: sv.step(scn.dt, 100, STEP_ALL))
        got = sv.get_densities()
    threads = os.cpu_count() or 1
    variant = "v3" if (O.reference_available("v3") and _host_has_avx2()) else "core2"
    r = O.Reference(scn, variant, threads=threads, cells_single_thread=False)
    r.run(3)
    secs = r.run(100)
    r.close()
    ref = O.oracle_run(scn, 100, 7)
    out["plain_50"] = {
        "workload": "50^3 x 1 FP64, all-boundary Dirichlet 1.0, 1000 uptake agents, 100 steps",
        "us_per_step_one_call": 1e3 * ms_all / 100,
        "us_per_step_one_step_calls": 1e3 * ms_one / 100,
        "reference_us_per_step": 1e6 * secs / 100, "reference_threads": threads,
        "max_rel_err_vs_oracle": float(O.max_rel_err(got, ref).max())}
    # ---- batched
    scns = W.batched_instances(count=64, steps=200)
    sols = []
    for sc in scns:
        sv = Solver(local)
        load_scenario(sv, sc)
        sols.append(sv)
    dt = scns[0].dt

    def reset():
        for sv, sc in zip(sols, scns):
            sv.set_densities(sc.initial_field())
        for sv in sols:
            sv.synchronize()

    for sv in sols:
        sv.step(dt, 1, STEP_ALL)
    reset()
    t0 = time.perf_counter()
    for sv in sols:
        sv.step(dt, 200, STEP_ALL)
        sv.synchronize()
    t_plain = time.perf_counter() - t0
    plain = [sv.get_densities() for sv in sols]
    bt = Batch(local)
    for sv in sols:
        bt.add(sv)
    modes = {}
    err = 0.0
    # (mode, group budget): -1 = half of L2, 0 = every member in one group
    for name, md, budget in (("branches", BATCH_BRANCHES, -1), ("persistent", BATCH_PERSISTENT, -1),
                             ("planes", BATCH_PLANES, -1), ("planes_one_group", BATCH_PLANES, 0)):
        bt.set_mode(md)
        bt.set_config((0, 0, 0), (0, 0, 0), budget)
        reset()
        bt.step(dt, 200, STEP_ALL)  # captures the graph
        bt.synchronize()
        reset()
        t0 = time.perf_counter()
        bt.step(dt, 200, STEP_ALL)
        bt.synchronize()
        t_b = time.perf_counter() - t0
        groups, kernels = bt.plan()
        e = max(float(O.max_rel_err(sv.get_densities(), ref_p).max())
                for sv, ref_p in zip(sols, plain))
        err = max(err, e)
        modes[name] = {"seconds": t_b, "speedup_vs_looped_plain": t_plain / t_b,
                       "groups": groups, "kernels_per_call": kernels}
    bt.close()
    for sv in sols:
        sv.close()
    vs = sum(sc.num_voxels * sc.S for sc in scns)
    t_batch = modes["branches"]["seconds"]
    out["batched"] = {
        "workload": "64 instances, grids 32^3..128^3, 1-8 substrates, 0-20k agents, 200 steps",
        "mode": "branches (default group budget, not tuned); the persistent and plane modes "
                "beside it",
        "batched_seconds": t_batch, "looped_plain_seconds": t_plain,
        "speedup_vs_looped_plain": t_plain / t_batch,
        "value": vs * 200 / t_batch, "unit": UNIT, "modes": modes,
        "max_rel_err_vs_looped_plain": err}
    return out


def run_sharded(args, world, rank, local):
    """One microenvironment (the headline 256^3 x 10 workload by default)
    split by substrate over the ranks, each rank a Solver stepping its block
    (biofvm_b200.sharding.SubstrateShard): no collective inside a step, total
    work fixed as N grows (strong scaling; 10 substrates over 8 ranks is
    blocks of 2 and 1).  Time: the max over ranks of each rank's device time
    (CUDA events on its solver's stream); then one all-gather of the whole
    field into device memory (NCCL), timed on its own."""
    import torch
    import torch.distributed as dist

    from biofvm_b200 import STEP_ALL
    from biofvm_b200 import workloads as W
    from biofvm_b200.sharding import SubstrateShard, substrate_range

    if world == 1 and not dist.is_initialized():
        import datetime

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29533")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=120))
    if args.size == 256 and args.substrates == 10 and args.agents == 100_000:
        scn = W.lod_256(steps=args.steps)
    else:
        scn = W.lod_cube(args.size, args.substrates, args.agents, steps=args.steps,
                         name=f"lod_{args.size}")
    N, S = scn.num_voxels, scn.S
    shard = SubstrateShard(scn, device=local)
    dt = scn.dt
    sv = shard.solver
    if sv is not None:
        sv.step(dt, args.warmup, STEP_ALL)
        if not args.no_tune:
            sv.tune_sweeps(dt, 3)
        sv.synchronize()
    stream = (torch.cuda.ExternalStream(sv.stream, device=torch.device("cuda", local))
              if sv is not None else torch.cuda.current_stream(local))
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    launches0 = sv.launch_count if sv is not None else 0
    with ClockSampler(local) as clocks:
        barrier(world)
        torch.cuda.synchronize(local)
        ev0.record(stream)
        shard.step(dt, args.steps, STEP_ALL)
        ev1.record(stream)
        ev1.synchronize()
        barrier(world)
    launches = (sv.launch_count - launches0) if sv is not None else 0
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    # one gather of the whole field into this GPU's memory
    barrier(world)
    torch.cuda.synchronize(local)
    t0 = time.perf_counter()
    full = shard.gather_device()
    torch.cuda.synchronize(local)
    t_gather = max_over_ranks(time.perf_counter() - t0, world)
    ok = bool(tuple(full.shape) == (N, S))
    del full
    shard.close()
    if rank == 0:
        _, peak_kind = peaks()
        vs = N * S * args.steps
        line = {
            "metric": METRIC + " (one microenvironment sharded by substrate)",
            "value": vs / (ms / 1e3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": f"{scn.name}: {args.size}^3 voxels x {S} substrates FP64, "
                                   f"{scn.num_agents} agents, bulk sphere r=500um",
                       "parallelism": f"substrates x{world}",
                       "substrates_per_rank": [b - a for a, b in (substrate_range(S, world, r)
                                                                  for r in range(world))],
                       "l2": "inputs larger than L2; no flush"},
            "hbm_gbs_step_per_gpu": BYTES_PER_VS_STEP * N * S / world / (ms / args.steps / 1e3)
            / 1e9,
            "gather_device_seconds": t_gather, "gather_ok": ok,
            "gpu_launches": int(launches), "peak_kind": peak_kind,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)


def run_batched(args, world, rank, local):
    """The batched workload: 64 independent microenvironments (grids drawn
    from 32^3 to 128^3, 1-8 substrates, 0-20k agents each; seeded), 200 steps,
    advanced by one bfvm_batch_step call (one CUDA-graph replay) against the
    same instances solved one after another with bfvm_step.  Both arms start
    from the same fields and are timed by the wall clock around the call plus
    a device synchronisation; the batched results must match the looped ones
    within 1e-10 relative max-norm per substrate."""
    import numpy as np

    from biofvm_b200 import STEP_ALL, Batch, Solver, load_scenario
    from biofvm_b200 import workloads as W

    count = args.instances
    scns = W.batched_instances(count=count, steps=args.steps)
    sols = []
    for scn in scns:
        sv = Solver(local)
        load_scenario(sv, scn)
        sols.append(sv)
    dt = scns[0].dt
    vs_per_step = sum(s.num_voxels * s.S for s in scns)

    def reset():
        for sv, scn in zip(sols, scns):
            sv.set_densities(scn.initial_field())
        for sv in sols:
            sv.synchronize()

    # looped plain solves (first one warms every instance up: Thomas setup, lists)
    for sv in sols:
        sv.step(dt, 1, STEP_ALL)
    reset()
    barrier(world)
    t0 = time.perf_counter()
    for sv in sols:
        sv.step(dt, args.steps, STEP_ALL)
        sv.synchronize()
    t_plain = max_over_ranks(time.perf_counter() - t0, world)
    plain = [sv.get_densities() for sv in sols]

    bt = Batch(local)
    for sv in sols:
        bt.add(sv)
    reset()
    t0 = time.perf_counter()
    if args.batch_mode == "tuned":
        bt.tune(dt, STEP_ALL, args.batch_trial_steps)
    else:
        from biofvm_b200._abi import BATCH_BRANCHES, BATCH_FUSED, BATCH_PERSISTENT, BATCH_PLANES
        bt.set_mode({"fused": BATCH_FUSED, "branches": BATCH_BRANCHES,
                     "persistent": BATCH_PERSISTENT, "planes": BATCH_PLANES}[args.batch_mode])
        bt.set_persistent_chunk(args.batch_chunk)
    t_tune = time.perf_counter() - t0
    cfg = bt.get_config()
    pch = bt.get_persistent_chunk()
    # first call captures the graph; the timed call replays it
    reset()
    t0 = time.perf_counter()
    bt.step(dt, args.steps, STEP_ALL)
    bt.synchronize()
    t_first = time.perf_counter() - t0
    reset()
    with ClockSampler(local) as clocks:
        barrier(world)
        t0 = time.perf_counter()
        bt.step(dt, args.steps, STEP_ALL)
        bt.synchronize()
        t_batch = max_over_ranks(time.perf_counter() - t0, world)
    groups, kernels = bt.plan()
    mode = bt.get_mode()
    # every mode with the tuned group budget, for comparison (captured, then
    # timed on a replay)
    per_mode = {}
    if args.batch_modes:
        from biofvm_b200._abi import BATCH_BRANCHES, BATCH_FUSED, BATCH_PERSISTENT, BATCH_PLANES
        for name, md in (("fused", BATCH_FUSED), ("branches", BATCH_BRANCHES),
                         ("persistent", BATCH_PERSISTENT), ("planes", BATCH_PLANES)):
            bt.set_mode(md)
            reset()
            bt.step(dt, args.steps, STEP_ALL)
            bt.synchronize()
            reset()
            t0 = time.perf_counter()
            bt.step(dt, args.steps, STEP_ALL)
            bt.synchronize()
            t_m = time.perf_counter() - t0
            per_mode[name] = {"seconds": t_m, "speedup_vs_looped_plain": t_plain / t_m,
                              "groups_kernels": list(bt.plan())}
        bt.set_mode(mode)
        reset()
        bt.step(dt, args.steps, STEP_ALL)  # the tuned mode's fields for the check below
        bt.synchronize()
    err = 0.0
    for sv, ref in zip(sols, plain):
        p = sv.get_densities()
        den = np.maximum(np.abs(ref).max(axis=0), 1e-300)
        err = max(err, float((np.abs(p - ref).max(axis=0) / den).max()))
    # for reference: the members keep the sweep kernels the batch tuner chose
    # for each of them; the same instances solved one by one with those
    reset()
    barrier(world)
    t0 = time.perf_counter()
    for sv in sols:
        sv.step(dt, args.steps, STEP_ALL)
        sv.synchronize()
    t_plain_tuned = max_over_ranks(time.perf_counter() - t0, world)
    bt.close()
    for sv in sols:
        sv.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference on the host cores, the instances one after another
        # (one Microenvironment each), a bounded number of steps
        try:
            from oracle import oracle as O

            threads = os.cpu_count() or 1
            variant = "v3" if (O.reference_available("v3") and _host_has_avx2()) else "core2"
            ref_steps = 5
            secs = 0.0
            for sc in scns:
                r = O.Reference(sc, variant, threads=threads, cells_single_thread=False)
                r.run(1)
                secs += r.run(ref_steps)
                r.close()
            cpu = {"value": vs_per_step * ref_steps / secs, "unit": UNIT, "cores": threads,
                   "kind": "reference",
                   "sample": f"the {count} instances one after another, {ref_steps} timed steps "
                             f"each after 1 warm-up; reference build {variant}"}
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {exc}"}
    if rank == 0:
        line = {
            "metric": METRIC + " (batched instances)", "value": vs_per_step * args.steps * world /
            t_batch, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": 1,
            "ms_per_step": 1e3 * t_batch / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": f"batched: {count} instances, grids 32^3..128^3, 1-8 "
                                   f"substrates, 0-20k agents, {args.steps} steps",
                       "voxel_substrates_per_step": vs_per_step,
                       "field_bytes": vs_per_step * 8},
            "looped_plain": {"value": vs_per_step * args.steps * world / t_plain,
                             "seconds": t_plain},
            "looped_with_tuned_members": {"value": vs_per_step * args.steps * world /
                                          t_plain_tuned, "seconds": t_plain_tuned},
            "batched_seconds": t_batch, "speedup_vs_looped_plain": t_plain / t_batch,
            "max_rel_err_vs_looped_plain": err,
            "tuned": {"mode": ["fused", "branches", "persistent", "planes"][mode], "chunk": cfg[0],
                      "threads": cfg[1], "group_bytes": cfg[2], "persistent_chunk": pch,
                      "tune_seconds": t_tune, "trial_steps": args.batch_trial_steps},
            "graph": {"groups": groups, "kernels_per_call": kernels,
                      "first_call_seconds": t_first},
            "modes_with_tuned_budget": per_mode,
            "gpu_launches": kernels,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)


def run_fp32(args, world, rank, local):
    """FP32 sweeps (FP64 Thomas coefficients rounded once to FP32, FP64
    arithmetic in the bulk and cell updates) at 512^3 voxels x 8 substrates
    with 1M agents, 50 steps, next to the FP64 path timed on the same
    workload; reports the max relative error per substrate of the FP32 field
    against the FP64 one after the run."""
    import numpy as np
    import torch

    from biofvm_b200 import FP32, STEP_ALL, Solver, load_scenario
    from biofvm_b200 import workloads as W
    from biofvm_b200._abi import FP32_FP64MATH

    n = args.size if "--size" in sys.argv else 512
    S = args.substrates if "--substrates" in sys.argv else 8
    A = args.agents if "--agents" in sys.argv else 1_000_000
    scn = W.lod_cube(n, S, A, steps=args.steps, name=f"lod_{n}")
    N = scn.num_voxels
    sv = Solver(local)
    load_scenario(sv, scn)
    dt = scn.dt
    stream = torch.cuda.ExternalStream(sv.stream, device=torch.device("cuda", local))
    p0 = scn.initial_field()

    def timed(clocks=None):
        sv.step(dt, args.warmup, STEP_ALL)
        sv.tune_sweeps(dt, 2)
        sv.set_densities(p0)
        sv.synchronize()
        barrier(world)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        sv.step(dt, args.steps, STEP_ALL)
        ev1.record(stream)
        ev1.synchronize()
        return max_over_ranks(ev0.elapsed_time(ev1), world)

    ms64 = timed()
    ref = sv.get_densities()
    sv.set_precision(FP32)
    sv.set_densities(p0)
    with ClockSampler(local) as clocks:
        ms32 = timed()
    got = sv.get_densities()
    den = np.maximum(np.abs(ref).max(axis=0), 1e-300)
    err = (np.abs(got - ref).max(axis=0) / den).tolist()
    # the FP32 field swept in FP64 arithmetic (FP32_FP64MATH)
    sv.set_precision(FP32_FP64MATH)
    sv.set_densities(p0)
    ms_mixed = timed()
    got = sv.get_densities()
    err_mixed = (np.abs(got - ref).max(axis=0) / den).tolist()
    sv.close()
    if rank == 0:
        hbm, peak_kind = peaks()
        bytes32 = 3 * 8 * N * S * args.steps
        line = {
            "metric": METRIC + " (FP32 sweeps)", "value": N * S * args.steps * world / (ms32 / 1e3),
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms32 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": f"lod_{n}: {n}^3 voxels x {S} substrates, {A} agents, "
                                   f"{args.steps} steps, FP32 sweeps / FP64 coefficients and "
                                   f"source arithmetic", "voxels": N, "substrates": S,
                       "agents": A, "l2": "inputs larger than L2; no flush"},
            "hbm_gbs_step": bytes32 / (ms32 / 1e3) / 1e9,
            "roofline": {"bound": "hbm", "kernel": "whole step (3 sweeps, 24 B/VS)",
                         "achieved": bytes32 / (ms32 / 1e3) / 1e9, "peak": hbm,
                         "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": bytes32 / (ms32 / 1e3) / 1e9 / hbm, "traffic": None},
            "fp64_same_workload": {"value": N * S * args.steps * world / (ms64 / 1e3),
                                   "ms_per_step": ms64 / args.steps},
            "max_rel_err_vs_fp64_per_substrate": err,
            "fp32_field_fp64_sweeps": {
                "value": N * S * args.steps * world / (ms_mixed / 1e3),
                "ms_per_step": ms_mixed / args.steps,
                "max_rel_err_vs_fp64_per_substrate": err_mixed},
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)


def run_plain50(args, world, rank, local):
    """The small launch-bound workload: 50^3 voxels x 1 substrate, all-boundary
    Dirichlet 1.0, 1000 uptake agents, 100 steps.  Reports microseconds per
    step for bfvm_step as a user calls it (a field this small runs all its
    steps in one cooperative launch: grid steps), for the sweep kernels
    launched from the host (grid steps off) and replayed from a CUDA graph (a
    one-member bfvm_batch), for the opt-in bit-exact thread-block-cluster
    mode, and the reference on the host cores for the same run."""
    import numpy as np
    import torch

    from biofvm_b200 import STEP_ALL, Batch, Solver, load_scenario
    from biofvm_b200 import workloads as W

    scn = W.plain_50(steps=args.steps)
    sv = Solver(local)
    load_scenario(sv, scn)
    p0 = scn.initial_field()
    dt = scn.dt
    stream = torch.cuda.ExternalStream(sv.stream, device=torch.device("cuda", local))

    def timed(fn):
        """Device time of fn() on the solver's stream (CUDA events), ms."""
        sv.set_densities(p0)
        sv.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        sv.synchronize()
        return e0.elapsed_time(e1)

    # bfvm_step as it runs by default: every step in one cooperative launch
    grid_blocks = sv.get_grid_steps()
    sv.step(dt, 3, STEP_ALL)
    l0 = sv.launch_count
    with ClockSampler(local) as clocks:
        ms_loop = timed(lambda: sv.step(dt, args.steps, STEP_ALL))
    launches = sv.launch_count - l0
    grid_field = sv.get_densities()

    def one_step_calls():
        for _ in range(args.steps):
            sv.step(dt, 1, STEP_ALL)

    # one step per call, as the drop-in's simulate_diffusion_decay calls it
    l0 = sv.launch_count
    ms_loop_1 = timed(one_step_calls)
    launches_1 = sv.launch_count - l0
    # the sweep kernels, launched from the host (seven kernels per step)
    sv.set_grid_steps(False)
    sv.step(dt, 3, STEP_ALL)
    l0 = sv.launch_count
    ms_sweep = timed(lambda: sv.step(dt, args.steps, STEP_ALL))
    sweep_launches = sv.launch_count - l0
    ms_sweep_1 = timed(one_step_calls)
    ref = sv.get_densities()
    # the same steps in one thread-block cluster (opt-in; bit-exact)
    sv.set_cluster_steps(True)
    blocks = sv.get_cluster_steps()
    sv.step(dt, 3, STEP_ALL)
    ms_cluster = timed(lambda: sv.step(dt, args.steps, STEP_ALL))
    cluster_field = sv.get_densities()
    sv.set_cluster_steps(False)
    # the sweep kernels replayed from a CUDA graph
    bt = Batch(local)
    bt.add(sv)
    sv.set_densities(p0)
    bt.step(dt, args.steps, STEP_ALL)  # captures the graph
    bt.synchronize()
    sv.set_densities(p0)
    sv.synchronize()
    t0 = time.perf_counter()
    bt.step(dt, args.steps, STEP_ALL)
    bt.synchronize()
    t_graph = time.perf_counter() - t0
    got = sv.get_densities()

    def rel(a, b):
        return float((np.abs(a - b).max(axis=0) / np.maximum(np.abs(b).max(axis=0), 1e-300)).max())

    err = rel(got, ref)
    err_cluster = rel(cluster_field, ref)
    err_grid = rel(grid_field, ref)
    groups, kernels = bt.plan()
    bt.close()
    sv.close()
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        threads = os.cpu_count() or 1
        variant = "v3" if (O.reference_available("v3") and _host_has_avx2()) else "core2"
        r = O.Reference(scn, variant, threads=threads, cells_single_thread=False)
        r.run(3)
        secs = r.run(args.steps)
        r.close()
        cpu = {"value": scn.num_voxels * args.steps / secs, "unit": UNIT, "cores": threads,
               "kind": "reference", "us_per_step": 1e6 * secs / args.steps,
               "sample": f"the whole workload ({args.steps} steps), reference build {variant}"}
    if rank == 0:
        vs = scn.num_voxels * scn.S * args.steps
        line = {
            "metric": METRIC + " (50^3 launch-bound case)", "value": vs * world / (ms_loop / 1e3),
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": 3,
            "ms_per_step": ms_loop / args.steps, "us_per_step": 1e3 * ms_loop / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": "plain_50: 50^3 x 1 FP64, all-boundary Dirichlet 1.0, 1000 "
                                   f"uptake agents, {args.steps} steps",
                       "path": "bfvm_step default: all steps in one cooperative launch "
                               f"of {grid_blocks} blocks (grid steps)"},
            "gpu_launches": int(launches),
            "sweep_kernels_host_launched": {"us_per_step": 1e3 * ms_sweep / args.steps,
                                            "launches": int(sweep_launches)},
            "one_step_per_call": {"bfvm_step_default_us_per_step": 1e3 * ms_loop_1 / args.steps,
                                  "launches": int(launches_1),
                                  "sweep_kernels_us_per_step": 1e3 * ms_sweep_1 / args.steps},
            "sweep_kernels_graph": {"us_per_step": 1e6 * t_graph / args.steps,
                                    "kernels_per_call": kernels},
            "cluster_steps_bit_exact": {"us_per_step": 1e3 * ms_cluster / args.steps,
                                        "blocks": blocks},
            "max_rel_err_grid_steps_vs_sweep_kernels": err_grid,
            "max_rel_err_cluster_vs_sweep_kernels": err_cluster,
            "max_rel_err_graph_vs_host_launched": err,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)


def run_lod2d(args, world, rank, local):
    """diffusion_decay_solver__constant_coefficients_LOD_2D
    (BioFVM_solvers.cpp:278-427) on a 1024 x 1024 x 32 FP64 plane (268 MB,
    larger than L2; lines are at most 1024 points) (dx = 10,
    D log-uniform in [1e3, 1e5], decay uniform in [0.01, 1], dt = 0.01):
    the x and y sweeps of the plane with the Dirichlet overwrites fused.
    Algorithmic bytes 32 B/VS per step (two sweeps, one read and one write of
    the field each); CUDA events on the solver's stream."""
    import numpy as np
    import torch

    from biofvm_b200 import Solver

    n = args.size if "--size" in sys.argv else 1024
    S = args.substrates if "--substrates" in sys.argv else 32
    rng = np.random.default_rng(12351)
    sv = Solver(local)
    sv.resize_densities(S)
    sv.resize_space(0, n * 10.0, 0, n * 10.0, -5.0, 5.0, 10.0)
    sv.set_coefficients(np.exp(rng.uniform(np.log(1e3), np.log(1e5), S)),
                        rng.uniform(0.01, 1.0, S))
    sv.set_densities(rng.random((n * n, S)))
    stream = torch.cuda.ExternalStream(sv.stream, device=torch.device("cuda", local))
    dt = 0.01
    for _ in range(max(3, args.warmup)):
        sv.simulate_diffusion_decay_2d(dt)
    # the sweep kernels timed on this plane (after the first step fixed the
    # LOD_2D Thomas coefficients; the field is restored)
    tuned = sv.tune_sweeps(dt, 3) if not args.no_tune else []
    sv.set_slab_planes(0)
    sv.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    l0 = sv.launch_count
    with ClockSampler(local) as clocks:
        barrier(world)
        e0.record(stream)
        for _ in range(args.steps):
            sv.simulate_diffusion_decay_2d(dt)
        e1.record(stream)
        e1.synchronize()
    launches = sv.launch_count - l0
    ms = max_over_ranks(e0.elapsed_time(e1), world) / args.steps
    sv.close()
    if rank == 0:
        hbm, peak_kind = peaks()
        vs = n * n * S
        achieved = 32.0 * vs / (ms / 1e3) / 1e9
        line = {
            "metric": METRIC + " (LOD_2D)", "value": vs * world / (ms / 1e3), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": f"lod2d: {n}^2 voxels x {S} substrates FP64",
                       "l2": "field larger than L2; no flush"},
            "tuned_sweeps": [{"axis": "xy"[i], "kernel": ["default", "register", "tma",
                                                          "direct"][k],
                              "chunk": ch, "columns": tw} for i, (k, ch, tw, *_) in
                             enumerate(tuned[:2])],
            "roofline": {"bound": "hbm", "kernel": "x and y sweeps of the plane",
                         "achieved": achieved, "peak": hbm, "peak_kind": peak_kind,
                         "unit": "GB/s", "frac": achieved / hbm, "traffic": None},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)


def run_gradients(args, world, rank, local):
    """Microenvironment::compute_all_gradient_vectors on the device field
    (BioFVM_microenvironment.cpp:702-787) at 256^3 voxels x 10 substrates FP64:
    central differences along each axis into [N][S][3] FP64.  Algorithmic
    bytes: the field read once (8 B/VS) and three gradients written (24 B/VS);
    timed with CUDA events on the solver's stream over the calls."""
    import numpy as np
    import torch

    from biofvm_b200 import Solver

    n = args.size if "--size" in sys.argv else 256
    S = args.substrates if "--substrates" in sys.argv else 10
    sv = Solver(local)
    sv.resize_densities(S)
    sv.resize_space(0, n * 10.0, 0, n * 10.0, 0, n * 10.0, 10.0)
    rng = np.random.default_rng(12350)
    sv.set_densities(rng.random((n ** 3, S)))
    stream = torch.cuda.ExternalStream(sv.stream, device=torch.device("cuda", local))
    for _ in range(max(3, args.warmup)):
        sv.compute_all_gradient_vectors()
    sv.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    l0 = sv.launch_count
    with ClockSampler(local) as clocks:
        barrier(world)
        e0.record(stream)
        for _ in range(args.steps):
            sv.compute_all_gradient_vectors()
        e1.record(stream)
        e1.synchronize()
    launches = sv.launch_count - l0
    ms = max_over_ranks(e0.elapsed_time(e1), world) / args.steps
    sv.close()
    if rank == 0:
        hbm, peak_kind = peaks()
        vs = n ** 3 * S
        achieved = 32.0 * vs / (ms / 1e3) / 1e9
        line = {
            "metric": "voxel-substrate gradients/s (compute_all_gradient_vectors)",
            "value": vs * world / (ms / 1e3), "unit": "voxel-substrate gradients/s",
            "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": f"gradients: {n}^3 voxels x {S} substrates FP64",
                       "l2": "field and gradients larger than L2; no flush"},
            "roofline": {"bound": "hbm", "kernel": "gradient_rows_kernel", "achieved": achieved,
                         "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": None,
                         "algorithmic_bytes_per_launch": 32 * vs},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)


def run_adjoint(args, world, rank, local):
    """The adjoint workload: 128^3 voxels x 4 substrates FP64, 20k agents,
    200 steps with checkpoints every 20.  Loss = 1/2 |p_T - target|^2, the
    target made by the forward run with every parameter scaled by
    (1 + 0.01 N(0,1)) (seeded).  Reports the forward (with checkpoints) and
    backward device times, their ratio, and the agreement of the gradient
    with central finite differences (h = 1e-6 relative) along a random
    direction in each parameter group and in all of them."""
    import numpy as np

    from biofvm_b200 import workloads as W
    from biofvm_b200.adjoint import AdjointProblem, loss_difference

    n = args.size if "--size" in sys.argv else 128
    S = args.substrates if "--substrates" in sys.argv else 4
    A = args.agents if "--agents" in sys.argv else 20_000
    k = 20
    scn = W.lod_cube(n, S, A, steps=args.steps, name=f"lod_{n}")
    th = [np.array(scn.agent_secretion, float), np.array(scn.agent_uptake, float),
          np.array(scn.D, float), np.array(scn.decay, float)]
    rng = np.random.default_rng(12349)
    prob = AdjointProblem(scn, args.steps, checkpoint_every=k, device=local)
    target = prob.run(*[x * (1 + 0.01 * rng.standard_normal(x.shape)) for x in th])
    prob.forward(*th)  # warm-up of both passes
    prob.backward(np.zeros((scn.num_voxels, S)))
    from biofvm_b200._abi import call

    sv = prob.solver
    with ClockSampler(local) as clocks:
        prob.set_parameters(*th)
        sv.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        call("bfvm_adjoint_forward", sv.handle, scn.dt, args.steps, prob.flags, k)
        sv.synchronize()
        t_fwd = time.perf_counter() - t0
        seed = sv.get_densities() - target
        t0 = time.perf_counter()
        g = prob.backward(seed)  # includes the seed upload and the gradient reads
        t_bwd = time.perf_counter() - t0
    prob.set_parameters(*th)
    sv.synchronize()
    t_plain = time.perf_counter()
    sv.step(scn.dt, args.steps)
    sv.synchronize()
    t_plain = time.perf_counter() - t_plain
    # central differences (h = 1e-6, relative: theta +- h * theta * N(0,1))
    # along a random direction in each parameter group, then in all groups
    # at once (the groups' contributions partly cancel there, so that check
    # sits closer to the differences' rounding floor)
    checks = []
    names = ["secretion", "uptake", "D", "decay"]
    for group in [0, 1, 2, 3, None]:
        v = [x * rng.standard_normal(x.shape) if group in (None, j) else np.zeros_like(x)
             for j, x in enumerate(th)]
        h = 1e-6
        pp = prob.run(*[a + h * b for a, b in zip(th, v)])
        pm = prob.run(*[a - h * b for a, b in zip(th, v)])
        fd = loss_difference(pp, pm, target) / (2 * h)
        adj = sum(float(np.sum(g[nm] * vj)) for nm, vj in zip(names, v))
        checks.append({"direction": names[group] if group is not None else "all",
                       "fd": fd, "adjoint": adj, "rel_diff": abs(adj - fd) / abs(fd)})
    prob.close()
    if rank == 0:
        vs = scn.num_voxels * S * args.steps
        line = {
            "metric": METRIC + " (adjoint: forward with checkpoints + backward)",
            "value": vs * world / (t_fwd + t_bwd), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": 1, "ms_per_step": 1e3 * (t_fwd + t_bwd) / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": f"adjoint: {n}^3 x {S} FP64, {A} agents, {args.steps} steps, "
                                   f"checkpoints every {k}", "loss": "1/2 |p_T - target|^2"},
            "forward_seconds": t_fwd, "backward_seconds": t_bwd,
            "plain_forward_seconds": t_plain, "backward_over_forward": t_bwd / t_plain,
            "gradient_vs_central_differences": checks,
            "max_rel_diff_per_group": max(c["rel_diff"] for c in checks
                                          if c["direction"] != "all"),
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="lod256: skip the brief 50^3 and batched measurements")
    ap.add_argument("--row-build", type=int, choices=[0, 1, 2], default=None,
                    help="lod256: x row-kernel build after tuning (0 any density count, "
                         "1 built for this density count, 2 the same with planar tables)")
    ap.add_argument("--sweep-chunks", default=None,
                    help="lod256: chunk lengths of the x, y and z sweeps after tuning, "
                         "e.g. 32,32,16")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default kernel per axis (for profiler launch lists)")
    ap.add_argument("--size", type=int, default=256, help="cube edge in voxels (default 256)")
    ap.add_argument("--substrates", type=int, default=10)
    ap.add_argument("--agents", type=int, default=100_000)
    ap.add_argument("--workload",
                    choices=["lod256", "plain50", "batched", "fp32", "adjoint", "gradients",
                             "lod2d"],
                    default="lod256",
                    help="lod256: the headline line (default); batched: 64 independent "
                         "instances vs looped plain solves; fp32: FP32 sweeps at 512^3 x 8 "
                         "with 1M agents against FP64; adjoint: gradients at 128^3 x 4, 200 "
                         "steps; plain50: the 50^3 launch-bound case, host-launched vs graph; "
                         "gradients: compute_all_gradient_vectors at 256^3 x 10; lod2d: the "
                         "LOD_2D solver on a 1024^2 x 32 plane")
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--shard", choices=["instances", "substrates"], default="instances",
                    help="lod256 on N GPUs: independent microenvironments per rank (weak "
                         "scaling, the default) or one microenvironment split by substrate "
                         "(strong scaling)")
    ap.add_argument("--batch-trial-steps", type=int, default=10,
                    help="steps per trial run of the batch tuner")
    ap.add_argument("--batch-modes", action="store_true",
                    help="batched: also time every batch mode with the tuned group budget")
    ap.add_argument("--batch-mode", choices=["tuned", "fused", "branches", "persistent", "planes"],
                    default="tuned", help="batched: the tuner's choice, or one mode untuned")
    ap.add_argument("--batch-chunk", type=int, default=8,
                    help="batched, persistent mode untuned: 4, 8, 16, 32 or 0 (whole lines)")
    args = ap.parse_args()
    if args.workload == "batched" and "--steps" not in sys.argv:
        args.steps = 200
    if args.workload == "fp32" and "--steps" not in sys.argv:
        args.steps = 50
    if args.workload == "adjoint" and "--steps" not in sys.argv:
        args.steps = 200
    if args.workload == "plain50" and "--steps" not in sys.argv:
        args.steps = 100
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    world, rank, local = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference_arm(args, world, rank)
        elif args.workload == "batched":
            run_batched(args, world, rank, local)
        elif args.workload == "fp32":
            run_fp32(args, world, rank, local)
        elif args.workload == "adjoint":
            run_adjoint(args, world, rank, local)
        elif args.workload == "lod2d":
            run_lod2d(args, world, rank, local)
        elif args.workload == "gradients":
            run_gradients(args, world, rank, local)
        elif args.workload == "plain50":
            run_plain50(args, world, rank, local)
        elif args.shard == "substrates":
            run_sharded(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        import torch.distributed as dist

        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
