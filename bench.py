#!/usr/bin/env python
"""Benchmark of the B200 simulation core on the 100k-neuron workload.

Workload (one bench step): a 1000 ms trial (10,000 steps at dt 0.1 ms) of the
100,000-neuron random K=100 Izhikevich network (80% RS / 20% FS, positions
U(-500,500)^3 um, delay = distance / 100 um/ms capped at 20 ms, |w| exc
U(0,0.5), inh U(0,1), x0.7, Dale's law), tau_syn 5 ms, Gaussian current noise
sd 1, fixed-point (int32, scale 4096) delay ring, reset to the initial state
at the start of every trial.  Inputs (the ~10M-synapse CSR, ~130 MB with the
ring) exceed the 126 MB L2, and L2 is also scrubbed between timed steps.

Prints ONE JSON line (rank 0).  `value` is neuron-updates/s timed with CUDA
events on the engine's stream; `e2e` is the same trial through the public C
ABI with the host<->device copies in the timed region; `roofline` relates the
step kernel's algorithmic bytes to the measured HBM peak; `cpu_baseline` is
the C restatement of the reference CPU step (single thread, as the reference
CpuSim) on a bounded sample of the same workload.

`--impl reference` times that CPU restatement (the reference is Rust and
cannot be built in this image) on the same workload and prints its line.
With torchrun (N > 1) every rank runs an independent replica (replicas only:
the path has no exchange step); value = all ranks' neuron-updates / max time.
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 100_000
K_OUT = 100
TRIAL_STEPS = 10_000  # 1000 ms at dt 0.1
SEED = 1
B_NEURON = 60  # algorithmic bytes per Izhikevich neuron-update
B_SPIKE = 24   # per spike
B_EVENT = 17   # per delivered synaptic event
ACTIVE_KICK_HZ = 100.0  # companion regime: Poisson kicks (sim/src/state.rs:15-22), ~22 Hz firing
ADEX_ACTIVE_KICK_HZ = 60.0  # the AdEx variant's kicks for ~20 Hz firing
LIQUID_KICK_HZ = 30.0  # the batched liquids' active variant: ~20 Hz firing
L2_NOTE = ("L2 scrubbed (256 MB write) before each timed trial; a trial is 10,000 dependent steps whose "
           "per-step working set (state ~7 MB + one ring slot) stays in L2 from step to step, as in any run of "
           "this net; the CSR (~90 MB) and ring (~67 MB) together exceed L2")


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured hbm_gbs (MEASURED_PEAKS.json)"
    return 6650.0, "fallback: MEASURED_PEAKS.json absent, the pool's earlier copy-bandwidth measurement"


def load_traffic():
    """DRAM bytes per launch of the headline's step kernel from a stored ncu
    capture (profiles/step_kernel_traffic.json): not measured in this run."""
    p = os.path.join(ROOT, "profiles", "step_kernel_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def headline_config(ring_depth: int, ws: int) -> dict:
    """The workload both arms measure (identical dict in both lines)."""
    return {"workload": "100k izh random K=100, 1000 ms trial at dt 0.1 ms from reset, Gaussian noise sd 1, "
                        "tau_syn 5 ms, int32 ring",
            "neurons": N, "synapses": N * K_OUT, "trial_steps": TRIAL_STEPS, "ring_depth": ring_depth,
            "l2": L2_NOTE, "parallelism": f"replicas x{ws}"}


class Clocks:
    """SM clocks and throttle reasons sampled during the timed region: an
    NVML thread polling every 10 ms (read-only queries), or nvidia-smi at
    200 ms where NVML is not available."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits: sw power cap, hw slowdown, sw thermal, hw thermal
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                   "hw_thermal_slowdown": 0x40}

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.rows = []
        self.thread = None
        import tempfile

        self.path = os.path.join(tempfile.gettempdir(), f"ne2b_clocks_{os.getpid()}.csv")

    def _nvml_handle(self):
        import pynvml

        pynvml.nvmlInit()
        try:
            import torch

            p = torch.cuda.get_device_properties(self.device)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def __enter__(self):
        import threading

        try:
            nv, h = self._nvml_handle()
            self.stop = threading.Event()
            smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)

            def poll():
                while not self.stop.is_set():
                    try:
                        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                        reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.rows.append((float(sm), float(smax), reasons))
                    except Exception:
                        pass
                    self.stop.wait(0.01)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        rows = []
        if self.thread:
            for sm, smax, bits in self.rows:
                rows.append((sm, smax, [k for k, b in self.REASON_BITS.items() if bits & b]))
            source = "nvml 10 ms"
        elif self.proc and os.path.exists(self.path):
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) < 9:
                        continue
                    try:
                        rows.append((float(parts[1]), float(parts[2]),
                                     [names[k] for k in range(4) if parts[5 + k].lower().startswith("active")]))
                    except ValueError:
                        continue
            source = "nvidia-smi 200 ms"
        if not rows:
            return None
        reasons = sorted({r for _, _, rs in rows for r in rs})
        load = [r[0] for r in rows if r[0] > 300] or [r[0] for r in rows]
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows), "source": source}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def _reduce(x: float, ws: int, op: str) -> float:
    """All-reduce one float over the replicas (NCCL on the GPUs, or the CPU
    tensors of a gloo group)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float, ws: int) -> float:
    return _reduce(x, ws, "max")


def sum_over_ranks(x: float, ws: int) -> float:
    return _reduce(x, ws, "sum")


def replica_aggregate(local_ms: float, local_units: float, ws: int) -> tuple[float, float, float]:
    """Weak-scaling aggregate of independent replicas: the slowest rank's
    device time, the units all ranks processed, and units per second over
    that time."""
    ms = max_over_ranks(local_ms, ws)
    units = sum_over_ranks(local_units, ws)
    return ms, units, units / (ms / 1000.0)


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def make_cfg(nb, active: bool, adex: bool = False):
    kick = (ADEX_ACTIVE_KICK_HZ if adex else ACTIVE_KICK_HZ) if active else 0.0
    return nb.default_config(int_weights=1, gauss_sd=1.0, synapse_tau_ms=5.0, noise_rate_hz=kick,
                             noise_kick_mv=20.0, seed=SEED)


def timed_trials(sim, steps: int, warmup: int, trial_steps: int, ws: int, torch, scrub):
    """Run warmup + steps trials; return (total device ms, spikes, launches)."""
    stream = torch.cuda.ExternalStream(sim.stream_handle())
    for _ in range(warmup):
        sim.reset_state()
        sim.run_steps(trial_steps)
    sim.synchronize()
    total_ms = 0.0
    spikes = 0
    launches0 = sim.kernel_launches()
    for _ in range(steps):
        with torch.cuda.stream(stream):
            scrub.fill_(1)  # L2 flush: 256 MB write, outside the timed interval
        barrier(ws)
        sim.synchronize()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("timed")  # lets a profiler select the timed launches
        e0.record(stream)
        sim.reset_state()
        sim.run_steps(trial_steps)
        e1.record(stream)
        torch.cuda.nvtx.range_pop()
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        spikes += sim.spikes_total()
    launches = sim.kernel_launches() - launches0
    return total_ms, spikes, launches


def run_profile(args):
    """Short run for ncu: 3 warm-up trials + 1 trial of --trial-steps steps."""
    import torch

    import neuro_edit_v2_b200 as nb

    if args.served_mix:
        return run_profile_served(args, nb, torch)
    if args.batched_liquids:
        return run_profile_batched(args, nb, torch)
    net = nb.random_kout(args.profile_neurons, K_OUT, SEED, w_scale=0.7 * (281.0 if args.adex else 1.0))
    if args.adex:  # the AdEx variant of the 1M workload (weights x C = 281 pF)
        nb.to_adex(net)
    sim = nb.B200Sim(net, make_cfg(nb, args.active, args.adex))
    if args.kernel:
        sim.set_kernel_mode({"stream": nb.KERNEL_STREAM, "resident": nb.KERNEL_RESIDENT}[args.kernel])
    if args.shape:
        b, npt = (int(x) for x in args.shape.split("x"))
        sim.set_tile_shape(b, npt)
    if args.delivery_warps:
        sim.set_delivery_warps(True)
    tiling = sim.autotune(128) if args.autotune else sim.tiling()
    scrub = torch.empty(256 << 20, dtype=torch.uint8, device="cuda:0")
    ms, spikes, launches = timed_trials(sim, 1, 3, args.trial_steps, 1, torch, scrub)
    print(json.dumps({"profile_run": True, "neurons": args.profile_neurons, "trial_steps": args.trial_steps,
                      "ms": ms, "spikes": spikes, "launches": launches, "tiling": tiling}), flush=True)


def run_profile_batched(args, nb, torch):
    """The first --batched-liquids liquids of the batched workload (with
    their input streams, or none with --no-inputs) stepped as one batch:
    3 warm-up trials + 1 trial of --trial-steps steps, for ncu."""
    from concurrent.futures import ThreadPoolExecutor

    from neuro_edit_v2_b200 import workloads as W

    count = args.batched_liquids
    sides = W.batched_liquid_sizes(256, 4)[:count]
    n_inputs = 0 if args.no_inputs else 8
    with ThreadPoolExecutor(8) as ex:
        nets = list(ex.map(lambda k: nb.liquid(sides[k], seed=1000 + k, n_inputs=n_inputs), range(count)))
    cfgs = [nb.default_config(int_weights=1, window_steps=W.WINDOW_STEPS, max_windows=20, seed=k) for k in range(count)]
    b = nb.Batch(nets, cfgs)
    if n_inputs:
        rng = np.random.default_rng(5)
        for k in range(count):
            b.set_input_matrix(k, W.bit_streams(rng, 1000))
    if args.kernel:
        b.set_kernel_mode({"stream": nb.KERNEL_STREAM, "resident": nb.KERNEL_RESIDENT}[args.kernel])
    if args.shape:
        bl, npt = (int(x) for x in args.shape.split("x"))
        b.set_tile_shape(bl, npt)
    stream = torch.cuda.ExternalStream(b.stream_handle())
    for _ in range(3):
        b.reset_state()
        b.run_steps(args.trial_steps)
    b.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    b.reset_state()
    e0.record(stream)
    b.run_steps(args.trial_steps)
    e1.record(stream)
    e1.synchronize()
    print(json.dumps({"profile_run": True, "batched_liquids": count, "inputs": n_inputs, "neurons": sum(n.n for n in nets),
                      "trial_steps": args.trial_steps, "ms": e0.elapsed_time(e1),
                      "spikes": sum(b.spikes_total(k) for k in range(count)), "tile_shape": b.tile_shape()}),
          flush=True)


def run_profile_served(args, nb, torch):
    """The first --served-mix requests of the serving stream stepped together
    in one batch (the serving kernels without the admission loop): 3 warm-up
    trials + 1 trial of --trial-steps steps, for ncu."""
    from neuro_edit_v2_b200 import workloads as W

    reqs = W.request_stream(args.served_mix)
    b = nb.Batch([q.net for q in reqs], [W.request_config(q, 11 + k) for k, q in enumerate(reqs)])
    for k, q in enumerate(reqs):
        b.set_input_matrix(k, q.inputs)
    if args.kernel:
        b.set_kernel_mode({"stream": nb.KERNEL_STREAM, "resident": nb.KERNEL_RESIDENT}[args.kernel])
    if args.shape:
        bl, npt = (int(x) for x in args.shape.split("x"))
        b.set_tile_shape(bl, npt)
    stream = torch.cuda.ExternalStream(b.stream_handle())
    for _ in range(3):
        b.reset_state()
        b.run_steps(args.trial_steps)
    b.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.reset_state()
    b.run_steps(args.trial_steps)
    e1.record(stream)
    e1.synchronize()
    spikes = sum(b.spikes_total(k) for k in range(len(reqs)))
    print(json.dumps({"profile_run": True, "served_mix": args.served_mix, "neurons": sum(q.n for q in reqs),
                      "trial_steps": args.trial_steps, "ms": e0.elapsed_time(e1), "spikes": spikes,
                      "tile_shape": b.tile_shape()}), flush=True)


def run_ours(args):
    ws, rank, local = dist_setup()
    import numpy as np
    import torch

    import neuro_edit_v2_b200 as nb

    torch.cuda.set_device(local)
    dev = local
    net = nb.random_kout(N, K_OUT, SEED + rank)
    sim = nb.B200Sim(net, make_cfg(nb, False), device=dev)

    def tune(s):
        if args.shape and args.kernel:
            s.set_kernel_mode({"stream": nb.KERNEL_STREAM, "resident": nb.KERNEL_RESIDENT}[args.kernel])
            b, npt = (int(x) for x in args.shape.split("x"))
            s.set_tile_shape(b, npt)
            return s.tiling()
        return s.autotune(256)

    tiling = tune(sim)
    scrub = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")

    with Clocks(dev) as clk:
        total_ms, spikes, launches = timed_trials(sim, args.steps, args.warmup, TRIAL_STEPS, ws, torch, scrub)
    n_updates = float(N) * TRIAL_STEPS * args.steps
    total_ms, _, value = replica_aggregate(total_ms, n_updates, ws)
    events = spikes * K_OUT
    step_launches = TRIAL_STEPS * args.steps
    launch_ms = total_ms / step_launches
    alg_bytes = B_NEURON * N + B_SPIKE * spikes / step_launches + B_EVENT * events / step_launches
    peak, peak_kind = load_peaks()
    achieved = alg_bytes / (launch_ms / 1000.0) / 1e9
    tr = load_traffic()

    # active companion regime (same net, Poisson kicks on top)
    act = nb.B200Sim(net, make_cfg(nb, True), device=dev)
    a_tiling = tune(act)
    a_ms, a_spikes, _ = timed_trials(act, max(1, args.steps // 2), 1, TRIAL_STEPS, ws, torch, scrub)
    a_ms = max_over_ranks(a_ms, ws)
    a_trials = max(1, args.steps // 2)
    a_events = a_spikes * K_OUT
    a_alg = B_NEURON * N + (B_SPIKE * a_spikes + B_EVENT * a_events) / (TRIAL_STEPS * a_trials)
    del act

    # end to end through the public API: pinned host drive in, v out
    ext = torch.zeros(N, dtype=torch.float32).pin_memory().numpy()
    e2e_steps = args.steps
    sim.synchronize()
    barrier(ws)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sim.set_external_all(ext)
        sim.reset_state()
        sim.run_steps(TRIAL_STEPS)
        v = sim.v()
        tot = sim.spikes_total()
    e2e_s = max_over_ranks(time.perf_counter() - t0, ws)
    e2e_val = sum_over_ranks(n_updates / args.steps * e2e_steps, ws) / e2e_s
    del v, tot

    extra = {}
    if not args.no_extras and ws == 1:
        peak_v, _ = load_peaks()
        jobs = (("c10k", lambda: bench_10k(nb, torch, scrub, args.steps, peak_v)),
                ("c1m_izh", lambda: bench_1m(nb, torch, scrub, nb.MODEL_IZH, 2, 3, peak_v)),
                ("c1m_adex", lambda: bench_1m(nb, torch, scrub, nb.MODEL_ADEX, 2, 3, peak_v)),
                ("fp32_ring_100k", lambda: bench_fp32_ring(nb, torch, scrub, net, args.steps, peak_v)),
                ("batched_256", lambda: bench_batched(nb, torch, scrub, 2, 3)),
                ("batched_256_active", lambda: bench_batched(nb, torch, scrub, 2, 3, kick_hz=LIQUID_KICK_HZ)),
                ("serving", lambda: bench_serving(nb, args.serving_requests, args.admission_threads)))
        only = set(args.extras.split(",")) if args.extras else None
        for name, fn in jobs:
            if only is not None and name not in only:
                continue
            try:
                extra[name] = fn()
            except Exception as e:  # report, never hide
                extra[name] = {"error": repr(e)}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(TRIAL_STEPS)

    line = {
        "metric": "neuron-updates/s (synaptic events/s reported beside)",
        "value": value,
        "unit": "neuron-updates/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 state, int32 fixed-point ring",
        "data": "synthetic: seeded generator of the 100k configuration (random K=100, distance delays)",
        "config": headline_config(sim.ring_depth(), ws),
        "synaptic_events_per_s": events / (total_ms / 1000.0) * ws,
        "firing_rate_hz": spikes / (N * args.steps * TRIAL_STEPS * 1e-4),
        "active_regime": {
            "what": f"same net + Poisson kicks {ACTIVE_KICK_HZ:g} Hz x 20 mV",
            "neuron_updates_per_s": float(N) * TRIAL_STEPS * a_trials / (a_ms / 1000.0) * ws,
            "synaptic_events_per_s": a_events / (a_ms / 1000.0) * ws,
            "firing_rate_hz": a_spikes / (N * a_trials * TRIAL_STEPS * 1e-4),
            "ms_per_trial": a_ms / a_trials,
            "roofline_frac": a_alg / (a_ms / (TRIAL_STEPS * a_trials) / 1000.0) / 1e9 / peak,
            "tiling": a_tiling,
        },
        "tiling": tiling,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind,
                     "alg_bytes_per_launch": alg_bytes, "launch_us": launch_ms * 1000.0,
                     "traffic": (tr or {}).get("bytes_per_launch"),
                     "traffic_kind": "stored ncu capture of this kernel and workload, not measured in this run",
                     "traffic_source": (tr or {}).get("source")},
        "e2e": {"value": e2e_val, "unit": "neuron-updates/s", "h2d_bytes_per_step": 4 * N,
                "d2h_bytes_per_step": 4 * N + 8},
        "gpu_launches": launches,
        "cpu_baseline": cpu,
        "extra": extra,
    }
    line["clocks"] = clk.summary()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# ----------------------------------------------------------------- extras
def bench_1m(nb, torch, scrub, model: int, steps: int, warmup: int, peak: float):
    """1,000,000 neurons x K=100 (~100M synapses), 500 ms trials, izh or AdEx
    (AdEx weights x C = 281 pF so a weight moves v by the same mV): the
    configuration as stated (Gaussian noise sd 1, silent), then the same sim
    in an active regime (Poisson kicks x 20 mV added: ~20 Hz, ~2e5 synaptic
    events per step into the HBM-resident ring)."""
    n, trial = 1_000_000, 5000
    adex = model == nb.MODEL_ADEX
    net = nb.random_kout(n, K_OUT, SEED, w_scale=0.7 * (281.0 if adex else 1.0))
    if adex:
        nb.to_adex(net)
    sim = nb.B200Sim(net, nb.default_config(int_weights=1, gauss_sd=1.0, synapse_tau_ms=5.0, seed=SEED))
    del net
    b_neuron = 84 if adex else B_NEURON

    def measure(kick_hz):
        sim.set_noise(kick_hz, 20.0 if kick_hz else 0.0)
        # tune on a state inside the regime (half a trial from reset), not on
        # the state the previous regime left
        sim.reset_state()
        sim.run_steps(trial // 2)
        tiling = sim.autotune(128)
        ms, spikes, launches = timed_trials(sim, steps, warmup, trial, 1, torch, scrub)
        per_launch_s = ms / 1000.0 / (trial * steps)
        events = spikes * K_OUT
        alg = b_neuron * n + (B_SPIKE * spikes + B_EVENT * events) / (trial * steps)
        achieved = alg / per_launch_s / 1e9
        return {"kick_hz": kick_hz, "neuron_updates_per_s": n * trial * steps / (ms / 1000.0),
                "synaptic_events_per_s": events / (ms / 1000.0),
                "firing_rate_hz": spikes / (n * steps * trial * 1e-4), "ms_per_trial": ms / steps,
                "events_per_step": events / (trial * steps),
                "roofline": {"achieved_gbs": achieved, "frac": achieved / peak, "alg_bytes_per_launch": alg,
                             "launch_us": per_launch_s * 1e6, "bytes_per_neuron": b_neuron,
                             "target_frac": 0.6},
                "gpu_launches": launches, "tiling": tiling}

    out = {"neurons": n, "synapses": n * K_OUT, "trial_steps": trial, "ring_depth": sim.ring_depth(),
           "dev_mem_bytes": sim.dev_mem_bytes()}
    out["quiet"] = measure(0.0)
    out["active"] = measure(ADEX_ACTIVE_KICK_HZ if adex else ACTIVE_KICK_HZ)
    sim.close()
    return out


def bench_10k(nb, torch, scrub, steps: int, peak: float):
    """The 10,000-neuron configuration (same generator, K=100, 1000 ms trials
    from reset, Gaussian noise sd 1, tau_syn 5 ms) in both ring modes, as
    configured (silent) and with Poisson kicks 100 Hz x 20 mV; the
    autotuner picks the kernel (the resident one fits at this size)."""
    n = 10_000
    net = nb.random_kout(n, K_OUT, SEED)
    out = {"neurons": n, "synapses": n * K_OUT, "trial_steps": TRIAL_STEPS}
    for ring, iw in (("int32", 1), ("f32", 0)):
        for name, kick in (("quiet", 0.0), ("active", ACTIVE_KICK_HZ)):
            sim = nb.B200Sim(net, nb.default_config(int_weights=iw, gauss_sd=1.0, synapse_tau_ms=5.0,
                                                    noise_rate_hz=kick, noise_kick_mv=20.0, seed=SEED))
            tiling = sim.autotune(256)
            ms, spikes, launches = timed_trials(sim, steps, 3, TRIAL_STEPS, 1, torch, scrub)
            events = spikes * K_OUT
            step_s = ms / 1000.0 / (TRIAL_STEPS * steps)
            alg = B_NEURON * n + (B_SPIKE * spikes + B_EVENT * events) / (TRIAL_STEPS * steps)
            out[f"{ring}_{name}"] = {"kick_hz": kick, "neuron_updates_per_s": n * TRIAL_STEPS * steps / (ms / 1000.0),
                                     "synaptic_events_per_s": events / (ms / 1000.0),
                                     "firing_rate_hz": spikes / (n * steps * TRIAL_STEPS * 1e-4),
                                     "ms_per_trial": ms / steps, "step_us": step_s * 1e6,
                                     "roofline_frac": alg / step_s / 1e9 / peak, "gpu_launches": launches,
                                     "tiling": tiling}
            sim.close()
    return out


def bench_fp32_ring(nb, torch, scrub, net, steps: int, peak: float):
    """The 100k configuration with the f32 ring (float atomics), quiet as
    stated and in the active regime: the fp32-ring mode of the benchmark
    configurations, beside the int32 headline."""
    out = {}
    for name, kick in (("quiet", 0.0), ("active", ACTIVE_KICK_HZ)):
        sim = nb.B200Sim(net, nb.default_config(int_weights=0, gauss_sd=1.0, synapse_tau_ms=5.0,
                                                noise_rate_hz=kick, noise_kick_mv=20.0, seed=SEED))
        tiling = sim.autotune(256)
        k = max(1, steps // 2) if kick else steps
        ms, spikes, launches = timed_trials(sim, k, 3, TRIAL_STEPS, 1, torch, scrub)
        events = spikes * K_OUT
        alg = B_NEURON * N + (B_SPIKE * spikes + B_EVENT * events) / (TRIAL_STEPS * k)
        step_s = ms / 1000.0 / (TRIAL_STEPS * k)
        out[name] = {"kick_hz": kick, "neuron_updates_per_s": N * TRIAL_STEPS * k / (ms / 1000.0),
                     "synaptic_events_per_s": events / (ms / 1000.0),
                     "firing_rate_hz": spikes / (N * k * TRIAL_STEPS * 1e-4), "ms_per_trial": ms / k,
                     "roofline_frac": alg / step_s / 1e9 / peak, "gpu_launches": launches, "tiling": tiling}
        sim.close()
    return out


def batch_trials(b, torch, scrub, steps: int, warmup: int, trial: int):
    stream = torch.cuda.ExternalStream(b.stream_handle())
    for _ in range(warmup):
        b.reset_state()
        b.run_steps(trial)
    b.synchronize()
    total = 0.0
    for _ in range(steps):
        with torch.cuda.stream(stream):
            scrub.fill_(1)
        b.synchronize()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.reset_state()
        b.run_steps(trial)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    return total


_LIQUIDS = None


def bench_batched(nb, torch, scrub, steps: int, warmup: int, serial_sample: int = 32, kick_hz: float = 0.0):
    """256 liquids with their input streams, one batch, 1000 ms trials, against
    the same kernels one net at a time on a sample of 32 nets spread over the
    size range; `kick_hz` > 0 adds Poisson kicks x 20 mV (the active variant)."""
    global _LIQUIDS
    from neuro_edit_v2_b200 import workloads as W

    if _LIQUIDS is None:
        _LIQUIDS = W.batched_liquids(256)
    nets, inputs = _LIQUIDS
    trial = TRIAL_STEPS
    wins = trial // W.WINDOW_STEPS
    cfgs = [nb.default_config(int_weights=1, window_steps=W.WINDOW_STEPS, max_windows=wins, seed=k,
                              noise_rate_hz=kick_hz, noise_kick_mv=20.0 if kick_hz else 0.0)
            for k in range(len(nets))]
    b = nb.Batch(nets, cfgs)
    for k, x in enumerate(inputs):
        b.set_input_matrix(k, x)
    shape = b.autotune(128)
    total_ms = batch_trials(b, torch, scrub, steps, warmup, trial)
    neurons = sum(n.n for n in nets)
    events = 0
    spikes = 0
    for k, net in enumerate(nets):
        deg = W.outdegree(net)
        for w in range(wins):
            c = b.window_counts(k, w).astype(np.int64)
            spikes += int(c.sum())
            events += int((c * deg).sum())
    launches = b.kernel_launches()
    b.close()
    # the same kernels, one network at a time (each autotuned, as the batch
    # is), on a sample of the set: every 8th net, so the sample spans the size
    # range (the nets are in a seeded random size order)
    sample = list(range(0, len(nets), max(1, len(nets) // serial_sample)))[:serial_sample]
    ser_ms = 0.0
    for k in sample:
        one = nb.Batch([nets[k]], [cfgs[k]])
        one.set_input_matrix(0, inputs[k])
        one.autotune(128)  # each net on its own best kernel and tiles, as the batch is
        ser_ms += batch_trials(one, torch, scrub, 1, 1, trial)
        one.close()
    batched_tps = len(nets) * steps / (total_ms / 1000.0)
    serial_tps = len(sample) / (ser_ms / 1000.0)
    sample_neurons = sum(nets[k].n for k in sample) / len(sample)
    # the same byte contract as the single net (all liquids are izh): the
    # per-step bytes over the per-step time of the timed trials
    peak, peak_kind = load_peaks()
    step_s = total_ms / 1000.0 / (steps * trial)
    alg = B_NEURON * neurons + (B_SPIKE * spikes + B_EVENT * events) / trial
    achieved = alg / step_s / 1e9
    return {"nets": len(nets), "neurons": neurons, "synapses": sum(n.n_syn for n in nets), "trial_steps": trial,
            "roofline": {"achieved_gbs": achieved, "frac": achieved / peak, "peak": peak,
                         "peak_kind": peak_kind, "alg_bytes_per_step": alg, "step_us": step_s * 1e6,
                         "bytes_per_neuron": B_NEURON},
            "windows_per_trial": wins, "tile_shape": {"block": shape[0], "neurons_per_thread": shape[1],
                                                      "blocks_per_sm": shape[2]},
            "trials_per_s": batched_tps, "ms_per_batch_trial": total_ms / steps,
            "neuron_updates_per_s": neurons * trial * steps / (total_ms / 1000.0),
            "synaptic_events_per_s": events / (total_ms / 1000.0 / steps),
            "firing_rate_hz": spikes / (neurons * trial * 1e-4),
            "kick_hz": kick_hz, "serial_trials_per_s": serial_tps, "serial_sample": len(sample),
            "serial_sample_mean_neurons": sample_neurons, "batch_mean_neurons": neurons / len(nets),
            "batched_vs_serial": batched_tps / serial_tps}


def bench_serving(nb, count: int, threads: int = 4):
    from neuro_edit_v2_b200 import workloads as W

    reqs = W.request_stream(count)
    outdeg = [W.outdegree(q.net) for q in reqs]

    def serve(arrivals):
        count = len(arrivals)
        srv = nb.Server(neuron_capacity=16 << 20, synapse_capacity=1 << 30, ring_capacity=6 << 30,
                        max_requests=512, steps_per_launch=100, admission_threads=threads)
        order = sorted(range(count), key=lambda r: arrivals[r])
        lat = [0.0] * count
        ids = {}
        nxt = 0
        done = 0
        refused = 0
        results = {}
        tm = {"admit_s": 0.0, "step_s": 0.0, "take_s": 0.0}
        t0 = time.perf_counter()
        while done < count:
            now = time.perf_counter() - t0
            budget = time.perf_counter() + 0.002  # admit for <= 2 ms, then keep the device fed
            while nxt < count and arrivals[order[nxt]] <= now:
                if time.perf_counter() > budget and srv.stats()["active"] > 0:
                    break
                r = order[nxt]
                ta = time.perf_counter()
                rid = srv.submit(reqs[r].net, W.request_config(reqs[r], 11 + r), reqs[r].inputs, reqs[r].steps)
                tm["admit_s"] += time.perf_counter() - ta
                if rid is None:
                    refused += 1
                    break
                ids[rid] = r
                nxt += 1
            if srv.stats()["active"] == 0:
                srv.synchronize()
            else:
                ts = time.perf_counter()
                srv.step()
                tm["step_s"] += time.perf_counter() - ts
            # results whose retiring launch has completed: taking them never
            # waits for the device
            tt = time.perf_counter()
            for rid in srv.finished():
                counts, tot = srv.take(rid)
                r = ids[rid]
                results[r] = (counts, tot)
                lat[r] = time.perf_counter() - t0 - arrivals[r]
                done += 1
            tm["take_s"] += time.perf_counter() - tt
            if srv.stats()["active"] == 0 and nxt < count and done == nxt:
                time.sleep(max(0.0, arrivals[order[nxt]] - (time.perf_counter() - t0)))
        span = time.perf_counter() - t0
        srv.close()
        tm["span_s"] = span
        serve.timing = tm
        serve.spikes = sum(tot for _, tot in results.values())
        serve.events = sum(int((c.astype(np.int64).sum(axis=0) * outdeg[r]).sum()) for r, (c, _) in results.items())
        return lat, span, refused

    arrivals = [q.arrival_s for q in reqs]
    # untimed warm-up: the first server of a process pays one-time costs
    # (pinned staging, memory pool growth, module loading) that halved the
    # throughput of whichever run came first
    serve([0.0] * min(48, count))
    lat, span, refused = serve(arrivals)
    t_poisson = dict(serve.timing)
    sat_lat, sat_span, _ = serve([0.0] * count)
    t_sat = dict(serve.timing)
    sat_spikes, sat_events = serve.spikes, serve.events
    # one at a time: the same server and kernels, each request admitted only
    # after the previous one finished (sample of the stream)
    sample = min(24, count)
    srv = nb.Server(neuron_capacity=16 << 20, synapse_capacity=1 << 30, ring_capacity=6 << 30, max_requests=1,
                    steps_per_launch=100, admission_threads=threads)
    t0 = time.perf_counter()
    for r in range(sample):
        rid = srv.submit(reqs[r].net, W.request_config(reqs[r], 11 + r), reqs[r].inputs, reqs[r].steps)
        while srv.stats()["active"]:
            srv.step()
        srv.take(rid)
    srv.close()
    one_tps = sample / (time.perf_counter() - t0)
    # one at a time, each request on its own engine with the kernel and tiles
    # the autotuner picks for it alone (the tuning itself untimed): building
    # it, running it from reset and reading its counts back
    tuned_sample = min(12, count)
    tuned_s = 0.0
    for r in range(tuned_sample):
        t1 = time.perf_counter()
        one = nb.Batch([reqs[r].net], [W.request_config(reqs[r], 11 + r)])
        one.set_input_matrix(0, reqs[r].inputs)
        t2 = time.perf_counter()
        one.autotune(128)
        one.reset_state()
        one.synchronize()
        t3 = time.perf_counter()
        one.run_steps(reqs[r].steps)
        one.window_counts(0, 0)
        one.synchronize()
        tuned_s += (t2 - t1) + (time.perf_counter() - t3)
        one.close()
    tuned_tps = tuned_sample / tuned_s
    q = np.quantile(np.array(lat), [0.5, 0.99])
    sq = np.quantile(np.array(sat_lat), [0.5, 0.99])
    neuron_steps = sum(q_.n * q_.steps for q_ in reqs)
    return {"requests": count, "admission_threads": threads, "offered_rate_hz": 200.0,
            "trials_per_s": count / span, "p50_ms": q[0] * 1e3,
            "p99_ms": q[1] * 1e3, "refused_admissions": refused,
            "saturated": {"trials_per_s": count / sat_span, "p50_ms": sq[0] * 1e3, "p99_ms": sq[1] * 1e3,
                          "neuron_updates_per_s": neuron_steps / sat_span,
                          "synaptic_events_per_s": sat_events / sat_span,
                          "firing_rate_hz": sat_spikes / (neuron_steps * 1e-4), "host_time": t_sat},
            "host_time": t_poisson,
            "one_at_a_time_trials_per_s": one_tps, "one_at_a_time_sample": sample,
            "served_vs_one_at_a_time": (count / span) / one_tps,
            "saturated_vs_one_at_a_time": (count / sat_span) / one_tps,
            "one_at_a_time_tuned": {"trials_per_s": tuned_tps, "sample": tuned_sample,
                                    "served_vs": (count / span) / tuned_tps,
                                    "saturated_vs": (count / sat_span) / tuned_tps},
            "mean_neurons": float(np.mean([q_.n for q_ in reqs])),
            "mean_steps": float(np.mean([q_.steps for q_ in reqs]))}


def cpu_baseline_sample(sample_steps: int):
    """The C restatement of the reference CPU step (single thread) on the
    same 100k net and config, `sample_steps` steps of the trial."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O

    onet = O.ONet.random_kout(N, K_OUT, SEED)
    sim = O.OSim(onet, O.cfg(int_weights=1, gauss_sd=1.0, synapse_tau_ms=5.0, seed=SEED))
    t0 = time.perf_counter()
    sim.run_steps(sample_steps)
    dt = time.perf_counter() - t0
    return {"value": N * sample_steps / dt, "unit": "neuron-updates/s", "cores": 1, "kind": "port",
            "sample": f"100k net, first {sample_steps} steps ({sample_steps / 10:g} ms) of the trial, "
                      f"{dt:.1f} s on 1 host core (the reference CpuSim is single-threaded)",
            "cpu": cpu_model()}


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip() + f" ({os.cpu_count()} cores visible)"
    except OSError:
        pass
    return "unknown"


REF_SAMPLE = 500  # reference arm: steps of the trial per bench step (its first 50 ms, from reset)
REF_MAX_COPIES = 64  # one 100k oracle net (~130 MB) per copy


def _reference_copy(steps: int, warmup: int, barrier, out):
    """One host core's copy of the workload: the oracle (the single-threaded
    reference CpuSim restated in C) on the 100k net, each bench step a reset
    followed by the first REF_SAMPLE steps of the trial; the timed region
    starts together with the other copies."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O

    onet = O.ONet.random_kout(N, K_OUT, SEED)
    sim = O.OSim(onet, O.cfg(int_weights=1, gauss_sd=1.0, synapse_tau_ms=5.0, seed=SEED))
    for _ in range(warmup):
        sim.reset_state()
        sim.run_steps(REF_SAMPLE // 5)
    barrier.wait()
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.reset_state()
        sim.run_steps(REF_SAMPLE)
    out.put((time.perf_counter() - t0, sim.ring_depth()))


def run_reference(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp

    # the reference CPU step is single-threaded (cpu.rs:216): it uses every
    # host core as independent copies of the same trial, one process each
    # (spawned; no GPU is touched), and the aggregate is their total work
    # over the slowest copy's time
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    copies = max(1, min(cores, REF_MAX_COPIES))
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(copies)
    out = ctx.Queue()
    procs = [ctx.Process(target=_reference_copy, args=(args.steps, args.warmup, barrier, out)) for _ in range(copies)]
    for p in procs:
        p.start()
    res = [out.get() for _ in range(copies)]
    for p in procs:
        p.join()
    times = [r[0] for r in res]
    dt = max(times)
    sample = REF_SAMPLE
    value = copies * N * sample * args.steps / dt
    print(json.dumps({
        "impl": "reference",
        "metric": "neuron-updates/s (synaptic events/s reported beside)",
        "value": value, "unit": "neuron-updates/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1000.0 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 state, int32 fixed-point ring",
        "data": "synthetic: seeded generator of the 100k configuration (random K=100, distance delays)",
        "config": headline_config(res[0][1], ws),
        "cpu_baseline": {"value": value, "unit": "neuron-updates/s", "cores": copies, "kind": "port",
                         "sample": f"each bench step: reset, then the first {sample} of the trial's "
                                   f"{TRIAL_STEPS} steps, in each of {copies} independent copies, one per host "
                                   f"core (of {cores}; at most {REF_MAX_COPIES}), timed together; the C "
                                   "restatement of the single-threaded reference CpuSim (the Rust reference "
                                   "cannot be built here)",
                         "per_copy_s": times, "cpu": cpu_model()},
        "e2e": {"value": value, "unit": "neuron-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the 1M, batched and serving measurements")
    ap.add_argument("--extras", default="",
                    help="comma-separated subset of the extras (c10k, c1m_izh, c1m_adex, fp32_ring_100k, batched_256, "
                         "batched_256_active, serving)")
    ap.add_argument("--serving-requests", type=int, default=200)
    ap.add_argument("--admission-threads", type=int, default=4,
                    help="serving: host threads that build admitted requests while the device steps")
    ap.add_argument("--profile", action="store_true", help="short run for ncu captures")
    ap.add_argument("--trial-steps", type=int, default=200, help="trial length in --profile mode")
    ap.add_argument("--active", action="store_true", help="--profile the active (Poisson-kick) regime")
    ap.add_argument("--profile-neurons", type=int, default=N, help="network size in --profile mode")
    ap.add_argument("--adex", action="store_true", help="--profile the AdEx variant of the random net")
    ap.add_argument("--kernel", choices=["stream", "resident"], default=None, help="force the step kernel")
    ap.add_argument("--autotune", action="store_true", help="--profile with the autotuned kernel and tiling")
    ap.add_argument("--shape", default=None,
                    help="tile shape BLOCKxNPT, e.g. 256x2 (with --kernel: fixes the headline tiling instead of "
                         "autotuning it, e.g. for an ncu launch list)")
    ap.add_argument("--delivery-warps", action="store_true",
                    help="--profile with separate delivery warps in the streaming kernel")
    ap.add_argument("--served-mix", type=int, default=0,
                    help="--profile the first N requests of the serving stream stepped as one batch")
    ap.add_argument("--batched-liquids", type=int, default=0,
                    help="--profile the first N liquids of the batched workload stepped as one batch")
    ap.add_argument("--no-inputs", action="store_true",
                    help="with --batched-liquids: build the liquids without input streams")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.profile:
        run_profile(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
