"""Shared helpers of the GPU parity tests: run the B200 backend and the C
oracle on the same flat network and compare rasters and state."""
from __future__ import annotations

import numpy as np

import pyoracle as O
import neuro_edit_v2_b200 as nb

# int ring: rasters and every state bit must match the oracle exactly.
# fp32 ring: the device sums ring arrivals with float atomics in arbitrary
# order (kernels.rs:200 does the same), so rasters must match up to a first
# divergence step and spike totals within FP32_COUNT_RTOL afterwards
# (sim/tests/gpu_vs_cpu.rs:82-112 allows 25%).
FP32_COUNT_RTOL = 0.25


def configs(int_weights: bool, chunk: int, exp_mode: int = 1, **kw):
    g = nb.default_config(record_spikes=1, spike_record_steps=chunk, int_weights=1 if int_weights else 0)
    o = O.cfg(record_spikes=1, spike_record_steps=chunk, int_weights=1 if int_weights else 0, exp_mode=exp_mode)
    for k, v in kw.items():
        setattr(g, k, v)
        setattr(o, k, v)
    return g, o


def rows_equal(g: nb.B200Sim, o: O.OSim, rows: int) -> int:
    """Index (back) of the first differing record row, or -1."""
    for back in range(rows - 1, -1, -1):
        a = g.spike_row(back)
        b = o.spike_row(back)
        if (a is None) != (b is None) or (a is not None and not np.array_equal(a, b)):
            return back
    return -1


def lockstep(onet: O.ONet, steps: int, int_weights: bool = True, chunk: int = 64, exp_mode: int = 1,
             drive=None, flat=None, mode: int | None = None, **cfg_kw):
    """Run both backends `steps` steps in chunks; return (gpu, oracle,
    first_divergent_step or -1).  `mode` forces the step kernel
    (nb.KERNEL_STREAM / nb.KERNEL_RESIDENT)."""
    flat = flat if flat is not None else onet.flat(cfg_kw.get("dt_ms", 0.1))
    gc, oc = configs(int_weights, chunk, exp_mode, **cfg_kw)
    g = nb.B200Sim(flat, gc)
    if mode is not None:
        g.set_kernel_mode(mode)
        assert g.kernel_mode()[1] == (mode == nb.KERNEL_RESIDENT)
    o = O.OSim(onet, oc)
    if drive:
        drive(g)
        drive(o)
    first = -1
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        g.run_steps(k)
        o.run_steps(k)
        bad = rows_equal(g, o, k)
        if bad >= 0 and first < 0:
            first = done + (k - 1 - bad)
            if int_weights:
                break
        done += k
    return g, o, first


def set_ext(sim, n: int, idx, amps) -> None:
    """Constant external current on the neurons `idx` of either backend."""
    if isinstance(sim, nb.B200Sim):
        ext = sim.external()
        ext[np.asarray(idx)] = amps
        sim.set_external_all(ext)
    else:
        for i in idx:
            sim.set_external(int(i), float(amps))


def assert_state_bits_equal(g: nb.B200Sim, o: O.OSim):
    for slot in (0, 1):
        a, b = g.state(slot), o.state(slot)
        bad = np.flatnonzero(a.view(np.uint32) != b.view(np.uint32))
        assert bad.size == 0, f"state {slot}: {bad.size} neurons differ, first {bad[:5]} {a[bad[:5]]} vs {b[bad[:5]]}"
    for name, a, b in (("s", g.syn_current(), o.syn_current()), ("trace", g.trace(), o.trace())):
        bad = np.flatnonzero(a.view(np.uint32) != b.view(np.uint32))
        assert bad.size == 0, f"{name}: {bad.size} neurons differ, first {bad[:5]}"
    assert g.spikes_total() == o.spikes_total()
    assert np.array_equal(g.spike_counts(2**63), o.spike_counts(2**63))


def lockstep_many(onet: O.ONet, steps: int, variants, int_weights: bool = True, chunk: int = 100,
                  exp_mode: int = 1, drive=None, **cfg_kw):
    """One oracle run against several GPU sims of the same net and config.

    `variants` is a list of dicts: {"mode": kernel mode or None, "records":
    True/False, "ws": (block, npt) to force the delivery-warp kernel in that
    tile shape}.  A sim with records off runs the step instance without the
    optional features (when nothing else is switched on); its spike totals
    and every state bit are compared after each chunk.  A sim with records on
    has every raster row compared as well.  Stops at the first difference;
    returns (gpu sims, oracle, first divergent step or -1 per sim)."""
    flat = onet.flat(cfg_kw.get("dt_ms", 0.1))
    _, oc = configs(int_weights, chunk, exp_mode, **cfg_kw)
    o = O.OSim(onet, oc)
    gs = []
    for v in variants:
        gc, _ = configs(int_weights, chunk, exp_mode, **cfg_kw)
        if not v.get("records", True):
            gc.record_spikes = 0
        g = nb.B200Sim(flat, gc)
        if v.get("mode") is not None:
            g.set_kernel_mode(v["mode"])
        if v.get("ws"):
            g.set_tile_shape(*v["ws"])
            g.set_delivery_warps(True)
            assert g.delivery_warps() == (True, True)
        gs.append(g)
    if drive:
        drive(o)
        for g in gs:
            drive(g)
    firsts = [-1] * len(gs)
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        o.run_steps(k)
        for j, (g, v) in enumerate(zip(gs, variants)):
            if firsts[j] >= 0:
                continue
            g.run_steps(k)
            if v.get("records", True):
                bad = rows_equal(g, o, k)
                if bad >= 0:
                    firsts[j] = done + (k - 1 - bad)
                    continue
            if g.spikes_total() != o.spikes_total():
                firsts[j] = done + k - 1
        if int_weights and all(f >= 0 for f in firsts):
            break
        done += k
    return gs, o, firsts
