"""B200 kernels vs the C oracle on identical seeded networks and inputs.

Fixed-point ring (int_weights): every spike raster row and every state bit
(v, u/w, s, trace) must equal the oracle's.  AdEx uses the deterministic exp
shared by kernel and oracle (exp_mode=1).  fp32 ring: rasters identical up to
a first divergence step (float atomics sum ring arrivals in arbitrary order),
then spike totals within helpers.FP32_COUNT_RTOL.  All calls go through the C
ABI (neuro_edit_v2_b200 is its ctypes mirror)."""
import numpy as np
import pytest

import pyoracle as O
import neuro_edit_v2_b200 as nb
from helpers import FP32_COUNT_RTOL, assert_state_bits_equal, lockstep, set_ext

pytestmark = pytest.mark.gpu

MODES = pytest.mark.parametrize("mode", [nb.KERNEL_STREAM, nb.KERNEL_RESIDENT], ids=["stream", "resident"])

ADEX_TONIC = [281.0, 30.0, -70.6, -50.4, 2.0, 4.0, 144.0, 80.5, -70.6, 20.0]


def fingerprint_net():
    """sim/tests/cpu_ref.rs:213-218"""
    net = O.ONet()
    r = O.rng(3)
    m = net.create_2d_grid(8, 8, 30.0)
    net.create_connections(m, 0.35, 80.0, 6.0, r)
    return net


def lsm_like_net(n_side, seed):
    """sim/tests/gpu_vs_cpu.rs:11-18"""
    net = O.ONet()
    r = O.rng(seed)
    m = net.create_3d_grid(n_side, n_side, n_side, 60.0)
    net.set_exc_inh_exact(m, n_side ** 3 // 5, r)
    net.create_connections(m, 0.4, 100.0, 5.0, r)
    return net


@MODES
def test_fingerprint_net_int_ring_bit_exact(mode):
    g, o, first = lockstep(fingerprint_net(), 400, int_weights=True, noise_rate_hz=20.0, noise_kick_mv=0.8, seed=7,
                           mode=mode)
    assert first < 0, f"raster diverged at step {first}"
    assert_state_bits_equal(g, o)


def test_fingerprint_net_fp32_ring_reproduces_reference_fingerprint():
    """The fp32 path on the net of cpu_ref.rs:208-244; its rasters must match
    the oracle (whose fingerprint is the reference's 0x9d792bd233132f5d)."""
    g, o, first = lockstep(fingerprint_net(), 400, int_weights=False, chunk=400, noise_rate_hz=20.0,
                           noise_kick_mv=0.8, seed=7)
    assert o.fingerprint(400) == 0x9D792BD233132F5D
    assert first < 0 or first > 100, f"fp32 raster diverged at step {first}"


@MODES
@pytest.mark.parametrize("n", [10_000])
def test_random_kout_gauss_noise_int_ring_bit_exact(n, mode):
    """10k workload net (random K=100, U(0,0.5)/U(0,1)x0.7 weights, distance
    delays), Gaussian current noise sd 1, tau_syn 5 ms, 2000 steps."""
    onet = O.ONet.random_kout(n, 100, 1)
    g, o, first = lockstep(onet, 2000, int_weights=True, chunk=100, gauss_sd=1.0, synapse_tau_ms=5.0,
                           drive=lambda s: set_ext(s, n, range(0, n, 7), 6.0), mode=mode)
    assert first < 0, f"raster diverged at step {first}"
    assert g.spikes_total() > 0
    assert_state_bits_equal(g, o)


@MODES
def test_bench_net_event_heavy_int_ring_bit_exact(mode):
    """bench_net regime (sim/src/bench.rs:10-52): 500 Hz x 20 mV kicks, w 4.2/5."""
    onet = O.ONet.bench_net(4000, 100, 5, 0.7, 5.0)
    g, o, first = lockstep(onet, 1500, int_weights=True, chunk=100, noise_rate_hz=500.0, noise_kick_mv=20.0,
                           seed=3, mode=mode)
    assert first < 0, f"raster diverged at step {first}"
    rate = o.mean_rate_hz()
    assert rate > 5.0, rate
    assert_state_bits_equal(g, o)


@MODES
def test_adex_random_net_int_ring_bit_exact(mode):
    onet = O.ONet.random_kout(3000, 50, 4, w_scale=0.7 * 281.0)
    for i in range(onet.n):
        onet.set_model(i, O.ADEX, ADEX_TONIC)
    g, o, first = lockstep(onet, 1500, int_weights=True, chunk=100, gauss_sd=1.0, exp_mode=1,
                           drive=lambda s: set_ext(s, 3000, range(0, 3000, 5), 900.0), mode=mode)
    assert first < 0, f"raster diverged at step {first}"
    assert g.spikes_total() > 0
    assert_state_bits_equal(g, o)


@MODES
@pytest.mark.parametrize("model", [O.IZH, O.ADEX])
def test_liquid_with_input_streams_int_ring_bit_exact(model, mode):
    onet = O.ONet.liquid(12, 7, model=model)
    rng = np.random.default_rng(3)
    bits = (rng.random((200, 8)) < 0.05).astype(np.float32)
    series = np.repeat(bits, 10, axis=0)  # each 1 ms bit held 10 steps

    def drive(s):
        for k in range(8):
            s.play_input(k, series[:, k])

    g, o, first = lockstep(onet, 2000, int_weights=True, chunk=100, drive=drive, mode=mode)
    assert first < 0, f"raster diverged at step {first}"
    assert g.spikes_total() > 0
    assert_state_bits_equal(g, o)


@pytest.mark.parametrize("int_weights", [True, False])
def test_adex_mixed_cpu_matches_gpu(int_weights):
    """sim/tests/adex.rs:54-123: izh/AdEx mixed net, exact per-neuron counts."""
    net = O.ONet()
    for i in range(8):
        net.add_neuron(i * 50.0, 0.0, 0.0, O.EXC)
    for i in (1, 3, 4, 6):
        net.set_model(i, O.ADEX, ADEX_TONIC)
    net.connect(0, 1, 8.0)
    net.connect(1, 2, 8.0)
    net.connect(3, 4, 5.0)

    def drive(s):
        for i, a in [(0, 15.0), (1, 900.0), (3, 800.0), (4, 1000.0), (6, 1200.0)]:
            s.set_external(i, a)

    g, o, first = lockstep(net, 3000, int_weights=int_weights, chunk=100, drive=drive)
    assert first < 0
    cc, gc = o.spike_counts(2**63), g.spike_counts(2**63)
    assert np.array_equal(cc, gc)
    assert all(cc[i] >= 2 for i in (1, 3, 4, 6))
    assert np.all(np.abs(g.state(0) - o.state(0)) < 0.5)


def test_gpu_matches_cpu_spike_counts_quiet():
    """sim/tests/gpu_vs_cpu.rs:24-49 (fp32 ring, no noise): equal totals."""
    onet = lsm_like_net(8, 42)
    g, o, first = lockstep(onet, 500, int_weights=False, chunk=500,
                           drive=lambda s: set_ext(s, 512, range(8), 12.0))
    assert o.spikes_total() > 0
    assert g.spikes_total() == o.spikes_total()


def test_fp32_ring_with_noise_first_divergence_and_counts():
    """sim/tests/gpu_vs_cpu.rs:82-112: fp32 ring with noise; rasters equal up
    to the first divergence, totals within the stated tolerance."""
    onet = lsm_like_net(8, 7)
    g, o, first = lockstep(onet, 1000, int_weights=False, chunk=100, noise_rate_hz=1000.0, noise_kick_mv=20.0,
                           seed=99)
    a, b = o.spikes_total(), g.spikes_total()
    assert a > 0
    assert abs(a - b) / max(a, 1) < FP32_COUNT_RTOL
    tr = g.trace()
    assert np.all((tr >= 0) & (tr <= 1))
    v = g.v()
    assert np.all((v < 100.0) & (v > -200.0))
    if first >= 0:
        print(f"fp32 first divergent step: {first}")


def test_int_weights_bitwise_deterministic():
    """sim/tests/gpu_vs_cpu.rs:116-141: two int-ring GPU runs are identical."""
    flat = lsm_like_net(8, 5).flat()
    cfg = dict(noise_rate_hz=2000.0, noise_kick_mv=20.0, seed=7, int_weights=1, record_spikes=1)
    a = nb.B200Sim(flat, **cfg)
    b = nb.B200Sim(flat, **cfg)
    a.run_steps(800)
    b.run_steps(800)
    assert a.spikes_total() == b.spikes_total() > 0
    assert np.array_equal(a.v().view(np.uint32), b.v().view(np.uint32))
    assert np.array_equal(a.spike_counts(64), b.spike_counts(64))


def test_int_weights_close_to_float():
    """sim/tests/gpu_vs_cpu.rs:145-177"""
    flat = lsm_like_net(8, 11).flat()
    base = dict(noise_rate_hz=2000.0, noise_kick_mv=20.0, seed=3)
    f = nb.B200Sim(flat, **base)
    i = nb.B200Sim(flat, int_weights=1, **base)
    f.run_steps(800)
    i.run_steps(800)
    tf, ti = f.spikes_total(), i.spikes_total()
    assert tf > 0 and ti > 0
    assert abs(tf - ti) / tf < 0.3


@MODES
def test_100k_workload_int_ring_bit_exact_first_1000_steps(mode):
    """The 100k configuration (random K=100, ~10M synapses) against the
    oracle for 1000 steps, every raster row compared."""
    onet = O.ONet.random_kout(100_000, 100, 1)
    g, o, first = lockstep(onet, 1000, int_weights=True, chunk=100, gauss_sd=1.0, synapse_tau_ms=5.0,
                           drive=lambda s: set_ext(s, 100_000, range(0, 100_000, 11), 8.0), mode=mode)
    assert first < 0, f"raster diverged at step {first}"
    assert g.spikes_total() > 0
    assert_state_bits_equal(g, o)


def test_auto_mode_streams_and_resident_runs_only_where_state_fits():
    small = nb.random_kout(20_000, 10, 1)
    g = nb.B200Sim(small)
    assert g.kernel_mode() == (nb.KERNEL_AUTO, False)
    g.set_kernel_mode(nb.KERNEL_RESIDENT)
    assert g.kernel_mode() == (nb.KERNEL_RESIDENT, True)
    g.run_steps(10)
    n = 3_000_000  # 16 B of on-chip state per neuron exceeds 148 SMs x 227 KB
    big = nb.FlatNet(model=np.zeros(n, np.uint8), params=np.tile(np.float32([0.02, 0.2, -65, 8]), (n, 1)),
                     src_ptr=np.zeros(n + 1, np.uint32), tgt=np.zeros(0, np.uint32), w=np.zeros(0, np.float32),
                     delay_steps=np.zeros(0, np.uint16))
    b = nb.B200Sim(big, int_weights=1)
    assert b.kernel_mode() == (nb.KERNEL_AUTO, False)
    with pytest.raises(nb.Ne2bError, match="UNSUPPORTED"):
        b.set_kernel_mode(nb.KERNEL_RESIDENT)
    assert b.kernel_mode() == (nb.KERNEL_AUTO, False)
    b.set_external_all(np.full(n, 10.0, np.float32))
    b.run_steps(20)
    assert b.step_count() == 20 and b.spikes_total() == 0


def test_resident_and_stream_agree_over_many_launches():
    """Long run crossing many resident launches (4096 steps each) and stimulus
    chunks: both kernels give the same state bit-for-bit."""
    onet = O.ONet.liquid(10, 3)
    flat = onet.flat()
    x = (np.random.default_rng(5).random((1000, 8)) < 0.05).astype(np.float32).repeat(10, axis=0)
    sims = []
    for mode in (nb.KERNEL_STREAM, nb.KERNEL_RESIDENT):
        s = nb.B200Sim(flat, int_weights=1, record_spikes=1, gauss_sd=2.0, noise_rate_hz=50.0)
        s.set_kernel_mode(mode)
        for k in range(8):
            s.play_input(k, x[:, k])
        s.run_steps(9000)
        s.run_steps(1000)
        sims.append(s)
    a, b = sims
    assert a.spikes_total() == b.spikes_total() > 0
    for slot in (0, 1):
        assert np.array_equal(a.state(slot).view(np.uint32), b.state(slot).view(np.uint32))
    assert np.array_equal(a.trace().view(np.uint32), b.trace().view(np.uint32))
    assert np.array_equal(a.spike_counts(400), b.spike_counts(400))


@MODES
@pytest.mark.parametrize("shape", [(64, 1), (256, 1), (128, 4)], ids=lambda s: f"{s[0]}x{s[1]}")
def test_synchronous_bursts_int_ring_bit_exact(mode, shape):
    """A strong constant drive on every neuron makes whole tiles spike in the
    same step, so a tile delivers up to BLOCK x NPT x 100 synapses: many
    passes of the block-strided delivery, each thread with its four
    synapses in flight, the last pass partial.  Bit-exact against the
    oracle, rows and state."""
    n = 20_000
    onet = O.ONet.random_kout(n, 100, 4)

    def drive(s):
        if isinstance(s, nb.B200Sim):
            s.set_tile_shape(*shape)
        set_ext(s, n, range(n), 40.0)

    g, o, first = lockstep(onet, 200, int_weights=True, chunk=50, gauss_sd=1.0, synapse_tau_ms=5.0, drive=drive,
                           mode=mode)
    assert first < 0, f"raster diverged at step {first}"
    assert g.spikes_total() > 5 * n  # ~390 Hz: every neuron fires every few steps
    assert_state_bits_equal(g, o)


def plain_lockstep(onet, steps, chunk, mode=None, adex=False, toggles=None, **kw):
    """Both backends without spike records (so the GPU runs the plain step
    instance while nothing else is switched on): after every chunk the
    spike totals and every state bit must agree.  `toggles[c]` (an external
    amplitude, or None) is applied to every third neuron before chunk c."""
    from helpers import configs

    gc, oc = configs(True, 64, 1, **kw)
    gc.record_spikes = oc.record_spikes = 0
    g = nb.B200Sim(onet.flat(0.1), gc)
    if mode is not None:
        g.set_kernel_mode(mode)
    o = O.OSim(onet, oc)
    n = g.n()
    for c in range(steps // chunk):
        amp = toggles[c] if toggles and c < len(toggles) else None
        if amp is not None:
            set_ext(g, n, range(0, n, 3), amp)
            set_ext(o, n, range(0, n, 3), amp)
        g.run_steps(chunk)
        o.run_steps(chunk)
        assert g.spikes_total() == o.spikes_total(), f"spike totals differ after chunk {c}"
        assert_state_bits_equal(g, o)
    return g


@pytest.mark.parametrize("n", [20_000, 100_000])
def test_plain_instance_random_net_bit_exact(n):
    """No records, no drive: the plain step instance, 768 steps in three
    full launch groups, state and spike totals bit-exact."""
    g = plain_lockstep(O.ONet.random_kout(n, 100, 2), 768, 256, mode=nb.KERNEL_STREAM, gauss_sd=1.0,
                       synapse_tau_ms=5.0, noise_rate_hz=100.0, noise_kick_mv=20.0)
    assert g.spikes_total() > 0


def test_plain_instance_1m_net_bit_exact():
    """The 1M-neuron workload (random K=100, ~1e8 synapses, Gaussian noise)
    on the plain instance for one full launch group: the state that stays in
    L2 between steps is every bit the oracle's."""
    g = plain_lockstep(O.ONet.random_kout(1_000_000, 100, 1), 256, 256, mode=nb.KERNEL_STREAM, gauss_sd=1.0,
                       synapse_tau_ms=5.0, noise_rate_hz=20.0, noise_kick_mv=20.0)
    assert g.spikes_total() > 0


def test_plain_instance_adex_bit_exact():
    onet = O.ONet.random_kout(20_000, 100, 5, w_scale=0.7 * 281.0)
    for i in range(onet.n):
        onet.set_model(i, O.ADEX, ADEX_TONIC)
    g = plain_lockstep(onet, 512, 256, mode=nb.KERNEL_STREAM, gauss_sd=1.0, synapse_tau_ms=5.0,
                       noise_rate_hz=100.0, noise_kick_mv=20.0)
    assert g.spikes_total() > 0


def test_features_switched_on_and_off_between_launches_stay_bit_exact():
    """An external current switched on, off and on again between launch
    groups moves the engine between the plain and the full step instance
    (its cached graphs included); state and spike totals stay bit-exact."""
    g = plain_lockstep(O.ONet.random_kout(20_000, 100, 6), 256 * 6, 256, mode=nb.KERNEL_STREAM, gauss_sd=1.0,
                       synapse_tau_ms=5.0, noise_rate_hz=50.0, noise_kick_mv=20.0,
                       toggles=[None, 9.0, 0.0, None, 12.0, 0.0])
    assert g.spikes_total() > 0


def run_both(net, steps, drive, **cfg_kw):
    """Both backends for `steps` steps without raster checks (the reference's
    AdEx bar compares counts and v only); returns (gpu, oracle)."""
    from helpers import configs

    gc, oc = configs(cfg_kw.pop("int_weights", True), 64, cfg_kw.pop("exp_mode", 1), **cfg_kw)
    g = nb.B200Sim(net.flat(), gc)
    o = O.OSim(net, oc)
    drive(g)
    drive(o)
    g.run_steps(steps)
    o.run_steps(steps)
    return g, o


@pytest.mark.parametrize("int_weights", [True, False])
def test_adex_mixed_against_glibc_exp_reference_tolerance(int_weights):
    """sim/tests/adex.rs:54-123 as the reference states it: the oracle calls
    glibc expf (exp_mode=0, the reference CPU path, adex.rs:168) while the
    device uses its deterministic exp; per-neuron spike counts must be equal
    and |dv| < 0.5 mV at the end."""
    net = O.ONet()
    for i in range(8):
        net.add_neuron(i * 50.0, 0.0, 0.0, O.EXC)
    for i in (1, 3, 4, 6):
        net.set_model(i, O.ADEX, ADEX_TONIC)
    net.connect(0, 1, 8.0)
    net.connect(1, 2, 8.0)
    net.connect(3, 4, 5.0)

    def drive(s):
        for i, a in [(0, 15.0), (1, 900.0), (3, 800.0), (4, 1000.0), (6, 1200.0)]:
            s.set_external(i, a)

    g, o = run_both(net, 3000, drive, int_weights=int_weights, exp_mode=0)
    cc, gc = o.spike_counts(2**63), g.spike_counts(2**63)
    assert np.array_equal(cc, gc)
    assert all(cc[i] >= 2 for i in (1, 3, 4, 6))
    assert np.all(np.abs(g.state(0) - o.state(0)) < 0.5)


def test_adex_population_against_glibc_exp_reference_tolerance():
    """3000 unconnected AdEx neurons under constant currents spread over the
    tonic range (600-1400 pA) for 3000 steps, oracle with glibc expf: equal
    per-neuron spike counts and |dv| < 0.5 mV (the adex.rs:104-122 bar) on a
    population that crosses the exponential upswing many thousand times."""
    n = 3000
    net = O.ONet()
    for i in range(n):
        net.add_neuron(float(i), 0.0, 0.0, O.EXC)
        net.set_model(i, O.ADEX, ADEX_TONIC)
    amps = np.linspace(600.0, 1400.0, n).astype(np.float32)

    def drive(s):
        if isinstance(s, nb.B200Sim):
            s.set_external_all(amps)
        else:
            for i in range(n):
                s.set_external(i, float(amps[i]))

    g, o = run_both(net, 3000, drive, int_weights=True, exp_mode=0)
    cc, gc = o.spike_counts(2**63), g.spike_counts(2**63)
    assert cc.sum() > 5 * n
    assert np.array_equal(cc, gc), f"{np.count_nonzero(cc != gc)} neurons differ in count"
    assert np.all(np.abs(g.state(0) - o.state(0)) < 0.5)
