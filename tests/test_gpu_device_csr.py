"""The synapse CSR built on the GPU (`ne2b_create_from_synapses`) against
the host build (`ne2b_net_from_synapses`, pinned on the reference's
cpu_ref.rs:246-255 CSR order and the oracle's `synapse_csr`): the same
stable source order (network.rs:656-657), Dale's sign (668-672), delay
steps (660-666) and fixed-point weights, bit for bit; the same sim; the
same errors."""
import numpy as np
import pytest

import pyoracle as O
import neuro_edit_v2_b200 as nb

pytestmark = pytest.mark.gpu

IZH = np.array([0.02, 0.2, -65.0, 8.0], np.float32)


def synapse_list(n, e, seed, srcs=None, max_delay_ms=20.0):
    rng = np.random.default_rng(seed)
    src = rng.integers(0, srcs if srcs else n, e).astype(np.uint32)
    tgt = rng.integers(0, n, e).astype(np.uint32)
    w = rng.uniform(-1.0, 1.0, e).astype(np.float32)  # the sign is Dale's, not the list's
    d = rng.uniform(0.0, max_delay_ms, e).astype(np.float32)
    d[: e // 50] = np.float32(0.05) * rng.integers(0, 3, e // 50).astype(np.float32)  # ties and sub-step delays
    kind = (rng.random(n) < 0.2).astype(np.uint8)
    model = np.zeros(n, np.uint8)
    params = np.tile(IZH, (n, 1))
    return model, params, kind, src, tgt, w, d


def both(n, e, seed, int_weights=1, srcs=None, max_delay_ms=20.0, **kw):
    model, params, kind, src, tgt, w, d = synapse_list(n, e, seed, srcs, max_delay_ms)
    cfg = nb.default_config(int_weights=int_weights, **kw)
    host = nb.B200Sim(nb.from_synapses(model, params, kind, src, tgt, w, d, dt_ms=cfg.dt_ms), cfg)
    dev = nb.B200Sim.from_synapses(model, params, kind, src, tgt, w, d, cfg)
    return host, dev


def same_csr(a, b):
    for x, y, what in zip(a.read_csr(), b.read_csr(), ("rowptr", "tgt", "w", "delay")):
        assert np.array_equal(x, y), what


@pytest.mark.parametrize("int_weights", [0, 1])
@pytest.mark.parametrize("n, e, srcs", [
    (2000, 150_000, None),      # many chunks, runs shared across chunks
    (5000, 40_000, 3),          # three sources: every run spans many chunks
    (300, 8192 * 3 + 17, 1),    # one source: a single run through every chunk
    (100_000, 20_000, None),    # more sources than synapses
])
def test_device_csr_equals_host_csr(int_weights, n, e, srcs):
    host, dev = both(n, e, 7 + n, int_weights, srcs)
    assert dev.syn_count() == host.syn_count() == e
    same_csr(host, dev)
    assert dev.ring_depth() == host.ring_depth()


def test_large_lists_stream_through_the_pinned_ring():
    """20M synapses: the device build uploads a 320 MB list and the host
    build a 180 MB CSR, both larger than two 32 MB staging blocks, so both
    stream through the stager's ring of pinned blocks."""
    host, dev = both(200_000, 20_000_000, 13)
    assert dev.syn_count() == host.syn_count() == 20_000_000
    same_csr(host, dev)


def test_long_delays_use_the_u16_ring_on_both_paths():
    host, dev = both(3000, 60_000, 5, max_delay_ms=60.0)
    assert dev.ring_depth() > 257
    same_csr(host, dev)


def test_device_built_sim_runs_like_the_host_built_one():
    host, dev = both(4000, 200_000, 11, 1, noise_rate_hz=300.0, record_spikes=1)
    host.run_steps(600)
    dev.run_steps(600)
    assert dev.spikes_total() == host.spikes_total() > 0
    assert np.array_equal(dev.v().view(np.uint32), host.v().view(np.uint32))
    assert np.array_equal(dev.spike_counts(512), host.spike_counts(512))


def test_device_csr_matches_the_oracle_csr():
    """The oracle's stable sort (network.rs:656-657) on the same list."""
    onet = O.ONet()
    rng = np.random.default_rng(2)
    n = 500
    for i in range(n):
        onet.add_neuron(0.0, 0.0, 0.0, O.INH if i % 5 == 0 else O.EXC)
    src = rng.integers(0, n, 30_000)
    tgt = rng.integers(0, n, 30_000)
    w = rng.uniform(0.1, 2.0, 30_000).astype(np.float32)
    d = rng.uniform(0.1, 15.0, 30_000).astype(np.float32)
    for a, b, x, y in zip(src, tgt, w, d):
        onet.push_synapse(int(a), int(b), float(x), float(y), 0.0)
    model, params = onet.models()
    sim = nb.B200Sim.from_synapses(model, params, onet.kinds(), src, tgt, w, d, int_weights=0)
    f = onet.flat(0.1)
    rowptr, tg, wb, dl = sim.read_csr()
    assert np.array_equal(rowptr, f.src_ptr)
    assert np.array_equal(tg, f.tgt)
    assert np.array_equal(wb, f.w.view(np.uint32))
    assert np.array_equal(dl, f.delay_steps)


def test_empty_lists():
    model, params, kind, *_ = synapse_list(10, 0, 1)
    e = np.zeros(0, np.uint32)
    sim = nb.B200Sim.from_synapses(model, params, kind, e, e, e.view(np.float32), e.view(np.float32))
    assert sim.syn_count() == 0
    assert np.array_equal(sim.read_csr()[0], np.zeros(11, np.uint32))
    sim.run_steps(10)
    assert sim.step_count() == 10


@pytest.mark.parametrize("case", ["src", "tgt", "delay", "nan"])
def test_errors_equal_the_host_build(case):
    model, params, kind, src, tgt, w, d = synapse_list(100, 20_000, 3)
    if case == "src":
        src[12345] = 100
    elif case == "tgt":
        tgt[777] = 1000
    elif case == "delay":
        d[4321] = np.float32(7000.0)
    else:
        d[99] = np.float32("nan")
    with pytest.raises(nb.Ne2bError) as h:
        nb.B200Sim(nb.from_synapses(model, params, kind, src, tgt, w, d, dt_ms=0.1), nb.default_config())
    with pytest.raises(nb.Ne2bError) as g:
        nb.B200Sim.from_synapses(model, params, kind, src, tgt, w, d)
    assert str(g.value) == str(h.value)


@pytest.mark.parametrize("which", ["all", "list_only"])
def test_device_resident_lists_are_read_in_place(which):
    """Synapse lists already in device memory (CUDA torch tensors here) give
    the CSR, ring and errors of the same list passed from the host."""
    torch = pytest.importorskip("torch")
    model, params, kind, src, tgt, w, d = synapse_list(3000, 120_000, 11)
    cfg = nb.default_config()
    host = nb.B200Sim.from_synapses(model, params, kind, src, tgt, w, d, cfg)
    cols = [torch.from_numpy(a).cuda() for a in (src.view(np.int32), tgt.view(np.int32), w, d)]
    cols[0], cols[1] = _u32(cols[0]), _u32(cols[1])
    k = torch.from_numpy(kind).cuda() if which == "all" else kind
    dev = nb.B200Sim.from_synapses(model, params, k, *cols, cfg)
    same_csr(host, dev)
    assert dev.ring_depth() == host.ring_depth()
    bad = d.copy()
    bad[4321] = np.float32(7000.0)
    with pytest.raises(nb.Ne2bError) as h:
        nb.B200Sim.from_synapses(model, params, kind, src, tgt, w, bad, cfg)
    with pytest.raises(nb.Ne2bError) as g:
        nb.B200Sim.from_synapses(model, params, k, *cols[:3], torch.from_numpy(bad).cuda(), cfg)
    assert str(g.value) == str(h.value)


def _u32(t):
    """A CUDA int32 tensor presented as uint32 through the array interface."""
    class View:
        def __init__(self, t):
            self.t = t
            cai = dict(t.__cuda_array_interface__)
            cai["typestr"] = "<u4"
            self.__cuda_array_interface__ = cai
    return View(t)
