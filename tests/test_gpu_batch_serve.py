"""Batched liquids and the serving loop: each net's result must equal the
same net run alone (bit-identical in fixed-point mode) and the oracle's."""
import numpy as np
import pytest

import pyoracle as O
import neuro_edit_v2_b200 as nb

pytestmark = pytest.mark.gpu

WIN = 100


def streams(seed, steps, n_inputs=8, p=0.05, hold=10):
    rng = np.random.default_rng(seed)
    bits = (rng.random((steps // hold + 1, n_inputs)) < p).astype(np.float32)
    return np.repeat(bits, hold, axis=0)[:steps]


def liquids():
    sides = [6, 9, 7, 11, 8, 5]
    models = [nb.MODEL_IZH, nb.MODEL_ADEX, nb.MODEL_IZH, nb.MODEL_IZH, nb.MODEL_ADEX, nb.MODEL_IZH]
    return [nb.liquid(s, 100 + k, model=m) for k, (s, m) in enumerate(zip(sides, models))]


def cfg(seed):
    return nb.default_config(int_weights=1, window_steps=WIN, max_windows=16, seed=seed, gauss_sd=0.5)


def test_batch_equals_alone_and_oracle():
    steps = 1000
    nets = liquids()
    cfgs = [cfg(7 + k) for k in range(len(nets))]
    b = nb.Batch(nets, cfgs)
    for k in range(len(nets)):
        x = streams(k, steps)
        for i in range(8):
            b.play_input(k, i, x[:, i])
    b.run_steps(steps)
    for k, net in enumerate(nets):
        alone = nb.B200Sim(net, cfgs[k])
        x = streams(k, steps)
        for i in range(8):
            alone.play_input(i, x[:, i])
        alone.run_steps(steps)
        for w in range(steps // WIN):
            assert np.array_equal(b.window_counts(k, w), alone.window_counts(w)), (k, w)
        assert b.spikes_total(k) == alone.spikes_total()
        assert np.array_equal(b.state(k, 0).view(np.uint32), alone.v().view(np.uint32))
    # oracle on two of them
    for k in (0, 1):
        side = [6, 9][k]
        onet = O.ONet.liquid(side, 100 + k, model=[O.IZH, O.ADEX][k])
        o = O.OSim(onet, O.cfg(int_weights=1, record_spikes=1, spike_record_steps=WIN, seed=7 + k, gauss_sd=0.5,
                               exp_mode=1))
        x = streams(k, steps)
        for i in range(8):
            o.play_input(i, x[:, i])
        for w in range(steps // WIN):
            o.run_steps(WIN)
            assert np.array_equal(b.window_counts(k, w).astype(np.uint32), o.spike_counts(WIN)), (k, w)


def test_batch_with_more_tiles_per_block_than_staged_equals_default_grid():
    """One block per SM gives every block more tiles than the streaming
    kernel stages before its dependency wait (16), from many nets: the tiles
    past the staged ones load their records and net descriptors as they
    come.  Results equal those of another tiling bit for bit, and the
    oracle's on an izh and an AdEx net."""
    import torch

    steps, n_nets, side = 300, 200, 12
    models = [nb.MODEL_ADEX if k % 3 == 0 else nb.MODEL_IZH for k in range(n_nets)]
    nets = [nb.liquid(side, 300 + k, model=models[k]) for k in range(n_nets)]
    cfgs = [cfg(11 + k) for k in range(n_nets)]
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert n_nets * -(-side**3 // 128) > 16 * sms  # tiles of 128 neurons per block of a one-per-SM grid
    a, b = nb.Batch(nets, cfgs), nb.Batch(nets, cfgs)
    for bb in (a, b):
        bb.set_kernel_mode(nb.KERNEL_STREAM)
        for k in range(n_nets):
            x = streams(k, steps)
            for i in range(8):
                bb.play_input(k, i, x[:, i])
    a.set_tile_shape(128, 1, 1)
    b.set_tile_shape(256, 2, 0)
    a.run_steps(steps)
    b.run_steps(steps)
    for k in range(n_nets):
        for w in range(steps // WIN):
            assert np.array_equal(a.window_counts(k, w), b.window_counts(k, w)), (k, w)
        assert a.spikes_total(k) == b.spikes_total(k)
        assert np.array_equal(a.state(k, 0).view(np.uint32), b.state(k, 0).view(np.uint32)), k
    assert sum(a.spikes_total(k) for k in range(n_nets)) > 0
    for k in (0, 1):
        onet = O.ONet.liquid(side, 300 + k, model=O.ADEX if models[k] == nb.MODEL_ADEX else O.IZH)
        o = O.OSim(onet, O.cfg(int_weights=1, record_spikes=1, spike_record_steps=WIN, seed=11 + k, gauss_sd=0.5,
                               exp_mode=1))
        x = streams(k, steps)
        for i in range(8):
            o.play_input(i, x[:, i])
        for w in range(steps // WIN):
            o.run_steps(WIN)
            assert np.array_equal(a.window_counts(k, w).astype(np.uint32), o.spike_counts(WIN)), (k, w)


def test_batch_autotune_keeps_results():
    nets = liquids()[:4]
    cfgs = [cfg(3 + k) for k in range(4)]
    a = nb.Batch(nets, cfgs)
    b = nb.Batch(nets, cfgs)
    for bb in (a, b):
        for k in range(4):
            x = streams(k, 600)
            for i in range(8):
                bb.play_input(k, i, x[:, i])
    shape = a.autotune(64)
    assert shape[0] in (64, 128, 256, 512)
    a.run_steps(600)
    b.run_steps(600)
    for k in range(4):
        for w in range(6):
            assert np.array_equal(a.window_counts(k, w), b.window_counts(k, w))


@pytest.mark.parametrize("threads", [0, 2])
def test_server_results_equal_alone_and_admission(threads):
    """Served requests equal the same nets run alone, with admission inside
    submit (threads = 0) or on admission threads while the device steps."""
    nets = liquids()
    steps = [500, 800, 300, 700, 400, 600]
    srv = nb.Server(neuron_capacity=3 * 2048, synapse_capacity=10**7, ring_capacity=10**8, max_requests=3,
                    steps_per_launch=50, admission_threads=threads)
    pending = list(range(len(nets)))
    ids = {}
    refused = 0
    for _ in range(10_000):
        while pending:
            k = pending[0]
            rid = srv.submit(nets[k], cfg(20 + k), streams(k, steps[k]), steps[k])
            if rid is None:
                refused += 1
                break
            ids[rid] = k
            pending.pop(0)
        srv.step()
        if not pending and srv.stats()["active"] == 0:
            break
    assert refused > 0  # capacity forced queueing
    srv.synchronize()
    results = {}
    for rid in srv.finished():
        counts, tot = srv.take(rid)
        results[ids[rid]] = (counts, tot)
    assert sorted(results) == list(range(len(nets)))
    for k, net in enumerate(nets):
        alone = nb.B200Sim(net, cfg(20 + k))
        x = streams(k, steps[k])
        for i in range(8):
            alone.play_input(i, x[:, i])
        alone.run_steps(steps[k])
        counts, tot = results[k]
        assert tot == alone.spikes_total()
        for w in range(steps[k] // WIN):
            assert np.array_equal(counts[w], alone.window_counts(w)), (k, w)


@pytest.mark.parametrize("threads", [0, 2])
def test_server_invalid_request_is_an_error(threads):
    """A net that fails validation (a target out of range) is refused by
    submit, or, with admission threads, finishes with the error that take
    reports; the server keeps serving."""
    one = O.ONet()
    one.add_neuron(0, 0, 0, O.EXC)
    bad = one.flat()
    bad.src_ptr = np.array([0, 1], np.uint32)
    bad.tgt = np.array([5], np.uint32)
    bad.w = np.array([1.0], np.float32)
    bad.delay_steps = np.array([1], np.uint16)
    good = liquids()[0]
    srv = nb.Server(neuron_capacity=4096, synapse_capacity=10**6, ring_capacity=10**7, max_requests=4,
                    steps_per_launch=50, admission_threads=threads)
    x = np.zeros((200, 0), np.float32)
    if threads == 0:
        with pytest.raises(nb.Ne2bError, match="EINVAL"):
            srv.submit(bad, cfg(1), x, 200)
    else:
        rid = srv.submit(bad, cfg(1), x, 200)
        gid = srv.submit(good, cfg(2), streams(2, 200), 200)
        for _ in range(100):
            srv.step()
            if srv.stats()["active"] == 0:
                break
        srv.synchronize()
        assert sorted(srv.finished()) == sorted([rid, gid])
        with pytest.raises(nb.Ne2bError, match="EINVAL"):
            srv.take(rid)
        counts, tot = srv.take(gid)
        assert counts.shape == (2, good.n)


def test_server_rejects_oversized_request():
    srv = nb.Server(neuron_capacity=512, synapse_capacity=10**6, ring_capacity=10**6, max_requests=2)
    big = nb.liquid(10, 1)
    with pytest.raises(nb.Ne2bError, match="total capacity"):
        srv.submit(big, cfg(1), streams(0, 100), 100)


def test_batch_input_matrix_equals_played_series():
    """Device-resident input matrices give the same trial as the host-packed
    stimulus program (stim.rs:118-127) across chunk boundaries."""
    nets = liquids()[:3]
    cfgs = [cfg(40 + k) for k in range(3)]
    steps = 4500  # crosses the 2048-step packing chunks
    a = nb.Batch(nets, cfgs)
    b = nb.Batch(nets, cfgs)
    for k in range(3):
        x = streams(50 + k, steps)
        a.set_input_matrix(k, x)
        for i in range(8):
            b.play_input(k, i, x[:, i])
    a.run_steps(steps)
    b.run_steps(steps)
    for k in range(3):
        assert a.spikes_total(k) == b.spikes_total(k) > 0
        for w in range(16):
            assert np.array_equal(a.window_counts(k, w), b.window_counts(k, w))
    # a second trial after reset replays the same matrix from t = 0
    tot = [a.spikes_total(k) for k in range(3)]
    a.reset_state()
    a.run_steps(steps)
    assert [a.spikes_total(k) for k in range(3)] == tot
