"""Readout training on the GPU (`ne2b_fit_ridge_multi`,
`ne2b_batch_fit_ridge_multi`) against the oracle's restatement of
fit_ridge_multi (sim/src/readout.rs:190-252): the weights are equal bit
for bit, from host or device memory and from a batch's on-device window
counts."""
import numpy as np
import pytest

import pyoracle as O
import neuro_edit_v2_b200 as nb

pytestmark = pytest.mark.gpu


def design(t, f, seed):
    rng = np.random.default_rng(seed)
    return rng.poisson(1.5, (t, f)).astype(np.float32), rng.integers(0, 1 << 30, t)


@pytest.mark.parametrize("t, f, k, lam", [
    (40, 37, 2, 1.0),      # F not a multiple of 4: the tail sum
    (97, 515, 3, 0.1),     # T across Gram tiles, a partial column chunk
    (300, 2000, 5, 2.0),
    (64, 64, 4, 0.5),
])
def test_weights_equal_the_oracle_bit_for_bit(t, f, k, lam):
    x, r = design(t, f, t + f)
    lab = r % k
    w = nb.fit_ridge_multi(x, lab, k, lam)
    ref = O.fit_ridge_multi(x, lab, k, lam)
    assert np.array_equal(w.view(np.uint64), ref.view(np.uint64))
    assert np.isfinite(w).all() and np.abs(w[:, :-1]).max() > 0


def test_design_in_device_memory():
    import torch

    x, r = design(120, 333, 5)
    lab = r % 3
    host = nb.fit_ridge_multi(x, lab, 3, 0.5)
    dev = nb.fit_ridge_multi(torch.from_numpy(x).cuda(), lab, 3, 0.5)
    assert np.array_equal(host.view(np.uint64), dev.view(np.uint64))


def test_singular_gram_matrix_follows_the_reference():
    """lambda = 0 and more rows than features: the centred Gram matrix is
    singular, and whatever its factorization meets (a non-positive pivot and
    zero dual weights, or tiny pivots) the device meets too."""
    x, r = design(50, 10, 9)
    lab = r % 2
    w = nb.fit_ridge_multi(x, lab, 2, 0.0)
    ref = O.fit_ridge_multi(x, lab, 2, 0.0)
    assert np.array_equal(np.nan_to_num(w).view(np.uint64), np.nan_to_num(ref).view(np.uint64))


def test_batch_window_counts_train_the_readout_on_the_device():
    """One liquid, 24 trials with different input streams, 10 windows of
    100 steps: the readout trained from the counts on the device equals the
    oracle's fit on the same counts copied out."""
    t, win, nwin = 24, 100, 10
    net = nb.liquid(8, 5)
    cfgs = [nb.default_config(int_weights=1, window_steps=win, max_windows=nwin, seed=3 + r) for r in range(t)]
    b = nb.Batch([net] * t, cfgs)
    rng = np.random.default_rng(1)
    for r in range(t):
        bits = (rng.random((win * nwin // 10 + 1, 8)) < 0.05).astype(np.float32)
        b.set_input_matrix(r, np.repeat(bits, 10, axis=0)[: win * nwin])
    b.run_steps(win * nwin)
    b.synchronize()
    lab = np.arange(t) % 3
    w = b.fit_ridge_multi(np.arange(t), nwin, lab, 3, 1.0)
    x = np.stack([np.concatenate([b.window_counts(r, q).astype(np.float32) for q in range(nwin)]) for r in range(t)])
    assert x.sum() > 0
    ref = O.fit_ridge_multi(x, lab, 3, 1.0)
    assert w.shape == ref.shape == (3, nwin * net.n + 1)
    assert np.array_equal(w.view(np.uint64), ref.view(np.uint64))


@pytest.mark.parametrize("t, f, lam", [(80, 31, 0.5), (200, 517, 1.0), (33, 64, 0.25)])
def test_binary_ridge_equals_the_oracle_bit_for_bit(t, f, lam):
    x, r = design(t, f, 3 * t + f)
    y = (r % 2).astype(np.float32) * 2 - 1
    w = nb.fit_ridge(x, y, lam)
    ref = O.fit_ridge(x, y, lam)
    assert np.array_equal(w.view(np.uint64), ref.view(np.uint64))
    assert np.abs(w).max() > 0


def test_binary_ridge_fallback_regularisation_matches():
    """A duplicated feature and lambda = 0: the normal matrix is singular, so
    the reference refactors with 1e-3 more on the diagonal (readout.rs:131-139)."""
    x, r = design(60, 12, 4)
    x[:, 5] = x[:, 4]
    y = (r % 2).astype(np.float32)
    w = nb.fit_ridge(x, y, 0.0)
    ref = O.fit_ridge(x, y, 0.0)
    assert np.array_equal(np.nan_to_num(w).view(np.uint64), np.nan_to_num(ref).view(np.uint64))


def test_batch_counts_train_the_binary_readout():
    t, win, nwin = 20, 100, 5
    net = nb.liquid(7, 9)
    cfgs = [nb.default_config(int_weights=1, window_steps=win, max_windows=nwin, seed=50 + r) for r in range(t)]
    b = nb.Batch([net] * t, cfgs)
    rng = np.random.default_rng(2)
    for r in range(t):
        bits = (rng.random((win * nwin // 10 + 1, 8)) < 0.05).astype(np.float32)
        b.set_input_matrix(r, np.repeat(bits, 10, axis=0)[: win * nwin])
    b.run_steps(win * nwin)
    b.synchronize()
    y = (np.arange(t) % 2).astype(np.float32)
    w = b.fit_ridge(np.arange(t), nwin, y, 1.0)
    x = np.stack([np.concatenate([b.window_counts(r, q).astype(np.float32) for q in range(nwin)]) for r in range(t)])
    ref = O.fit_ridge(x, y, 1.0)
    assert np.array_equal(w.view(np.uint64), ref.view(np.uint64))


def test_arguments_the_reference_rejects():
    x, _ = design(10, 5, 1)
    with pytest.raises(nb.Ne2bError, match="label"):
        nb.fit_ridge_multi(x, np.full(10, 3), 3, 1.0)
    with pytest.raises(nb.Ne2bError, match="T >= 2"):
        nb.fit_ridge_multi(x[:1], np.zeros(1), 2, 1.0)


def test_reference_readout_cases_on_the_device():
    """The reference's own readout tests (sim/src/readout.rs:310-376) through
    the device solvers: the weights equal the oracle's bit for bit and meet
    the reference's bars (weights 2, -1, bias 0.5 within 1e-3; dual and
    primal scores within 1e-4)."""
    from test_oracle_kats import reference_ridge_dual_case, reference_ridge_linear_case, ridge_output

    x, y = reference_ridge_linear_case()
    w = nb.fit_ridge(x, y, 1e-9)
    assert np.array_equal(w.view(np.uint64), O.fit_ridge(x, y, 1e-9).view(np.uint64))
    assert abs(w[0] - 2.0) < 1e-3 and abs(w[1] + 1.0) < 1e-3 and abs(w[2] - 0.5) < 1e-3, w
    x, lab, k = reference_ridge_dual_case()
    ws = nb.fit_ridge_multi(x, lab, k, 0.7)
    assert np.array_equal(ws.view(np.uint64), O.fit_ridge_multi(x, lab, k, 0.7).view(np.uint64))
    for c in range(k):
        wp = nb.fit_ridge(x, (lab == c).astype(np.float32), 0.7)
        for r in range(x.shape[0]):
            assert abs(ridge_output(wp, x[r]) - ridge_output(ws[c], x[r])) < 1e-4, (c, r)
