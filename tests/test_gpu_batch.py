"""Batched chains (one persistent launch per (parity, mu) phase for all chains, CUDA-graph sweeps)
against separate single-chain runs through the C ABI."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LS = [(4, 4, 4, 4), (4, 4, 4, 4), (6, 6, 6, 6), (4, 6, 2, 8), (8, 8, 8, 8)]
BETAS = [5.7, 6.3, 6.0, 5.9, 6.1]
SEEDS = [0, 1, 2, 3, 4]


def single_runs(gpu, n_hits, n_sweeps, prec=64, store=0):
    out = []
    for L, b, s in zip(LS, BETAS, SEEDS):
        f = gpu.GaugeField(L, prec, store)
        f.hot_start(s)
        for k in range(n_sweeps):
            f.hb_sweep(b, n_hits, s, k)
        out.append((f.download(), f.plaquette()))
    return out


def test_batch_matches_single_chains(gpu):
    b = gpu.Batch(LS, BETAS, SEEDS)
    b.hot_start()
    b.sweep(2, 3)
    plaq = b.plaquette()
    ref = single_runs(gpu, 2, 3)
    for i, (U, p) in enumerate(ref):
        assert np.max(np.abs(b.download(i) - U)) < 1e-12, i
        assert abs(plaq[i] - p) < 1e-12, i
    assert b.info()["sweep"] == 3


def test_graph_replay_equals_single_calls(gpu):
    a = gpu.Batch(LS, BETAS, SEEDS)
    a.hot_start()
    a.sweep(1, 4)
    c = gpu.Batch(LS, BETAS, SEEDS)
    c.hot_start()
    for _ in range(4):
        c.sweep(1, 1)
    for i in range(len(LS)):
        assert np.array_equal(a.download(i), c.download(i))


@pytest.mark.parametrize("variant", [0, 2])
def test_launch_shape_does_not_change_results(gpu, variant):
    a = gpu.Batch(LS, BETAS, SEEDS)
    a.hot_start()
    a.sweep(1, 2)
    c = gpu.Batch(LS, BETAS, SEEDS)
    c.set_variant(variant)
    c.hot_start()
    c.sweep(1, 2)
    for i in range(len(LS)):
        assert np.array_equal(a.download(i), c.download(i))


def test_tuner_sweeps_are_ordinary_sweeps(gpu):
    t = gpu.Batch(LS, BETAS, SEEDS)
    t.hot_start()
    v, ms = t.tune(1, n_trial=1)
    assert 0 <= v <= 2 and all(x > 0 for x in ms[:3])
    n = t.info()["sweep"]
    assert n == 3 * 2  # per shape: one warm-up + n_trial sweeps
    r = gpu.Batch(LS, BETAS, SEEDS)
    r.hot_start()
    r.sweep(1, n)
    for i in range(len(LS)):
        assert np.array_equal(t.download(i), r.download(i))


def test_tuner_storage_change_keeps_state(gpu):
    t = gpu.Batch(LS, BETAS, SEEDS)
    t.hot_start()
    t.sweep(1, 1)
    before = [t.download(i) for i in range(len(LS))]
    v, ms = t.tune(1, n_trial=1, allow_store_change=True)
    assert ms[3] > 0
    info = t.info()
    # whichever storage won, the chains continue from the state reached by the tuning sweeps
    assert info["sweep"] == 1 + 3 * 2
    for i in range(len(LS)):
        assert t.download(i).shape == before[i].shape
    t.sweep(1, 1)
    assert np.all(np.isfinite(t.plaquette()))


def test_fp32_batch_stays_unitary(gpu):
    b = gpu.Batch(LS, BETAS, SEEDS, prec=32)
    b.hot_start()
    b.sweep(2, 5)
    for i in range(len(LS)):
        U = b.download(i).reshape(-1, 3, 3)
        err = np.abs(U @ np.conj(np.swapaxes(U, 1, 2)) - np.eye(3)).max()
        assert err < 1e-6
    ref = single_runs(gpu, 2, 5, prec=32)
    for i, (U, p) in enumerate(ref):
        assert np.max(np.abs(b.download(i) - U)) < 1e-5


def test_batch_invalid_arguments(gpu):
    with pytest.raises(gpu.QcbError):
        gpu.Batch([(5, 4, 4, 4)], [6.0], [0])
    with pytest.raises(gpu.QcbError):
        gpu.Batch([(4, 4, 4, 4)], [-1.0], [0])
    b = gpu.Batch([(4, 4, 4, 4)], [6.0], [0])
    with pytest.raises(gpu.QcbError):
        b.set_variant(7)


def test_fp64_twelve_real_chains_stay_on_su3(gpu):
    """12-real storage rebuilds the third row as conj(r0 x r1), which is SU(3) only for orthonormal
    rows; every update therefore reprojects in FP64.  Without it the stored rows' norm errors grow
    from sweep to sweep (a 16^4 FP64 chain of a 256-chain batch diverged after ~180 sweeps)."""
    n = 32
    b = gpu.Batch([(8, 8, 8, 8)] * n, [5.7] * n, list(range(500, 500 + n)), prec=64, store=1)
    b.hot_start()
    b.sweep(1, 300)
    p = b.plaquette()
    assert np.all(np.isfinite(p)) and np.all((p > 0.5) & (p < 0.6))
    for i in range(n):
        V = b.download(i).reshape(-1, 3, 3)
        assert np.abs(V @ np.conj(np.swapaxes(V, 1, 2)) - np.eye(3)).max() < 1e-12
