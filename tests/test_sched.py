"""The learned scheduler: its cost model's gradient (CPU oracle pinned by
finite differences; the GPU training kernels against the oracle), training
from the engine's own timing samples, and results that do not depend on the
schedule."""
import ctypes

import numpy as np
import pytest

from oracle import mlp_oracle
from tagmatch_b200 import TagMatch, _native, workload


def test_oracle_gradient_matches_finite_differences():
    r = np.random.default_rng(3)
    p = mlp_oracle.init(7)
    x = r.random((40, 8))
    t = r.standard_normal(40)
    _, g, _ = mlp_oracle.loss_grad(p, x, t)
    idx = np.concatenate([r.choice(mlp_oracle.N_PARAMS, 60, replace=False), [mlp_oracle.B3, mlp_oracle.W3]])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mlp_oracle.loss(pp, x, t) - mlp_oracle.loss(pm, x, t)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_param_count_matches_header_layout():
    assert _native.load().tm_mlp_param_count() == mlp_oracle.N_PARAMS


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 127, 128, 300, 1000])
def test_gpu_gradient_matches_oracle(n):
    """Forward outputs and the mean-squared-error gradient of the GPU kernels
    (fp32) against the float64 oracle: relative error <= 1e-3 of the
    gradient's norm per parameter, and every output within 1e-4."""
    from tagmatch_b200.tagmatch import mlp_loss_grad
    r = np.random.default_rng(n)
    p = mlp_oracle.init(n)
    x = r.random((n, 8))
    t = r.standard_normal(n)
    y, g, loss = mlp_loss_grad(p.astype(np.float32), x.astype(np.float32), t.astype(np.float32))
    ey, eg, eloss = mlp_oracle.loss_grad(p.astype(np.float32).astype(np.float64), x.astype(np.float32), t.astype(np.float32))
    assert np.allclose(y, ey, rtol=1e-4, atol=1e-4)
    assert abs(loss - eloss) <= 1e-4 * max(1.0, eloss)
    scale = np.linalg.norm(eg)
    assert np.max(np.abs(g - eg)) <= 1e-3 * scale, (np.max(np.abs(g - eg)), scale)
    # a gradient step on the GPU's gradient lowers the oracle's loss
    assert mlp_oracle.loss(p - 1e-3 * g / scale, x, t) < eloss


@pytest.mark.gpu
def test_trained_scheduler_keeps_results_and_predicts():
    """Timing samples from the engine's own batches train the cost model on
    the GPU; the learned work-queue order changes no result; the model beats
    predicting the mean on held-out samples."""
    f, ko, k = workload.generate_filters(400_000, 61)
    q = workload.generate_queries(60_000, f, 61)
    tm = TagMatch()
    tm.set_persistence(False)
    tm.add_many(f, ko, k)
    tm.consolidate(4096, 1)
    tm.sched_record(True)
    off0 = keys0 = None
    for seg, b in ((64, 4096), (256, 8192), (1024, 16384), (8192, 30000), (128, 60000)):
        tm.set_tiles_per_item(seg)
        tm.set_batch_limit(b)
        off, keys = tm.match_batch(q)
        if off0 is None:
            off0, keys0 = off, keys
    tm.sched_record(False)
    x, t = tm.sched_samples()
    assert x.shape[0] > 1000 and np.all(np.isfinite(x)) and np.all(np.isfinite(t))
    rep = tm.sched_train(epochs=30)
    assert rep["samples"] == x.shape[0] and rep["steps"] > 0
    assert rep["val_mse"] < 0.5 * rep["mean_mse"], rep
    assert tm.sched_predict_batch_ms(16384) > 0
    tm.sched_use_order(True)
    tm.set_tiles_per_item(256)
    off1, keys1 = tm.match_batch(q)
    assert np.array_equal(off0, off1)
    for i in range(0, q.shape[0], 37):
        assert np.array_equal(np.sort(keys0[off0[i]:off0[i + 1]]), np.sort(keys1[off1[i]:off1[i + 1]]))
    tm.close()


@pytest.mark.gpu
def test_learned_flush_mode_same_results():
    """Serving in the learned flush mode: every request's result equals the
    same queries matched alone."""
    import threading
    f, ko, k = workload.generate_filters(50_000, 62)
    q = workload.generate_queries(4000, f, 62)
    tm = TagMatch()
    tm.set_persistence(False)
    tm.add_many(f, ko, k)
    tm.consolidate(4096, 1)
    tm.sched_record(True)
    for b in (256, 1024, 4000):
        tm.set_batch_limit(b)
        tm.match_batch(q)
    tm.sched_train(epochs=20)
    tm.set_batch_limit(65536)
    tm.set_flush_mode(_native.TM_FLUSH_LEARNED)
    tm.set_latency_target_ms(20)
    tm.start()
    rng = np.random.default_rng(9)
    reqs, at = [], 0
    while at < q.shape[0]:
        n = int(min(q.shape[0] - at, rng.integers(1, 500)))
        reqs.append((at, n))
        at += n
    got, lock = {}, threading.Lock()

    def handler(i):
        def h(off, keys, status):
            with lock:
                got[i] = (off.copy(), keys.copy(), status)
        return h
    for i, (a, n) in enumerate(reqs):
        tm.submit(q[a:a + n], handler(i))
    tm.stop()
    assert len(got) == len(reqs)
    for i, (a, n) in enumerate(reqs):
        off, keys, st = got[i]
        assert st == 0
        eo, ek = tm.match_batch(q[a:a + n])
        assert np.array_equal(off, eo)
        for j in range(n):
            assert np.array_equal(np.sort(keys[off[j]:off[j + 1]]), np.sort(ek[eo[j]:eo[j + 1]]))
    tm.close()
