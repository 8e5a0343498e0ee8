"""Surrogate start of the rate-dependent return mapping on the GPU.

The network kernels (forward, backward, Adam, tensor-core inference) are
checked against the oracle's FP64 network; the resident loop with the
learned start is checked against the plain Newton path it replaces (same
answer to the Newton tolerance, fewer iterations) and against the oracle.
"""
import numpy as np
import pytest

from taylor_b200 import _lib, cases, mega

from oracle import oracle as O

pytestmark = pytest.mark.gpu

RATE_LAW = (90e6, 292e6, 0.31, 0.025, 1.0)  # A, B, n, C, epsdot0


def _features(n, seed):
    rng = np.random.default_rng(seed)
    x = np.empty((n, 4), np.float32)
    x[:, 0] = rng.uniform(-8.0, 0.5, n)
    x[:, 1] = rng.uniform(0.0, 0.8, n)
    x[:, 2] = rng.uniform(0.0, 1.4, n)
    x[:, 3] = rng.uniform(0.5, 1.5, n)
    return x


def _theta(seed):
    th = mega.mlp_init(seed)
    rng = np.random.default_rng(seed + 100)
    return (th + rng.normal(0.0, 0.05, th.shape)).astype(np.float32)  # non-zero biases too


def test_mlp_gradient_matches_oracle():
    th = _theta(1)
    x = _features(1000, 2)
    t = np.random.default_rng(3).uniform(0.05, 1.0, 1000).astype(np.float32)
    loss, g = mega.mlp_grad(th, x, t)
    lo, _, go = O.mlp_forward_backward(64, th.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - lo) <= 1e-5 * abs(lo)
    # FP32 forward / backward with block-partial sums vs FP64
    assert np.linalg.norm(g - go) <= 1e-4 * np.linalg.norm(go)
    assert np.abs(g - go).max() <= 1e-4 * np.abs(go).max()


def test_mlp_eval_fp32_and_tensor_cores_match_oracle():
    th = _theta(4)
    x = _features(1000 + 7, 5)  # a partial last warp
    _, yo, _ = O.mlp_forward_backward(64, th.astype(np.float64), x.astype(np.float64), None, grad=False)
    y32 = mega.mlp_eval(th, x)
    assert np.abs(y32 - yo).max() <= 1e-5 * (1.0 + np.abs(yo).max())
    ytc = mega.mlp_eval(th, x, tensor_cores=True)
    # bf16 hidden activations and W2 (8-bit mantissa), fp32 accumulation
    err = np.abs(ytc - yo)
    assert err.max() <= 2e-2 * (1.0 + np.abs(yo).max())
    assert err.mean() <= 4e-3 * (1.0 + np.abs(yo).max())


def test_mlp_training_fits_a_smooth_map():
    x = _features(20000, 6)
    t = (0.5 + 0.3 * np.tanh(0.5 * x[:, 0] + 1.0) - 0.2 * x[:, 1] + 0.1 * x[:, 2]).astype(np.float32)
    th0 = mega.mlp_init(7)
    l0, _ = mega.mlp_grad(th0, x, t)
    th, loss = mega.mlp_train(th0, x, t, epochs=30, batch=1024, lr=2e-3, seed=8)
    assert np.all(np.isfinite(loss))
    l1, _ = mega.mlp_grad(th, x, t)
    assert l1 <= 0.02 * l0
    assert loss[-1] <= 0.2 * loss[0]
    # one Adam step agrees with the oracle's Adam on the same gradient
    g = mega.mlp_grad(th0, x[:1024], t[:1024])[1]
    th_gpu, _ = mega.mlp_train(th0, x[:1024], t[:1024], epochs=1, batch=1024, lr=1e-3, seed=9)
    ref = th0.astype(np.float64).copy()
    m = np.zeros_like(ref)
    v = np.zeros_like(ref)
    O.adam(ref, g.astype(np.float64), m, v, 1e-3, 1)
    # the batch is the whole set, so the shuffle only reorders the gradient
    # sum; the first Adam step is lr g / (|g| + eps), whose sign is only
    # defined where g stands clear of the float summation noise
    big = np.abs(g) > 1e-4 * np.abs(g).max()
    assert big.mean() > 0.5
    assert np.abs(th_gpu - ref)[big].max() <= 1e-5
    assert np.abs(th_gpu - th0).max() <= 1.001e-3


def _rate_case(h=0.4e-3):
    return cases.taylor_bar(h=h, rate_law=RATE_LAW)


def _params(c, **kw):
    return _lib.params(**cases.param_kwargs(c, newton_max_iter=60, **kw))


def test_rate_law_resident_matches_oracle():
    c = _rate_case(0.8e-3)
    m = mega.Mega(c, _params(c))
    m.search_and_shapes()
    r = O.Run(c, O.params(**cases.param_kwargs(c, newton_max_iter=60)), nthreads=8)
    dt = cases.stable_dt(c, r.nb["gn"], r.nb["gstart"], r.nb["gstack"])
    m.step(60, dt)
    r.step(60, dt)
    eps = m.download(_lib.F_EPS)
    assert r.state[:, 2].max() > 0.0
    assert np.abs(eps - r.state[:, 2]).max() <= 1e-6 * r.state[:, 2].max()
    x = m.download(_lib.F_COO_CURRENT)
    uo = r.coo_cur.reshape(-1, 3) - c["coo"]
    assert np.abs(x - c["coo"] - uo).max() <= 1e-7 * np.abs(uo).max()
    m.close()


def test_learned_start_same_answer_fewer_iterations():
    """Plain Newton logs samples for 120 steps, the network trains on them on
    the device, then two copies continue from the same state: plain and
    learned start.  Newton polishes both to the same tolerance."""
    c = _rate_case()
    plain = mega.Mega(c, _params(c))
    learn = mega.Mega(c, _params(c))
    plain.search_and_shapes()
    learn.search_and_shapes()
    dt = 3.5e-8
    learn.log_rate_samples(cap=1 << 20, stride=1, seed=11)
    plain.step(120, dt, mode="mixed")
    learn.step(120, dt, mode="mixed")
    samples = learn.rate_samples()
    assert len(samples) > 10000
    assert np.all(np.isfinite(samples))
    assert samples[:, 4].min() > 0.0 and samples[:, 4].max() <= 1.0 + 1e-6
    th, loss = learn.train_surrogate(mega.mlp_init(12), epochs=40, batch=2048, lr=2e-3, seed=13)
    assert loss[-1] < 0.25 * loss[0]
    learn.log_rate_samples(0)
    it_plain = it_learn = pl_plain = pl_learn = 0
    for _ in range(40):
        plain.step(1, dt, mode="mixed")
        learn.step(1, dt, mode="mixed", learned=True)
        sp, sl = plain.scalars(), learn.scalars()
        it_plain += sp["newton_iters"]
        it_learn += sl["newton_iters"]
        pl_plain += sp["plastic_nodes"]
        pl_learn += sl["plastic_nodes"]
    assert pl_plain > 0 and abs(pl_plain - pl_learn) <= 0.01 * pl_plain
    # the iteration-count reduction the learned start buys
    assert it_learn <= 0.8 * it_plain, (it_plain / pl_plain, it_learn / pl_learn)
    ep, el = plain.download(_lib.F_EPS), learn.download(_lib.F_EPS)
    assert np.abs(el - ep).max() <= 1e-6 * ep.max()
    xp, xl = plain.download(_lib.F_COO_CURRENT), learn.download(_lib.F_COO_CURRENT)
    assert np.abs(xl - xp).max() <= 1e-6 * np.abs(xp - c["coo"]).max()
    plain.close()
    learn.close()


def test_learned_flag_without_network_is_refused():
    c = _rate_case(0.8e-3)
    m = mega.Mega(c, _params(c))
    m.search_and_shapes()
    with pytest.raises(_lib.MegaError):
        m.step(2, 3.5e-8, mode="mixed", learned=True)
    m.close()
