"""The CPU restatement of the learned early stop's network (oracle/cnn.py):
its backward pass against finite differences in float64, and the record
helpers of ems_b200/learn.py (example layout, verification, splicing and the
S11 of a spliced record) on analytic signals. CPU only."""
import numpy as np

from ems_b200 import learn as Lr
from oracle import cnn


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    k_in, t_out = 256, 8  # a short input keeps the check fast; the layers are the real ones
    p = Lr.init_params(3, k_in, t_out).astype(np.float64)
    x = rng.standard_normal((3, k_in, 2))
    dout = rng.standard_normal((3, 2 * t_out))
    _, cache = cnn.forward(p, x, t_out, round_bf16=False)
    g = cnn.backward(cache, dout, t_out, round_bf16=False)
    assert g.shape == p.shape
    loss = lambda q: float(np.sum(cnn.forward(q, x, t_out, round_bf16=False)[0] * dout))  # noqa: E731
    idx = rng.choice(p.size, 40, replace=False)
    for q in idx:
        h = 1e-4 * max(1.0, abs(p[q]))
        a, b = p.copy(), p.copy()
        a[q] += h
        b[q] -= h
        fd = (loss(a) - loss(b)) / (2 * h)
        assert abs(fd - g[q]) <= 1e-4 * max(1.0, abs(fd)), (q, fd, g[q])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-39, 65504.0], dtype=np.float32)
    r = cnn.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # halfway, even mantissa kept
    assert r[2] == 1.0078125             # rounds up
    assert r[3] == -2.5
    assert np.all(np.isfinite(r))


def _ringdown(n, f, tau, dt, phase=0.0):
    t = np.arange(n) * dt
    env = np.where(t < 2e-9, t / 2e-9, np.exp(-(t - 2e-9) / tau))
    return env * np.sin(2 * np.pi * f * t + phase)


def test_example_verify_and_splice_on_an_exact_prediction():
    dt = 2e-12
    n = Lr.steps_needed(dt)
    v = _ringdown(n, 2.4e9, 3e-9, dt)
    i = _ringdown(n, 2.4e9, 3e-9, dt, 0.3) / 80.0
    x, y = Lr.example(v, i, dt)
    assert x.shape == (Lr.K_IN, 2) and y.shape == (2 * Lr.T_OUT,)
    d = Lr.verify(y, v, i, dt)
    assert d.stop and d.residual < 1e-6  # the exact tail passes the window check
    d = Lr.verify(0.5 * y, v, i, dt)
    assert not d.stop                    # a wrong tail does not
    stop = Lr.decision_step(dt)
    steps, vv, ii = Lr.spliced(v, i, y, stop, dt)
    assert np.array_equal(steps, np.arange(len(steps))) and np.array_equal(vv[:stop], v[:stop])
    m = len(steps)
    freqs = np.linspace(1e9, 3e9, 41)
    full = Lr.s11_db(np.arange(m), v[:m], i[:m], dt, freqs)
    sp = Lr.s11_db(steps, vv, ii, dt, freqs)
    cut = Lr.s11_db(np.arange(stop), v[:stop], i[:stop], dt, freqs)
    err_sp, err_cut = np.max(np.abs(sp - full)), np.max(np.abs(cut - full))
    assert err_sp < 0.1 and err_cut > 5 * err_sp  # the predicted tail is what makes the early stop exact
