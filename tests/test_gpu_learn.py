"""The learned early stop's CUDA kernels (libems_learn.so) against their CPU
restatements: the bf16 tcgen05 tensor-core GEMM (f32 accumulator in tensor
memory) against numpy on bf16-rounded
operands, im2col/col2im as adjoints, Adam against its formula, and the
network's forward pass and gradients against oracle/cnn.py; then a short
training run that must learn (the loss falls below 40 % of its start)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def _bf16_bits(x):
    from oracle.cnn import bf16

    r = bf16(np.asarray(x, dtype=np.float32)).astype(np.float32)
    return r.view(np.uint32) >> 16, r.astype(np.float64)


@pytest.mark.parametrize("M,N,K,trans_a,trans_b,beta", [
    (64, 64, 32, False, False, 0.0), (100, 37, 70, False, True, 0.0), (5, 300, 513, True, False, 0.5),
    (129, 65, 17, True, True, 1.0), (1, 1, 1, False, False, 0.0), (128, 128, 64, False, False, 0.0),
    (16320, 32, 16, False, True, 0.0), (896, 128, 512, False, True, 0.0), (64, 768, 64, True, False, 0.0),
    (512, 1792, 64, True, False, 1.0)])
def test_gemm_matches_numpy(M, N, K, trans_a, trans_b, beta):
    t = _torch()
    from ems_b200.learn import learn_lib

    lib = learn_lib()
    rng = np.random.default_rng(M * 7 + N)
    a = rng.standard_normal((K, M) if trans_a else (M, K)).astype(np.float32)
    b = rng.standard_normal((N, K) if trans_b else (K, N)).astype(np.float32)
    c0 = rng.standard_normal((M, N)).astype(np.float32)
    ab, af = _bf16_bits(a)
    bb, bf = _bf16_bits(b)
    A = t.from_numpy(ab.astype(np.uint16).view(np.int16)).cuda()
    B = t.from_numpy(bb.astype(np.uint16).view(np.int16)).cuda()
    Cd = t.from_numpy(c0.copy()).cuda()
    sa = (1, M) if trans_a else (K, 1)
    sb = (1, K) if trans_b else (N, 1)
    st = lib.ems_learn_gemm_bf16(A.data_ptr(), sa[0], sa[1], B.data_ptr(), sb[0], sb[1], Cd.data_ptr(), N, M, N, K,
                                 1.0, beta, None)
    assert st == 0
    t.cuda.synchronize()
    assert lib.ems_learn_check() == 0
    want = (af.T if trans_a else af) @ (bf.T if trans_b else bf) + beta * c0
    got = Cd.cpu().numpy()
    err = np.max(np.abs(got - want)) / max(1.0, np.max(np.abs(want)))
    assert err < 1e-5, err  # f32 accumulation of exact bf16 products


def test_im2col_col2im_are_adjoints():
    t = _torch()
    from ems_b200.learn import learn_lib

    lib = learn_lib()
    rng = np.random.default_rng(1)
    B, T, Cc, k, s = 3, 61, 5, 8, 4
    To = (T - k) // s + 1
    x = rng.standard_normal((B, T, Cc)).astype(np.float32)
    x = _bf16_bits(x)[1].astype(np.float32)  # exactly representable, so im2col is exact
    d = rng.standard_normal((B * To, k * Cc)).astype(np.float32)
    X, D = t.from_numpy(x).cuda(), t.from_numpy(d).cuda()
    col = t.empty(B * To * k * Cc, dtype=t.int16, device="cuda")
    dx = t.empty(B * T * Cc, dtype=t.float32, device="cuda")
    assert lib.ems_learn_im2col(X.data_ptr(), col.data_ptr(), B, T, Cc, k, s, None) == 0
    assert lib.ems_learn_col2im(D.data_ptr(), dx.data_ptr(), B, T, Cc, k, s, None) == 0
    t.cuda.synchronize()
    colf = (col.cpu().numpy().astype(np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    from oracle.cnn import col2im, im2col

    assert np.array_equal(colf.reshape(B * To, -1), im2col(x.astype(np.float64), k, s))
    np.testing.assert_allclose(dx.cpu().numpy().reshape(B, T, Cc), col2im(d.astype(np.float64), B, T, Cc, k, s),
                               rtol=1e-6, atol=1e-6)
    lhs = float(np.sum(colf.reshape(B * To, -1) * d))
    rhs = float(np.sum(x * dx.cpu().numpy().reshape(B, T, Cc)))
    assert abs(lhs - rhs) <= 1e-4 * max(1.0, abs(lhs))


def test_adam_matches_formula():
    t = _torch()
    from ems_b200.learn import learn_lib

    lib = learn_lib()
    rng = np.random.default_rng(2)
    n = 1000
    p, g = rng.standard_normal(n).astype(np.float32), rng.standard_normal(n).astype(np.float32)
    m, v = rng.standard_normal(n).astype(np.float32) * 0.1, np.abs(rng.standard_normal(n)).astype(np.float32)
    P, G, Mm, V = (t.from_numpy(a.copy()).cuda() for a in (p, g, m, v))
    Pb = t.empty(n, dtype=t.int16, device="cuda")
    assert lib.ems_learn_adam(P.data_ptr(), Pb.data_ptr(), G.data_ptr(), Mm.data_ptr(), V.data_ptr(), n, 1e-3, 0.9,
                              0.999, 1e-8, 3, None) == 0
    m2 = 0.9 * m + 0.1 * g
    v2 = 0.999 * v + 0.001 * g * g
    p2 = p - 1e-3 * (m2 / (1 - 0.9 ** 3)) / (np.sqrt(v2 / (1 - 0.999 ** 3)) + 1e-8)
    np.testing.assert_allclose(P.cpu().numpy(), p2, rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(Mm.cpu().numpy(), m2, rtol=1e-6, atol=1e-7)


def test_forward_and_gradients_match_the_oracle():
    t = _torch()
    from ems_b200 import learn as Lr
    from oracle import cnn

    rng = np.random.default_rng(3)
    B = 6
    p = Lr.init_params(5)
    net = Lr.Net(p)
    x = rng.standard_normal((B, Lr.K_IN, 2)).astype(np.float32)
    dout = rng.standard_normal((B, 2 * Lr.T_OUT)).astype(np.float32)
    out = net.forward(t.from_numpy(x).cuda()).cpu().numpy()
    net.backward(t.from_numpy(dout).cuda())
    g = net.g.cpu().numpy()
    want, cache = cnn.forward(p, x, Lr.T_OUT)
    gw = cnn.backward(cache, dout, Lr.T_OUT)
    assert np.linalg.norm(out - want) / np.linalg.norm(want) < 5e-3
    o = 0
    for (name, co, fi) in Lr.layer_shapes()[0]:
        for part, size in (("W", co * fi), ("b", co)):
            a, b = g[o:o + size], gw[o:o + size]
            o += size
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
            assert rel < 2e-2, (name, part, rel)


def test_training_reduces_the_loss():
    """Damped sinusoids of random frequency, decay and phase: the network
    learns their continuation (in 400 Adam steps the loss falls below 40 %
    of the loss of the untrained network, whose output is near zero)."""
    t = _torch()
    from ems_b200 import learn as Lr

    rng = np.random.default_rng(4)
    dt = 4e-12
    n = Lr.steps_needed(dt)
    X, Y = [], []
    for _ in range(256):
        f, tau, ph = rng.uniform(1.5e9, 3e9), rng.uniform(2e-9, 10e-9), rng.uniform(0, 2 * np.pi)
        tt = np.arange(n) * dt
        env = np.where(tt < 1e-9, tt / 1e-9, np.exp(-(tt - 1e-9) / tau))
        v = env * np.sin(2 * np.pi * f * tt + ph)
        i = env * np.sin(2 * np.pi * f * tt + ph + 0.4) * 0.02
        x, y = Lr.example(v, i, dt)
        X.append(x)
        Y.append(y)
    X, Y = t.from_numpy(np.stack(X)).cuda(), t.from_numpy(np.stack(Y)).cuda()
    net = Lr.Net(seed=1)
    losses = []
    for step in range(400):
        sel = t.from_numpy(rng.choice(256, 32, replace=False)).cuda()
        loss = net.train_step(X[sel], Y[sel], lr=1e-3)
        if step % 50 == 0 or step == 399:
            losses.append(float(loss.item()))
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.4 * losses[0], losses
