"""Learned early stop: a 1-D CNN that predicts a port's ring-down.

No counterpart in the reference, which ends a run by its energy criterion
(src/engine/run.rs:231-262) or by the Settle spectral-tail rule
(src/engine/run.rs:309-382). Here a small network reads a lumped port's
voltage and current over the first K_IN·DT_REF of a run (K_IN samples,
over the amplitude the input ends with, asinh-compressed) and predicts the rest of the
ring-down, T_OUT samples per signal spaced STRIDE·DT_REF. A run stops once
the samples of a short window after the input have arrived, when they
agree with the prediction within a threshold; otherwise it runs on to the
energy criterion as it would have without the network. The port's spectrum, and so Z_in/S11, is
then taken from the live samples followed by the predicted tail.

Layers (channels-last activations, weights W[out][fan_in]):

    conv 2→32, kernel 8, stride 4, SiLU    (K_IN 2048 → 511)
    conv 32→64, kernel 8, stride 4, SiLU   (511 → 126)
    conv 64→128, kernel 8, stride 4, SiLU  (126 → 30)
    dense 3840→64, SiLU
    dense 64→2·T_OUT                       (V then I)

about 0.38 M parameters. Every layer runs on the kernels of
libems_learn.so (include/ems_learn.h): im2col, the bf16 tcgen05
tensor-core GEMM (f32 accumulator in tensor memory), bias + activation, their adjoints, MSE and Adam; the
f32 master weights are copied to bf16 for the GEMMs. torch only holds the
device buffers and the stream.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

K_IN = 2048      # samples of V and I the network reads
T_OUT = 384      # predicted samples per signal
DT_REF = 6.4e-12  # [s] spacing of the input samples (K_IN of them: 13.1 ns)
STRIDE = 16      # spacing of the predicted samples, in DT_REF (102.4 ps; 39 ns of ring-down)
WINDOW = 4 * STRIDE  # verification window after the input, in DT_REF
CONVS = [(2, 32, 8, 4), (32, 64, 8, 4), (64, 128, 8, 4)]  # (c_in, c_out, kernel, stride)
HIDDEN = 64

_lib = None


def learn_lib() -> C.CDLL:
    """The learned early stop's kernels. Raises if missing: there is no CPU path."""
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "libems_learn.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: build it (python -m ems_b200.build)")
        L = C.CDLL(path)
        p, i, f, sz, i64 = C.c_void_p, C.c_int, C.c_float, C.c_size_t, C.c_int64
        sig = {
            "ems_learn_gemm_bf16": [p, i64, i64, p, i64, i64, p, i64, i, i, i, f, f, p],
            "ems_learn_to_bf16": [p, p, sz, p],
            "ems_learn_im2col": [p, p, i, i, i, i, i, p],
            "ems_learn_col2im": [p, p, i, i, i, i, i, p],
            "ems_learn_bias_act": [p, p, p, i, i, i, p],
            "ems_learn_act_grad": [p, p, p, i, i, i, p],
            "ems_learn_bias_grad": [p, p, i, i, p],
            "ems_learn_mse": [p, p, p, p, sz, p],
            "ems_learn_adam": [p, p, p, p, p, sz, f, f, f, f, i, p],
            "ems_learn_check": [],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.restype = C.c_int
            fn.argtypes = args
        _lib = L
    return _lib


def layer_shapes(k_in: int = K_IN, t_out: int = T_OUT):
    """(name, out, fan_in) of every layer and the sequence lengths."""
    shapes, T = [], [k_in]
    for q, (ci, co, k, s) in enumerate(CONVS):
        shapes.append((f"conv{q + 1}", co, k * ci))
        T.append((T[-1] - k) // s + 1)
    flat = T[-1] * CONVS[-1][1]
    shapes.append(("fc1", HIDDEN, flat))
    shapes.append(("fc2", 2 * t_out, HIDDEN))
    return shapes, T


def init_params(seed: int = 0, k_in: int = K_IN, t_out: int = T_OUT) -> np.ndarray:
    """Flat f32 parameters: per layer W[out][fan_in] then b[out]; He-normal
    weights (the output layer scaled by 0.1), zero biases."""
    rng = np.random.default_rng(seed)
    shapes, _ = layer_shapes(k_in, t_out)
    parts = []
    for q, (_, co, fi) in enumerate(shapes):
        std = math.sqrt(2.0 / fi) * (0.1 if q == len(shapes) - 1 else 1.0)
        parts.append((rng.standard_normal((co, fi)) * std).astype(np.float32).ravel())
        parts.append(np.zeros(co, dtype=np.float32))
    return np.concatenate(parts)


def param_views(flat, k_in: int = K_IN, t_out: int = T_OUT):
    """(W, b) views of a flat parameter array (numpy or torch) per layer."""
    shapes, _ = layer_shapes(k_in, t_out)
    out, o = [], 0
    for _, co, fi in shapes:
        W = flat[o:o + co * fi].reshape(co, fi)
        o += co * fi
        b = flat[o:o + co]
        o += co
        out.append((W, b))
    return out


class Net:
    """The network on one CUDA device, with its training state."""

    def __init__(self, params: np.ndarray | None = None, device: int = 0, seed: int = 0, k_in: int = K_IN,
                 t_out: int = T_OUT):
        import torch

        self.torch = torch
        self.lib = learn_lib()
        self.dev = f"cuda:{device}"
        self.k_in, self.t_out = k_in, t_out
        self.shapes, self.T = layer_shapes(k_in, t_out)
        p = init_params(seed, k_in, t_out) if params is None else np.asarray(params, dtype=np.float32)
        self.p = torch.from_numpy(p.copy()).to(self.dev)
        self.pb = torch.empty(self.p.numel(), dtype=torch.int16, device=self.dev)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.t = 0
        self._ck(self.lib.ems_learn_to_bf16(self._ptr(self.p), self._ptr(self.pb), self.p.numel(), self._s()))
        self.W = param_views(self.p, k_in, t_out)
        self.Wb = param_views(self.pb, k_in, t_out)
        self.G = param_views(self.g, k_in, t_out)
        self._buf_b = -1

    # -- plumbing
    def _ptr(self, t) -> int:
        return t.data_ptr()

    def _s(self) -> int:
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    @staticmethod
    def _ck(st: int) -> None:
        if st != 0:
            raise RuntimeError(f"ems_learn call failed ({st})")

    def _gemm(self, A, sa0, sa1, B, sb0, sb1, Cm, ldc, M, N, K, beta=0.0):
        self._ck(self.lib.ems_learn_gemm_bf16(A, sa0, sa1, B, sb0, sb1, Cm, ldc, M, N, K, 1.0, beta, self._s()))

    def _bufs(self, B: int):
        """Activation buffers for batch size B."""
        if self._buf_b == B:
            return
        t = self.torch
        f32, bf = dict(dtype=t.float32, device=self.dev), dict(dtype=t.int16, device=self.dev)
        self.cols, self.ys, self.acts, self.dys, self.dcols, self.das = [], [], [], [], [], []
        for q, (ci, co, k, s) in enumerate(CONVS):
            rows = B * self.T[q + 1]
            self.cols.append(t.empty(rows * k * ci, **bf))
            self.ys.append(t.empty(rows * co, **f32))
            self.acts.append(t.empty(rows * co, **f32))
            self.dys.append(t.empty(rows * co, **f32))
            self.dcols.append(t.empty(rows * k * ci, **f32))
            self.das.append(t.empty(B * self.T[q] * ci, **f32))
        flat = self.shapes[3][2]
        self.flat_b = t.empty(B * flat, **bf)
        self.y4 = t.empty(B * HIDDEN, **f32)
        self.a4 = t.empty(B * HIDDEN, **f32)
        self.a4_b = t.empty(B * HIDDEN, **bf)
        self.y5 = t.empty(B * 2 * self.t_out, **f32)
        self.out = t.empty(B * 2 * self.t_out, **f32)
        self.dy5 = t.empty(B * 2 * self.t_out, **f32)
        self.dy5_b = t.empty(B * 2 * self.t_out, **bf)
        self.da4 = t.empty(B * HIDDEN, **f32)
        self.dy4 = t.empty(B * HIDDEN, **f32)
        self.dy4_b = t.empty(B * HIDDEN, **bf)
        self.da3 = t.empty(B * flat, **f32)
        self.dy_b = [t.empty(B * self.T[q + 1] * CONVS[q][1], **bf) for q in range(len(CONVS))]
        self.loss = t.zeros(1, **f32)
        self._buf_b = B

    # -- forward / backward
    def forward(self, x):
        """x: (B, k_in, 2) f32 on the device → (B, 2·t_out)."""
        B = x.shape[0]
        self._bufs(B)
        L, s = self.lib, self._s()
        inp = x.contiguous()
        for q, (ci, co, k, st) in enumerate(CONVS):
            T = self.T[q]
            rows, fi = B * self.T[q + 1], k * ci
            self._ck(L.ems_learn_im2col(self._ptr(inp), self._ptr(self.cols[q]), B, T, ci, k, st, s))
            Wb, _ = self.Wb[q]
            self._gemm(self._ptr(self.cols[q]), fi, 1, self._ptr(Wb), 1, fi, self._ptr(self.ys[q]), co, rows, co, fi)
            self._ck(L.ems_learn_bias_act(self._ptr(self.ys[q]), self._ptr(self.W[q][1]), self._ptr(self.acts[q]),
                                          rows, co, 1, s))
            inp = self.acts[q]
        flat = self.shapes[3][2]
        self._ck(L.ems_learn_to_bf16(self._ptr(inp), self._ptr(self.flat_b), B * flat, s))
        self._gemm(self._ptr(self.flat_b), flat, 1, self._ptr(self.Wb[3][0]), 1, flat, self._ptr(self.y4), HIDDEN,
                   B, HIDDEN, flat)
        self._ck(L.ems_learn_bias_act(self._ptr(self.y4), self._ptr(self.W[3][1]), self._ptr(self.a4), B, HIDDEN, 1, s))
        self._ck(L.ems_learn_to_bf16(self._ptr(self.a4), self._ptr(self.a4_b), B * HIDDEN, s))
        no = 2 * self.t_out
        self._gemm(self._ptr(self.a4_b), HIDDEN, 1, self._ptr(self.Wb[4][0]), 1, HIDDEN, self._ptr(self.y5), no, B,
                   no, HIDDEN)
        self._ck(L.ems_learn_bias_act(self._ptr(self.y5), self._ptr(self.W[4][1]), self._ptr(self.out), B, no, 0, s))
        return self.out.view(B, no)

    def backward(self, dout):
        """Gradients of the last forward's output dout (B, 2·t_out) → self.g."""
        B = dout.shape[0]
        L, s = self.lib, self._s()
        no, flat = 2 * self.t_out, self.shapes[3][2]
        # fc2 (identity activation): dW5 = dy5ᵀ a4, db5, da4 = dy5 W5.
        self.dy5.copy_(dout.reshape(-1))
        self._ck(L.ems_learn_to_bf16(self._ptr(self.dy5), self._ptr(self.dy5_b), B * no, s))
        self._gemm(self._ptr(self.dy5_b), 1, no, self._ptr(self.a4_b), HIDDEN, 1, self._ptr(self.G[4][0]), HIDDEN, no,
                   HIDDEN, B)
        self._ck(L.ems_learn_bias_grad(self._ptr(self.dy5), self._ptr(self.G[4][1]), B, no, s))
        self._gemm(self._ptr(self.dy5_b), no, 1, self._ptr(self.Wb[4][0]), HIDDEN, 1, self._ptr(self.da4), HIDDEN, B,
                   HIDDEN, no)
        # fc1.
        self._ck(L.ems_learn_act_grad(self._ptr(self.y4), self._ptr(self.da4), self._ptr(self.dy4), B, HIDDEN, 1, s))
        self._ck(L.ems_learn_to_bf16(self._ptr(self.dy4), self._ptr(self.dy4_b), B * HIDDEN, s))
        self._gemm(self._ptr(self.dy4_b), 1, HIDDEN, self._ptr(self.flat_b), flat, 1, self._ptr(self.G[3][0]), flat,
                   HIDDEN, flat, B)
        self._ck(L.ems_learn_bias_grad(self._ptr(self.dy4), self._ptr(self.G[3][1]), B, HIDDEN, s))
        self._gemm(self._ptr(self.dy4_b), HIDDEN, 1, self._ptr(self.Wb[3][0]), flat, 1, self._ptr(self.da3), flat, B,
                   flat, HIDDEN)
        # convolutions, last to first.
        da = self.da3
        for q in range(len(CONVS) - 1, -1, -1):
            ci, co, k, st = CONVS[q]
            rows, fi = B * self.T[q + 1], k * ci
            self._ck(L.ems_learn_act_grad(self._ptr(self.ys[q]), self._ptr(da), self._ptr(self.dys[q]), rows, co, 1, s))
            self._ck(L.ems_learn_to_bf16(self._ptr(self.dys[q]), self._ptr(self.dy_b[q]), rows * co, s))
            self._gemm(self._ptr(self.dy_b[q]), 1, co, self._ptr(self.cols[q]), fi, 1, self._ptr(self.G[q][0]), fi, co,
                       fi, rows)
            self._ck(L.ems_learn_bias_grad(self._ptr(self.dys[q]), self._ptr(self.G[q][1]), rows, co, s))
            if q == 0:
                break
            self._gemm(self._ptr(self.dy_b[q]), co, 1, self._ptr(self.Wb[q][0]), fi, 1, self._ptr(self.dcols[q]), fi,
                       rows, fi, co)
            self._ck(L.ems_learn_col2im(self._ptr(self.dcols[q]), self._ptr(self.das[q]), B, self.T[q], ci, k, st, s))
            da = self.das[q]

    def adam(self, lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8) -> None:
        self.t += 1
        self._ck(self.lib.ems_learn_adam(self._ptr(self.p), self._ptr(self.pb), self._ptr(self.g), self._ptr(self.m),
                                         self._ptr(self.v), self.p.numel(), lr, b1, b2, eps, self.t, self._s()))

    def train_step(self, x, y, lr: float = 1e-3) -> float:
        """One Adam step on a minibatch; returns the loss (MSE)."""
        out = self.forward(x)
        grad = self.torch.empty_like(out)
        self._ck(self.lib.ems_learn_mse(self._ptr(out), self._ptr(y), self._ptr(grad), self._ptr(self.loss),
                                        out.numel(), self._s()))
        self.backward(grad)
        self.adam(lr)
        return self.loss

    def params(self) -> np.ndarray:
        return self.p.detach().cpu().numpy()


# ---------------------------------------------------------------------------
# Data: port records → network inputs and targets, on a fixed time grid.
#
# The network works in physical time, whatever a model's time step: its
# input is V and I at t_k = (k + 1)·DT_REF (k < K_IN), its output the tail
# at t = (K_IN + STRIDE·(q + 1))·DT_REF (q < T_OUT), both interpolated
# (cubic) from the port series, V sampled at (n + 1)·dt and I at
# (n + ½)·dt for step n (src/engine/port.rs:191-205).

def _at(x: np.ndarray, dt: float, half: bool, t: np.ndarray) -> np.ndarray:
    """x (one sample per step) at times t, linearly interpolated (a record
    has 80 or more samples per period of the band here)."""
    n = np.arange(len(x), dtype=np.float64)
    return np.interp(t, (n + (0.5 if half else 1.0)) * dt, x)


def steps_needed(dt: float, k_in: int = K_IN, t_out: int = T_OUT, stride: int = STRIDE) -> int:
    """Steps a record needs to cover the input and the predicted tail."""
    return int(math.ceil((k_in + stride * t_out) * DT_REF / dt)) + 2


def decision_step(dt: float, k_in: int = K_IN, window: int = WINDOW) -> int:
    """The step after which the window's samples have all arrived."""
    return int(math.ceil((k_in + window) * DT_REF / dt)) + 2


def tail_times(k_in: int = K_IN, t_out: int = T_OUT, stride: int = STRIDE) -> np.ndarray:
    return (k_in + stride * (np.arange(t_out) + 1)) * DT_REF


TAIL_RMS = 128  # input samples whose RMS sets a signal's scale


def normalise(vk: np.ndarray, ik: np.ndarray):
    """Scales of V and I: their RMS over the last TAIL_RMS input samples,
    the amplitude the ring-down continues from."""
    sv = float(np.sqrt(np.mean(vk[-TAIL_RMS:] ** 2))) or 1.0
    si = float(np.sqrt(np.mean(ik[-TAIL_RMS:] ** 2))) or 1.0
    return sv, si


def example_input(v: np.ndarray, i: np.ndarray, dt: float, k_in: int = K_IN):
    """The network input of a record, (k_in, 2), and the scales: the input
    samples over their scale, compressed by asinh (the excitation is orders
    of magnitude above the ring-down it leaves)."""
    t = (np.arange(k_in) + 1.0) * DT_REF
    vk, ik = _at(v, dt, False, t), _at(i, dt, True, t)
    sv, si = normalise(vk, ik)
    return np.stack([np.arcsinh(vk / sv), np.arcsinh(ik / si)], axis=1).astype(np.float32), (sv, si)


def example(v: np.ndarray, i: np.ndarray, dt: float, k_in: int = K_IN, t_out: int = T_OUT, stride: int = STRIDE):
    """(x (k_in, 2), y (2·t_out,)) of one record of at least steps_needed(dt)
    steps: the tail of V, then of I, over the input's scales (linear)."""
    x, (sv, si) = example_input(v, i, dt, k_in)
    tt = tail_times(k_in, t_out, stride)
    y = np.concatenate([_at(v, dt, False, tt) / sv, _at(i, dt, True, tt) / si]).astype(np.float32)
    return x, y


@dataclass
class Decision:
    stop: bool       # stop at the decision step
    residual: float  # relative misfit over the window


TAIL_FLOOR = 0.02  # the prediction must decay below this (of the input's end amplitude)


def verify(pred: np.ndarray, v: np.ndarray, i: np.ndarray, dt: float, k_in: int = K_IN, t_out: int = T_OUT,
           stride: int = STRIDE, window: int = WINDOW, threshold: float = 0.1,
           floor: float = TAIL_FLOOR) -> Decision:
    """Whether a run may stop on its prediction: the predicted points inside
    the window after the input agree with the live samples (relative L2
    misfit of V and I together at most `threshold`; records of at least
    decision_step(dt) steps), and the predicted ring-down has died out
    within the horizon (RMS of its last 32 points below `floor`), so the
    reported record holds the whole decay."""
    _, (sv, si) = example_input(v, i, dt, k_in)
    n = window // stride
    tt = tail_times(k_in, t_out, stride)[:n]
    live = np.concatenate([_at(v, dt, False, tt) / sv, _at(i, dt, True, tt) / si])
    want = np.concatenate([pred[:n], pred[t_out:t_out + n]])
    r = float(np.linalg.norm(live - want) / max(np.linalg.norm(live), 1e-12))
    end = max(float(np.sqrt(np.mean(pred[t_out - 32:t_out] ** 2))), float(np.sqrt(np.mean(pred[-32:] ** 2))))
    return Decision(r <= threshold and end <= floor, r)


def spliced(v: np.ndarray, i: np.ndarray, pred: np.ndarray, stop: int, dt: float, k_in: int = K_IN,
            t_out: int = T_OUT, stride: int = STRIDE):
    """The record a stopped run reports, at every step: the live samples up
    to step `stop`, then the predicted tail (denormalised) beyond it, joined
    and filled in by a cubic spline through the last live samples and the
    predicted points. Returns (step indices, V, I)."""
    from scipy.interpolate import CubicSpline

    _, (sv, si) = example_input(v, i, dt, k_in)
    tt = tail_times(k_in, t_out, stride)
    lead = np.arange(max(0, stop - 64), stop)
    last = int(tt[-1] / dt - 1.0)
    fill = np.arange(stop, last + 1)
    out = []
    for x, half, p, sc in ((v, False, pred[:t_out], sv), (i, True, pred[t_out:], si)):
        off = 0.5 if half else 1.0
        tk = tt[tt > (stop - 1 + off) * dt]
        pk = p[tt > (stop - 1 + off) * dt] * sc
        knots = np.concatenate([(lead + off) * dt, tk])
        vals = np.concatenate([x[lead], pk])
        out.append(np.concatenate([x[:stop], CubicSpline(knots, vals)((fill + off) * dt)]))
    return np.arange(last + 1), out[0], out[1]


def s11_db(steps: np.ndarray, v: np.ndarray, i: np.ndarray, dt: float, freqs: np.ndarray, z_ref: float = 50.0):
    """|S11| in dB of a port record at step indices `steps` (one sample per
    step: the reference's DFT sum, src/post/dft.rs:218; V at (n+1)·dt, I at
    (n+½)·dt, src/engine/port.rs:191-205)."""
    s = np.asarray(steps, dtype=np.float64)
    ph_v = np.exp(-2j * np.pi * np.outer(freqs, (s + 1.0) * dt))
    ph_i = np.exp(-2j * np.pi * np.outer(freqs, (s + 0.5) * dt))
    V = ph_v @ v * dt
    I = ph_i @ i * dt
    a = (V + z_ref * I) / (2.0 * np.sqrt(z_ref))
    b = (V - z_ref * I) / (2.0 * np.sqrt(z_ref))
    return 20.0 * np.log10(np.abs(b / a))


# ---------------------------------------------------------------------------
# Runs: records from the batched solver, training, and the early-stop driver.

def port_records(models, ports, steps, device: int = 0):
    """Port V and I series of every model, stepped as one batch: model q
    runs steps[q] steps (an int: all the same) and is frozen there while the
    others go on. List of (v, i) float64 arrays of length steps[q]."""
    from ems_b200 import Batch

    n = len(models)
    need = [int(steps)] * n if np.isscalar(steps) else [int(x) for x in steps]
    b = Batch(models, device=device, max_steps=max(need))
    done = 0
    for target in sorted(set(need)):
        b.run(target - done)
        done = target
        for q in range(n):
            if need[q] == target:
                b.set_active(q, False)
    out = [(b.samples(q, ports[q], 1), b.samples(q, ports[q], 2)) for q in range(n)]
    b.close()
    return out


def train(net: Net, X, Y, epochs: int, batch: int = 64, lr: float = 1e-3, seed: int = 0, log=None):
    """Adam over shuffled minibatches of device tensors X (N, K_IN, 2) and
    Y (N, 2·T_OUT), the rate falling linearly from lr to lr/20 over the
    epochs; returns the per-epoch mean loss."""
    torch = net.torch
    rng = np.random.default_rng(seed)
    n = X.shape[0]
    hist = []
    for ep in range(epochs):
        rate = lr * (1.0 - 0.95 * ep / max(1, epochs - 1))
        order = rng.permutation(n)
        tot = torch.zeros(1, device=net.dev)
        nb = 0
        for q in range(0, n - batch + 1, batch):
            sel = torch.from_numpy(order[q:q + batch]).to(net.dev)
            tot += net.train_step(X[sel], Y[sel], lr=rate)
            nb += 1
        hist.append(float(tot.item()) / max(nb, 1))
        if log:
            log(ep, hist[-1])
    return hist


class LearnedStop:
    """A batch seen by the run loop (ems_b200.run_until_batch), with the
    learned stop folded in: at a model's decision step its port record goes
    through the network; a model whose window samples agree with the
    prediction (verify) is frozen there, the others run on under the energy
    criterion unchanged. A frozen model reads as zero energy at the loop's
    next check, which ends its loop; `stopped[m]` keeps the step it really
    stopped at."""

    def __init__(self, batch, ports, dts, net: Net, threshold: float = 0.1):
        self.b, self.ports, self.dts, self.net, self.threshold = batch, ports, list(dts), net, threshold
        self.n = batch.n
        self.steps = 0
        self.due = {}
        for q, dt in enumerate(self.dts):
            self.due.setdefault(decision_step(dt), []).append(q)
        self.stopped: dict[int, int] = {}
        self.pred: dict[int, np.ndarray] = {}
        self.residual: dict[int, float] = {}
        self.active = [True] * self.n

    def _decide(self, models):
        torch = self.net.torch
        live = [q for q in models if self.active[q]]
        if not live:
            return
        recs = [(self.b.samples(q, self.ports[q], 1), self.b.samples(q, self.ports[q], 2)) for q in live]
        X = np.stack([example_input(v, i, self.dts[q])[0] for q, (v, i) in zip(live, recs)])
        out = self.net.forward(torch.from_numpy(X).to(self.net.dev)).cpu().numpy()
        for q, (v, i), p in zip(live, recs, out):
            d = verify(p, v, i, self.dts[q], threshold=self.threshold)
            self.residual[q] = d.residual
            if d.stop:
                self.pred[q] = p
                self.stopped[q] = self.steps
                self.b.set_active(q, False)
                self.active[q] = False

    def _advance(self, c: int) -> None:
        self.b.run(c)
        self.steps += c
        if self.steps in self.due:
            self._decide(self.due[self.steps])

    def run(self, k: int) -> None:
        while k:
            nxt = [s for s in self.due if s > self.steps]
            c = min([k] + [s - self.steps for s in nxt])
            self._advance(c)
            k -= c

    def step_with_energy(self):
        w = self.b.step_with_energy()
        self.steps += 1
        if self.steps in self.due:
            self._decide(self.due[self.steps])
        return w

    def set_active(self, m: int, a: bool) -> None:
        self.active[m] = self.active[m] and a
        self.b.set_active(m, a and m not in self.stopped)
