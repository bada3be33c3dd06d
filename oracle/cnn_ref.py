"""CPU oracle of the learned initial guess's network (test infrastructure only:
tests and the smoke check import it to check the GPU kernels; nothing on the
product path uses it).

The network has no counterpart in the reference (its pressure solves start
from zero, pressure_poisson.m:61-70; cg.F:207-229 with x_in = 0).  This module
restates the library's definition in numpy:

  six 3x3 convolutions, zero padding, no biases, channels 1 -> 32 -> 32 -> 32
  -> 32 -> 32 -> 1, ReLU after layers 1..5, output scaled by out_scale;
  parameters (flat float32): W1 [32][9], W2..W5 [32][9][32] ([out][tap][in]),
  W6 [9][32]; tap t = (dy+1)*3 + (dx+1) reads the pixel at (x+dx, y+dy).
  Loss = mean((out - tgt)^2) over all pixels of the batch.

``bf16=True`` emulates the device's rounding points (layer outputs 1..5 and
the gradients dZ1..dZ5 rounded to BF16, round-to-nearest-even; the 32 -> 32
weights rounded to BF16 for the tensor cores); sums are float64 here (float32
on the device).  ``bf16=False`` is exact float64 arithmetic, the form the
finite-difference check pins.
"""
import numpy as np

C = 32
TAPS = 9
K = TAPS * C
NMID = 4
OFF_WM = C * TAPS
SZ_WM = C * K
OFF_W6 = OFF_WM + NMID * SZ_WM
NPARAM = OFF_W6 + K


def bf16(a):
    """Round float32 values to BF16 (nearest, ties to even) and return them as float64."""
    u = np.ascontiguousarray(np.asarray(a, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    v = ((u + r) & 0xFFFF0000).astype(np.uint32)
    return v.view(np.float32).astype(np.float64)


def split(w):
    w = np.asarray(w, dtype=np.float64)
    W1 = w[:OFF_WM].reshape(C, TAPS)
    Wm = [w[OFF_WM + l * SZ_WM: OFF_WM + (l + 1) * SZ_WM].reshape(C, TAPS, C) for l in range(NMID)]
    W6 = w[OFF_W6:].reshape(TAPS, C)
    return W1, Wm, W6


def join(W1, Wm, W6):
    return np.concatenate([W1.ravel()] + [m.ravel() for m in Wm] + [W6.ravel()])


def _shift(a, dy, dx):
    """a[b, y+dy, x+dx, ...] with zeros outside (a: (B, H, W, ...))."""
    B, H, W = a.shape[:3]
    out = np.zeros_like(a)
    ys, ye = max(0, -dy), min(H, H - dy)
    xs, xe = max(0, -dx), min(W, W - dx)
    if ys < ye and xs < xe:
        out[:, ys:ye, xs:xe] = a[:, ys + dy:ye + dy, xs + dx:xe + dx]
    return out


def _taps():
    return [(t // 3 - 1, t % 3 - 1) for t in range(TAPS)]


def forward(w, out_scale, inp, bf16_mode=True):
    """Returns (y, activations [A0, A1..A5]); inp: (B, H, W)."""
    rnd = bf16 if bf16_mode else (lambda a: np.asarray(a, dtype=np.float64))
    W1, Wm, W6 = split(w)
    A0 = np.asarray(inp, dtype=np.float64)
    Z = np.zeros(A0.shape + (C,))
    for t, (dy, dx) in enumerate(_taps()):
        Z += _shift(A0, dy, dx)[..., None] * W1[:, t][None, None, None, :]
    acts = [A0, rnd(np.maximum(Z, 0.0))]
    for l in range(NMID):
        Wl = rnd(Wm[l]) if bf16_mode else Wm[l]
        Z = np.zeros_like(acts[-1])
        for t, (dy, dx) in enumerate(_taps()):
            Z += _shift(acts[-1], dy, dx) @ Wl[:, t, :].T
        acts.append(rnd(np.maximum(Z, 0.0)))
    y6 = np.zeros(A0.shape)
    for t, (dy, dx) in enumerate(_taps()):
        y6 += _shift(acts[-1], dy, dx) @ W6[t]
    return out_scale * y6, acts


def layer(w, l, a_prev, bf16_mode=True):
    """Output of layer l (1..6) from the given input activations (teacher
    forcing: the device's own inputs of that layer); layers 1..5 after ReLU
    and rounding, layer 6 before out_scale."""
    rnd = bf16 if bf16_mode else (lambda a: np.asarray(a, dtype=np.float64))
    W1, Wm, W6 = split(w)
    a_prev = np.asarray(a_prev, dtype=np.float64)
    if l == 1:
        Z = np.zeros(a_prev.shape + (C,))
        for t, (dy, dx) in enumerate(_taps()):
            Z += _shift(a_prev, dy, dx)[..., None] * W1[:, t][None, None, None, :]
        return rnd(np.maximum(Z, 0.0))
    if l == 6:
        y6 = np.zeros(a_prev.shape[:3])
        for t, (dy, dx) in enumerate(_taps()):
            y6 += _shift(a_prev, dy, dx) @ W6[t]
        return y6
    Wl = rnd(Wm[l - 2]) if bf16_mode else Wm[l - 2]
    Z = np.zeros_like(a_prev)
    for t, (dy, dx) in enumerate(_taps()):
        Z += _shift(a_prev, dy, dx) @ Wl[:, t, :].T
    return rnd(np.maximum(Z, 0.0))


def loss_grad(w, out_scale, inp, tgt, bf16_mode=True, acts=None, A=None):
    """(loss, flat gradient) of mean((y - tgt)^2).  ``acts`` = [A1..A5] uses
    given forward activations (the device's) instead of recomputing them.
    With a sparse pressure operator ``A`` (Np x Np, x fastest) the loss is the
    residual loss mean((A y - diag(A) inp)^2) per field instead (tgt unused)."""
    rnd = bf16 if bf16_mode else (lambda a: np.asarray(a, dtype=np.float64))
    W1, Wm, W6 = split(w)
    if acts is None:
        y, acts = forward(w, out_scale, inp, bf16_mode)
    else:
        acts = [np.asarray(inp, dtype=np.float64)] + [np.asarray(a, dtype=np.float64) for a in acts]
        y = out_scale * layer(w, 6, acts[5], bf16_mode)
    n = y.size
    if A is None:
        d = y - np.asarray(tgt, dtype=np.float64)
        loss = float(np.sum(d * d) / n)
        dy6 = 2.0 * d / n * out_scale
    else:
        dg = A.diagonal()
        x0 = np.asarray(inp, dtype=np.float64)
        loss, dy6 = 0.0, np.zeros_like(y)
        for b in range(y.shape[0]):
            r = A @ y[b].ravel() - dg * x0[b].ravel()
            loss += float(r @ r)
            dy6[b] = (2.0 / n * out_scale) * (A @ r).reshape(y.shape[1:])
        loss /= n
    taps = _taps()
    A5 = acts[5]
    gW6 = np.zeros_like(W6)
    G = np.zeros(A5.shape)
    for t, (dy, dx) in enumerate(taps):
        gW6[t] = np.einsum("bhw,bhwc->c", dy6, _shift(A5, dy, dx))
        G += _shift(dy6, -dy, -dx)[..., None] * W6[t][None, None, None, :]
    dZ = rnd(G * (A5 > 0))
    gWm = [None] * NMID
    for l in range(NMID - 1, -1, -1):
        Ain = acts[l + 1]
        Wl = rnd(Wm[l]) if bf16_mode else Wm[l]
        g = np.zeros((C, TAPS, C))
        G = np.zeros(Ain.shape)
        for t, (dy, dx) in enumerate(taps):
            g[:, t, :] = np.einsum("bhwo,bhwi->oi", dZ, _shift(Ain, dy, dx))
            G += _shift(dZ, -dy, -dx) @ Wl[:, t, :]
        gWm[l] = g
        dZ = rnd(G * (Ain > 0))
    gW1 = np.zeros_like(W1)
    for t, (dy, dx) in enumerate(taps):
        gW1[:, t] = np.einsum("bhwc,bhw->c", dZ, _shift(acts[0], dy, dx))
    return loss, join(gW1, gWm, gW6)


def he_init(seed):
    """He-normal weights (numpy generator; the library seeds its own)."""
    rng = np.random.default_rng(seed)
    w = np.empty(NPARAM)
    w[:OFF_WM] = rng.standard_normal(OFF_WM) * np.sqrt(2.0 / TAPS)
    w[OFF_WM:OFF_W6] = rng.standard_normal(OFF_W6 - OFF_WM) * np.sqrt(2.0 / K)
    w[OFF_W6:] = rng.standard_normal(K) * np.sqrt(1.0 / K)
    return w.astype(np.float32)
