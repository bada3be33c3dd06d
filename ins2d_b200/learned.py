"""The learned initial guess of the pressure solve (include/ins2d.h,
``ins2d_cnn_*``): a six-layer 3x3 convolutional network, trained on the GPU by
the library's own BF16 tensor-core forward and backward kernels on
(right-hand side, pressure) pairs recorded from the solver's own PCG solves.

There is no counterpart in the reference, whose solves start from zero
(pressure_poisson.m:61-70).  Attached to a context, the network's output
(scaled by the Rayleigh-Ritz factor) is where PCG starts; CG still iterates
to ||r|| <= CG_acc ||f||, so solutions change only within that tolerance.

Device buffers here are torch CUDA tensors (plumbing); every computation runs
in libins2d.so.
"""
import ctypes

import numpy as np

from . import _lib
from .api import Ins2dError

NPARAM = _lib.CNN_NPARAM


def _require_cuda(t, dtype, name):
    import torch
    if not (hasattr(t, "is_cuda") and t.is_cuda and t.dtype == dtype and t.is_contiguous()):
        raise ValueError(f"{name}: need a contiguous CUDA tensor of {dtype}")
    return t


class ConvNet:
    """The network (device-resident FP32 master weights, BF16 copies for the
    tensor-core layers, Adam moments).  ``seed`` fixes the He-normal initial
    weights."""

    def __init__(self, device=0, seed=0):
        self._lib = _lib.load()
        self._h = ctypes.c_void_p()
        self.device = int(device)
        rc = self._lib.ins2d_cnn_create(self.device, ctypes.c_uint64(int(seed)), ctypes.byref(self._h))
        if rc != 0:
            raise Ins2dError(rc, "cnn_create failed")

    def _check(self, rc):
        if rc != 0:
            m = self._lib.ins2d_cnn_last_error(self._h)
            raise Ins2dError(rc, m.decode() if m else "")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ins2d_cnn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream):
        self._check(self._lib.ins2d_cnn_set_stream(self._h, ctypes.c_void_p(stream)))

    def set_path(self, path):
        """Tensor-core instructions of the 32 -> 32 layers: 'tcgen05' (default)
        or 'mma_sync'."""
        code = {"tcgen05": _lib.CNN_PATH_TCGEN05, "mma_sync": _lib.CNN_PATH_MMA_SYNC}[path]
        self._check(self._lib.ins2d_cnn_set_path(self._h, code))

    def params(self):
        """(FP32 weights as a numpy array of NPARAM, out_scale)."""
        w = np.empty(NPARAM, dtype=np.float32)
        sc = ctypes.c_float()
        self._check(self._lib.ins2d_cnn_get_params(self._h, w.ctypes.data, ctypes.byref(sc)))
        return w, float(sc.value)

    def set_params(self, w=None, out_scale=1.0):
        ptr = None
        if w is not None:
            w = np.ascontiguousarray(np.asarray(w, dtype=np.float32).ravel())
            if w.size != NPARAM:
                raise ValueError(f"need {NPARAM} weights")
            ptr = w.ctypes.data
        self._check(self._lib.ins2d_cnn_set_params(self._h, ptr, float(out_scale)))

    def forward(self, inp):
        """out_scale * net(inp) for a float32 CUDA tensor of shape (B, H, W)."""
        import torch
        _require_cuda(inp, torch.float32, "inp")
        B, H, W = inp.shape
        y = torch.empty_like(inp)
        torch.cuda.synchronize(inp.device)
        self._check(self._lib.ins2d_cnn_forward(self._h, inp.data_ptr(), y.data_ptr(), B, H, W))
        return y

    def activations(self, layer, pixels):
        """BF16 output of layer 1..5 of the last forward pass, as float32
        numpy values of shape (pixels, 32)."""
        raw = np.empty((int(pixels), 32), dtype=np.uint16)
        self._check(self._lib.ins2d_cnn_get_activations(self._h, int(layer), int(pixels), raw.ctypes.data))
        return (raw.astype(np.uint32) << 16).view(np.float32)

    def loss_grad(self, inp, tgt):
        """(mean squared error, gradient as a numpy float32 array); no update."""
        import torch
        _require_cuda(inp, torch.float32, "inp")
        _require_cuda(tgt, torch.float32, "tgt")
        B, H, W = inp.shape
        g = np.empty(NPARAM, dtype=np.float32)
        loss = ctypes.c_double()
        torch.cuda.synchronize(inp.device)
        self._check(self._lib.ins2d_cnn_loss_grad(self._h, inp.data_ptr(), tgt.data_ptr(), B, H, W,
                                                  ctypes.byref(loss), g.ctypes.data))
        return loss.value, g

    def loss_grad_residual(self, options, inp):
        """Residual loss mean((A net(inp) - diag(A) inp)^2) on ``options``'
        grid and its gradient (numpy float32); no update."""
        import torch
        _require_cuda(inp, torch.float32, "inp")
        g = np.empty(NPARAM, dtype=np.float32)
        loss = ctypes.c_double()
        torch.cuda.synchronize(inp.device)
        options._check(self._lib.ins2d_cnn_loss_grad_residual(options._ctx, self._h, inp.data_ptr(), inp.shape[0],
                                                              ctypes.byref(loss), g.ctypes.data))
        return loss.value, g

    def train_step_residual(self, options, inp, lr):
        """One Adam step on the residual loss; returns the loss before it."""
        import torch
        _require_cuda(inp, torch.float32, "inp")
        loss = ctypes.c_double()
        options._check(self._lib.ins2d_cnn_train_step_residual(options._ctx, self._h, inp.data_ptr(), inp.shape[0],
                                                               float(lr), ctypes.byref(loss)))
        return loss.value

    def train_step(self, inp, tgt, lr):
        """One Adam step on the mean squared error; returns the loss before it."""
        import torch
        _require_cuda(inp, torch.float32, "inp")
        _require_cuda(tgt, torch.float32, "tgt")
        B, H, W = inp.shape
        loss = ctypes.c_double()
        self._check(self._lib.ins2d_cnn_train_step(self._h, inp.data_ptr(), tgt.data_ptr(), B, H, W, float(lr),
                                                   ctypes.byref(loss)))
        return loss.value


def record_pairs(options, capacity):
    """Starts recording the (f, dp) pairs of ``options``' next PCG solves into
    new device buffers; returns them as (f_buf, p_buf), shape (capacity, Np)."""
    import torch
    dev = torch.device("cuda", options._desc[2].device)
    f_buf = torch.zeros((capacity, options.Np), dtype=torch.float64, device=dev)
    p_buf = torch.zeros((capacity, options.Np), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    options._check(options._lib.ins2d_record_pairs(options._ctx, f_buf.data_ptr(), p_buf.data_ptr(), int(capacity)))
    options._rec = (f_buf, p_buf)
    return f_buf, p_buf


def recorded_pairs(options):
    """Number of pairs recorded so far; stops recording when called with stop."""
    return int(options._lib.ins2d_recorded_pairs(options._ctx))


def stop_recording(options):
    options._check(options._lib.ins2d_record_pairs(options._ctx, None, None, 0))


def singular(options):
    """True when A has the constant null space (no pressure boundary): the
    targets are then centred (their mean is arbitrary)."""
    return not any(options.BC[c][s] == "pres" for c in ("u", "v") for s in ("left", "right", "low", "up"))


def prepare_pairs(options, f, p, n=None):
    """Network inputs and targets (float32, shape (n, Npy, Npx)) from n
    recorded pairs: in = (f / diag A) / s, tgt = (p - mean) / s, s = rms(f / diag A)."""
    import torch
    n = f.shape[0] if n is None else int(n)
    inp = torch.empty((n, options.Npy, options.Npx), dtype=torch.float32, device=f.device)
    tgt = torch.empty_like(inp)
    torch.cuda.synchronize(f.device)
    options._check(options._lib.ins2d_cnn_prepare_pairs(options._ctx, f.data_ptr(), p.data_ptr(), n,
                                                        int(singular(options)), inp.data_ptr(), tgt.data_ptr()))
    return inp, tgt


def train(net, inp, tgt=None, steps=300, batch=4, lr=2e-3, seed=0, lr_final=None, options=None, noise=0):
    """Adam on random mini-batches of the pairs (cosine-decayed learning
    rate).  With ``options`` the loss is the residual loss on its grid
    (``tgt`` unused; out_scale first matched to the inputs' rms; every batch
    holds each input and its negation, since the solver applies the network's
    odd part; ``noise`` white-noise fields are added to every batch -- the
    residual loss needs no targets, and the residuals a preconditioner sees
    inside CG are rougher than the right-hand sides), else the
    squared error against ``tgt`` (out_scale first set to the targets' rms).
    Returns the losses relative to the first one."""
    import torch
    n = inp.shape[0]
    w, _ = net.params()
    gen = torch.Generator(device="cpu").manual_seed(int(seed))
    if options is None:
        scale = float(torch.sqrt(torch.mean(tgt.double() ** 2)).item()) or 1.0
    else:
        net.set_params(w, 1.0)
        x0 = inp[: min(batch, n)].contiguous()
        y0 = net.forward(x0)
        scale = float(torch.sqrt(torch.mean(x0.double() ** 2) / torch.mean(y0.double() ** 2).clamp_min(1e-30)))
    net.set_params(w, scale)
    lr_final = lr * 0.05 if lr_final is None else lr_final
    losses = []
    for k in range(int(steps)):
        idx = torch.randint(0, n, (min(batch, n),), generator=gen).to(inp.device)
        xb = inp.index_select(0, idx)
        if options is not None:
            if noise:
                z = torch.randn((int(noise),) + tuple(inp.shape[1:]), generator=gen).to(inp.device)
                xb = torch.cat([xb, z])
            xb = torch.cat([xb, -xb])  # the solver uses the odd part (N(v) - N(-v)) / 2
        xb = xb.contiguous()
        rate = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * k / max(steps - 1, 1)))
        if options is None:
            yb = tgt.index_select(0, idx).contiguous()
            losses.append(net.train_step(xb, yb, rate))
        else:
            losses.append(net.train_step_residual(options, xb, rate))
    return [l / losses[0] for l in losses] if losses and losses[0] > 0 else losses


def train_from_steps(options, net, V, p, t, dt, record_steps=24, max_pairs=200, steps=300, batch=4, lr=2e-3,
                     noise=0, seed=0):
    """The library's own training recipe (``ins2d_learned_train``): record the
    pairs of ``record_steps`` time steps from (V, p) (host arrays, not
    modified), then train on the residual loss.  Returns (first, last) loss."""
    V = np.ascontiguousarray(np.asarray(V, dtype=np.float64))
    p = np.ascontiguousarray(np.asarray(p, dtype=np.float64))
    l0, l1 = ctypes.c_double(), ctypes.c_double()
    options._check(options._lib.ins2d_learned_train(
        options._ctx, net.handle, V.ctypes.data, p.ctypes.data, float(t), float(dt), int(record_steps),
        int(max_pairs), int(steps), int(batch), float(lr), int(noise), ctypes.c_uint64(int(seed)), _lib.MEM_HOST,
        ctypes.byref(l0), ctypes.byref(l1)))
    return l0.value, l1.value


def attach(options, net, mode="guess"):
    """Use ``net`` in ``options``' PCG solves (None detaches): mode 'guess'
    starts the context's PCG from the network's guess; 'precond' runs a
    flexible CG with the network as the preconditioner (plain PCG finishes
    if it stalls)."""
    options._check(options._lib.ins2d_set_learned_guess(options._ctx, net.handle if net is not None else None))
    options._check(options._lib.ins2d_set_learned_mode(options._ctx, {"guess": 0, "precond": 1}[mode]))
    options._net = net


def _main():
    """Times the network's forward pass on one random N x N field with CUDA
    events (``python -m ins2d_b200.learned --forward 1024 --path tcgen05``)."""
    import argparse
    import json
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--forward", type=int, default=1024, help="field size N (N x N pixels)")
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--path", default="tcgen05", choices=["tcgen05", "mma_sync"])
    a = ap.parse_args()
    net = ConvNet(device=0, seed=0)
    net.set_path(a.path)
    x = torch.randn(a.batch, a.forward, a.forward, dtype=torch.float32, device="cuda")
    net.forward(x)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(a.reps):
        net.forward(x)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.reps
    flops = 2 * 9 * (1 * 32 + 4 * 32 * 32 + 32 * 1) * a.batch * a.forward ** 2
    print(json.dumps({"path": a.path, "pixels": a.batch * a.forward ** 2, "ms_per_forward": ms,
                      "tflops": flops / ms / 1e9}))


if __name__ == "__main__":
    _main()
