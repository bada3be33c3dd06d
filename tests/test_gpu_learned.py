"""The learned initial guess on the GPU, through the C-ABI (ins2d_cnn_*):
forward pass and loss gradient of the BF16 tensor-core network against the
CPU oracle (oracle/cnn_ref.py, which emulates the same rounding points),
training on the solver's own (f, dp) pairs, and what the trained network
gains over the PCG without it at an unchanged residual tolerance."""
import numpy as np
import pytest

from oracle import cnn_ref as N

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _net(seed=5, scale=0.8, path="tcgen05"):
    from ins2d_b200.learned import ConvNet
    net = ConvNet(device=0, seed=seed)
    net.set_path(path)
    w = N.he_init(seed)
    net.set_params(w, scale)
    return net, w.astype(np.float64), scale


def _inputs(seed, B, H, W):
    torch = _torch()
    rng = np.random.default_rng(seed)
    inp = rng.standard_normal((B, H, W)).astype(np.float32)
    tgt = rng.standard_normal((B, H, W)).astype(np.float32)
    return inp, tgt, torch.from_numpy(inp).cuda(), torch.from_numpy(tgt).cuda()


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def _check_layers(net, w, scale, inp, y):
    """Teacher-forced check of every layer: the oracle's layer l from the
    device's own input of that layer must equal the device's BF16 output,
    except for rare one-ulp rounding flips (FP32 sums on the device, FP64 in
    the oracle) and ReLU decisions at |Z| ~ 0."""
    B, H, W = inp.shape
    acts = [net.activations(l, B * H * W).reshape(B, H, W, 32) for l in range(1, 6)]
    prev = inp
    for l in range(1, 6):
        ref = N.layer(w, l, prev)
        got = acts[l - 1].astype(np.float64)
        diff = np.abs(got - ref)
        bad = diff > 2.0 ** -7 * np.maximum(np.abs(ref), np.abs(got)) + 1e-6 * np.max(np.abs(ref))
        assert not bad.any(), (l, int(bad.sum()), float(diff.max()))
        assert np.mean(got != ref) < 5e-3, (l, float(np.mean(got != ref)))
        prev = got
    y_ref = scale * N.layer(w, 6, prev)
    assert _rel(y, y_ref) < 1e-5, _rel(y, y_ref)
    return acts


@pytest.mark.parametrize("path", ["tcgen05", "mma_sync"])
@pytest.mark.parametrize("shape", [(1, 8, 16), (2, 37, 29), (1, 70, 131)])
def test_forward_matches_oracle(shape, path):
    B, H, W = shape
    net, w, scale = _net(path=path)
    inp, _, ti, _ = _inputs(1, B, H, W)
    y = net.forward(ti).cpu().numpy()
    _check_layers(net, w, scale, inp, y)
    # end to end, the rounding flips cascade: a looser bound
    y_ref, _ = N.forward(w, scale, inp, bf16_mode=True)
    assert _rel(y, y_ref) < 3e-2, _rel(y, y_ref)


@pytest.mark.parametrize("path", ["tcgen05", "mma_sync"])
@pytest.mark.parametrize("shape", [(2, 37, 29), (1, 24, 48)])
def test_loss_gradient_matches_oracle(shape, path):
    B, H, W = shape
    net, w, scale = _net(seed=7, scale=1.3, path=path)
    inp, tgt, ti, tt = _inputs(2, B, H, W)
    loss, g = net.loss_grad(ti, tt)
    acts = [net.activations(l, B * H * W).reshape(B, H, W, 32) for l in range(1, 6)]
    loss_ref, g_ref = N.loss_grad(w, scale, inp, tgt, bf16_mode=True, acts=acts)
    assert abs(loss - loss_ref) / loss_ref < 1e-5
    # every layer's gradient block (the backward pass's BF16 rounding flips
    # of dZ cascade like the forward's)
    bounds = [0, N.OFF_WM] + [N.OFF_WM + (l + 1) * N.SZ_WM for l in range(N.NMID)] + [N.NPARAM]
    for a, b in zip(bounds[:-1], bounds[1:]):
        assert _rel(g[a:b], g_ref[a:b]) < 1e-2, (a, b, _rel(g[a:b], g_ref[a:b]))
    # the layer-6 gradient sees no rounding after the device's activations
    assert _rel(g[N.OFF_W6:], g_ref[N.OFF_W6:]) < 1e-5


@pytest.mark.parametrize("path", ["tcgen05", "mma_sync"])
def test_residual_loss_gradient_matches_oracle(path):
    """The residual loss on a context's grid (FP32 stencil of the context's
    own operator tables) against the oracle with the oracle's sparse A."""
    import ins2d_b200
    from ins2d_b200 import cases
    from oracle import ins2d_ref as R
    x = cases.tanh_grid(29, 0.0, 1.0, 1.05)
    y = cases.tanh_grid(21, 0.0, 1.0, 1.05)
    m = ins2d_b200.Options(x, y, cases.BC_CAVITY, Re=100.0, poisson=4, device=0)
    A = R.make_options(x, y, cases.BC_CAVITY, Re=100.0, poisson=4).discretization.A
    net, w, scale = _net(seed=13, scale=0.7, path=path)
    inp, _, ti, _ = _inputs(3, 2, m.Npy, m.Npx)
    loss, g = net.loss_grad_residual(m, ti)
    acts = [net.activations(l, ti.numel()).reshape(2, m.Npy, m.Npx, 32) for l in range(1, 6)]
    loss_ref, g_ref = N.loss_grad(w, scale, inp, None, bf16_mode=True, acts=acts, A=A)
    assert abs(loss - loss_ref) / loss_ref < 1e-4, (loss, loss_ref)
    bounds = [0, N.OFF_WM] + [N.OFF_WM + (l + 1) * N.SZ_WM for l in range(N.NMID)] + [N.NPARAM]
    for a, b in zip(bounds[:-1], bounds[1:]):
        assert _rel(g[a:b], g_ref[a:b]) < 1e-2, (a, b, _rel(g[a:b], g_ref[a:b]))
    assert _rel(g[N.OFF_W6:], g_ref[N.OFF_W6:]) < 1e-4


@pytest.mark.parametrize("path", ["tcgen05", "mma_sync"])
@pytest.mark.parametrize("shape", [(1, 1, 1), (3, 2, 5), (1, 9, 1), (2, 1, 33)])
def test_degenerate_field_shapes(shape, path):
    """Fields thinner than a tile and than the 3x3 stencil: every tap falls on
    the zero padding somewhere."""
    net, w, scale = _net(seed=4, scale=1.1, path=path)
    inp, _, ti, _ = _inputs(5, *shape)
    y = net.forward(ti).cpu().numpy()
    _check_layers(net, w, scale, inp, y)


def test_params_round_trip_and_reuse_after_larger_batch():
    torch = _torch()
    net, w, _ = _net(seed=6, scale=0.5)
    w2, sc = net.params()
    assert np.array_equal(w2, w.astype(np.float32)) and sc == 0.5
    big = torch.randn(3, 64, 80, dtype=torch.float32, device="cuda")
    small = big[1:2, :17, :23].contiguous()
    y_small = net.forward(small)
    net.forward(big)  # grows the buffers
    assert torch.equal(net.forward(small), y_small)


def test_tensor_core_paths_agree_on_large_field():
    """Both instruction paths on a field larger than the persistent grid
    (several tiles per block) give the same network output."""
    torch = _torch()
    a, _, _ = _net(seed=9, path="tcgen05")
    b, _, _ = _net(seed=9, path="mma_sync")
    x = torch.randn(2, 301, 517, dtype=torch.float32, device="cuda")
    ya, yb = a.forward(x), b.forward(x)
    assert float(torch.linalg.norm(ya - yb) / torch.linalg.norm(yb)) < 1e-5


def test_invalid_arguments_rejected():
    from ins2d_b200.api import Ins2dError
    torch = _torch()
    net, _, _ = _net()
    host = torch.zeros((1, 8, 8), dtype=torch.float32)  # host memory
    with pytest.raises((Ins2dError, ValueError)):
        net.forward(host)
    dev = torch.zeros((1, 8, 8), dtype=torch.float32, device="cuda")
    with pytest.raises(Ins2dError):
        net.train_step(dev, dev, -1.0)
    with pytest.raises(Ins2dError):
        net.set_params(None, 0.0)


def _cavity(N_=48, precond="jacobi", tol=1e-10):
    import ins2d_b200
    from ins2d_b200 import cases
    x = cases.tanh_grid(N_, 0.0, 1.0, 1.05)
    return ins2d_b200.Options(x, x.copy(), cases.BC_CAVITY, Re=1000.0, poisson=4, CG_acc=tol, CG_maxit=100000,
                              uBC=cases.lid_uBC(1.0, 1.0), precond=precond, device=0)


def _record(m, steps, capacity):
    from ins2d_b200 import learned
    f_buf, p_buf = learned.record_pairs(m, capacity)
    V = np.zeros(m.NV)
    p = m.pressure_additional_solve(V, np.zeros(m.Np), 0.0)
    V, p = m.time_ERK(V, p, 0.0, 2e-3, nsteps=steps)
    n = learned.recorded_pairs(m)
    learned.stop_recording(m)
    return f_buf, p_buf, n


def test_training_gains_over_plain_pcg():
    """Pairs from the solver's own first steps (a stretched lid-driven cavity);
    the network trained on the first 80% and evaluated on the held-out rest: the
    same tolerance is reached in fewer iterations than the Jacobi-PCG without
    it from the learned guess, and in far fewer by the flexible CG with the
    network (trained with white-noise fields as well) as its preconditioner;
    the solutions agree within the tolerance."""
    from ins2d_b200 import learned
    torch = _torch()
    m = _cavity()
    f_buf, p_buf, n = _record(m, 24, 160)
    assert n >= 96  # p_initial + 4 stage solves per RK44 step
    ntr = int(0.8 * n)
    inp, tgt = learned.prepare_pairs(m, f_buf[:ntr], p_buf[:ntr])
    net = learned.ConvNet(device=0, seed=11)
    losses = learned.train(net, inp, None, steps=400, batch=8, lr=3e-3, seed=1, options=m)
    assert np.mean(losses[-20:]) < 0.5 * np.mean(losses[:5]), (losses[:5], losses[-20:])
    # the same network trained with white-noise fields in every batch, for
    # the preconditioner role
    net_p = learned.ConvNet(device=0, seed=11)
    learned.train(net_p, inp, None, steps=400, batch=8, lr=3e-3, seed=1, options=m, noise=8)
    it_plain, it_learned, it_fcg, it_fcg_n, res = [], [], [], [], []
    for k in range(ntr, n):
        f = f_buf[k].contiguous()
        fh = f.cpu().numpy()
        learned.attach(m, None)
        dp0, s0 = m.pressure_poisson(f, return_stats=True)
        it_plain.append(s0["iters"])
        for nn, mode, its in ((net, "guess", it_learned), (net, "precond", it_fcg), (net_p, "precond", it_fcg_n)):
            learned.attach(m, nn, mode)
            dp1, s1 = m.pressure_poisson(f, return_stats=True)
            its.append(s1["iters"])
            assert s1["norm1"] <= 1e-10 * (1 + 1e-9)
            r = fh - m.laplacian(dp1.cpu().numpy())
            res.append(np.linalg.norm(r) / np.linalg.norm(fh))
    learned.attach(m, None)
    print(f"\nheld-out solves: plain Jacobi-PCG {np.mean(it_plain):.1f} iterations, "
          f"from the learned guess {np.mean(it_learned):.1f}, flexible CG with the network as the "
          f"preconditioner {np.mean(it_fcg):.1f} (trained with noise fields: {np.mean(it_fcg_n):.1f}); "
          f"max relative residual {max(res):.2e}")
    assert max(res) < 2e-10
    # the learned guess saves iterations on the held-out solves; the flexible
    # CG reaches the same tolerance with the network as its preconditioner
    assert np.mean(it_learned) < np.mean(it_plain)
    assert max(it_fcg) < 2000
    # trained with noise fields, the network is a better preconditioner than
    # the Jacobi diagonal (measured on a B200: 153.6 against 224.3 iterations)
    assert np.mean(it_fcg_n) < 0.85 * np.mean(it_plain)


def test_library_training_recipe():
    """ins2d_learned_train (the one-call recipe a MATLAB gateway uses):
    records the solver's pairs, trains with noise fields, and the network
    then preconditions the flexible CG better than the Jacobi diagonal on
    right-hand sides from later steps."""
    from ins2d_b200 import learned
    m = _cavity()
    V = np.zeros(m.NV)
    p = m.pressure_additional_solve(V, np.zeros(m.Np), 0.0)
    net = learned.ConvNet(device=0, seed=11)
    l0, l1 = learned.train_from_steps(m, net, V, p, 0.0, 2e-3, record_steps=20, max_pairs=120, steps=400,
                                      batch=8, lr=3e-3, noise=8, seed=1)
    assert l1 < 0.5 * l0, (l0, l1)
    V1, p1 = m.time_ERK(V, p, 0.0, 2e-3, nsteps=20)
    f_buf, p_buf = learned.record_pairs(m, 12)
    m.time_ERK(V1, p1, 0.04, 2e-3, nsteps=3)
    n = learned.recorded_pairs(m)
    learned.stop_recording(m)
    it_plain, it_fcg = [], []
    for k in range(n):
        f = f_buf[k].contiguous()
        learned.attach(m, None)
        it_plain.append(m.pressure_poisson(f, return_stats=True)[1]["iters"])
        learned.attach(m, net, "precond")
        dp, st = m.pressure_poisson(f, return_stats=True)
        it_fcg.append(st["iters"])
        assert st["norm1"] <= 1e-10 * (1 + 1e-9)
    learned.attach(m, None)
    print(f"\nlibrary recipe: Jacobi-PCG {np.mean(it_plain):.1f}, network-preconditioned FCG {np.mean(it_fcg):.1f}")
    assert np.mean(it_fcg) < 0.85 * np.mean(it_plain)


def test_learned_guess_with_multigrid_and_time_steps():
    """With the multigrid preconditioner and inside time steps the learned
    guess leaves the flow unchanged within the solver tolerance."""
    from ins2d_b200 import learned
    m = _cavity(precond="mg", tol=1e-12)
    f_buf, p_buf, n = _record(m, 6, 40)
    inp, tgt = learned.prepare_pairs(m, f_buf[:n], p_buf[:n])
    net = learned.ConvNet(device=0, seed=3)
    learned.train(net, inp, None, steps=60, batch=4, lr=3e-3, options=m)
    V = np.zeros(m.NV)
    p = m.pressure_additional_solve(V, np.zeros(m.Np), 0.0)
    V0, p0 = m.time_ERK(V, p, 0.0, 2e-3, nsteps=5)
    learned.attach(m, net)
    V1, p1 = m.time_ERK(V, p, 0.0, 2e-3, nsteps=5)
    learned.attach(m, None)
    assert _rel(V1, V0) < 1e-9
