"""The learned warm start's BF16 tensor-core kernels against the numpy oracle
(oracle/cnn_oracle.py, itself pinned by finite differences), and the warm-started
time loop on a small shear-band case."""
import os
import sys

import numpy as np
import pytest

from conftest import fem

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import cnn_oracle as co  # noqa: E402  (the oracle is test infrastructure)

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
ws = fem.warmstart


def dev_bf16(x):
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.float32)).to("cuda").to(torch.bfloat16).contiguous()


def host(t):
    return t.float().cpu().numpy()


def rand_layer(rng, ci, co_):
    w = np.zeros((co_, co.kpad(ci)), dtype=np.float32)
    w[:, :9 * ci] = co.bf16(rng.standard_normal((co_, 9 * ci)).astype(np.float32) * 0.2)
    return w, rng.standard_normal(co_).astype(np.float32) * 0.1


def call_conv(x, w, b, mask, B, H, W, ci, co_, mode):
    lib, h = fem.solver._Handle.get()
    out = torch.empty(B * H * W * co_, dtype=torch.float32 if mode == 1 else torch.bfloat16, device="cuda")
    wb = dev_bf16(w)
    bb = torch.as_tensor(b, device="cuda") if b is not None else None
    rc = lib.femb200_conv3x3_forward(h, ws._p(x), ws._p(wb), ws._p(bb), ws._p(mask), ws._p(out), B, H, W, ci, co_, mode)
    assert rc == 0, lib.femb200_last_error(h)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("ci,co_", [(16, 16), (16, 32), (32, 16), (32, 32)])
@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("W", [19, 150])
def test_conv_forward_matches_oracle(ci, co_, mode, W):
    rng = np.random.default_rng(ci * 100 + co_ + mode + W)
    B, H = 2, 11     # one ragged 128-pixel row segment (W = 19), or a full one and a ragged one
    x = co.bf16(rng.standard_normal((B, H, W, ci)).astype(np.float32))
    w, b = rand_layer(rng, ci, co_)
    mask = co.bf16(rng.standard_normal((B, H, W, co_)).astype(np.float32)) if mode == 2 else None
    y = call_conv(dev_bf16(x), w, b if mode != 2 else None, dev_bf16(mask) if mode == 2 else None, B, H, W, ci, co_, mode)
    ref = co.conv3x3(x, w, None if mode == 2 else b)
    if mode == 0:
        ref = np.maximum(ref, 0)
    if mode == 2:
        ref = ref * (mask > 0)
    got = host(y).reshape(B, H, W, co_)
    tol = 1e-5 if mode == 1 else 8e-3     # BF16 outputs carry 8 mantissa bits
    assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref)), np.max(np.abs(got - ref))


@pytest.mark.parametrize("ci,co_", [(16, 16), (16, 32), (32, 16), (32, 32)])
@pytest.mark.parametrize("W", [21, 133])
def test_weight_gradient_matches_oracle(ci, co_, W):
    rng = np.random.default_rng(7 + ci + co_ + W)
    B, H = 3, 13
    x = co.bf16(rng.standard_normal((B, H, W, ci)).astype(np.float32))
    dy = co.bf16(rng.standard_normal((B, H, W, co_)).astype(np.float32))
    lib, h = fem.solver._Handle.get()
    dw = torch.zeros(co_ * co.kpad(ci), dtype=torch.float32, device="cuda")
    db = torch.zeros(co_, dtype=torch.float32, device="cuda")
    xd, dyd = dev_bf16(x), dev_bf16(dy)     # kept alive until the kernel has run
    rc = lib.femb200_conv3x3_weight_grad(h, ws._p(xd), ws._p(dyd), ws._p(dw), ws._p(db), B, H, W, ci, co_)
    assert rc == 0
    torch.cuda.synchronize()
    w0 = np.zeros((co_, co.kpad(ci)))
    _, rdw, rdb = co.conv3x3_backward(x, w0, dy)
    gdw = host(dw).reshape(co_, co.kpad(ci))
    assert np.max(np.abs(gdw - rdw)) <= 1e-5 * np.max(np.abs(rdw))
    assert np.all(gdw[:, 9 * ci:] == 0)
    assert np.max(np.abs(host(db) - rdb)) <= 1e-5 * np.max(np.abs(rdb))


@pytest.mark.parametrize("ci,co_,mode", [(32, 32, 0), (16, 16, 2), (32, 16, 1)])
def test_conv_forward_many_segments_per_cta(ci, co_, mode):
    # more 128-pixel segments than resident CTAs: every CTA runs its staging / MMA /
    # epilogue pipeline over several segments and both halo stages
    rng = np.random.default_rng(11 + ci + co_ + mode)
    B, H, W = 2, 300, 150
    x = co.bf16(rng.standard_normal((B, H, W, ci)).astype(np.float32))
    w, b = rand_layer(rng, ci, co_)
    mask = co.bf16(rng.standard_normal((B, H, W, co_)).astype(np.float32)) if mode == 2 else None
    y = call_conv(dev_bf16(x), w, b if mode != 2 else None, dev_bf16(mask) if mode == 2 else None, B, H, W, ci, co_, mode)
    ref = co.conv3x3(x, w, None if mode == 2 else b)
    if mode == 0:
        ref = np.maximum(ref, 0)
    if mode == 2:
        ref = ref * (mask > 0)
    got = host(y).reshape(B, H, W, co_)
    tol = 1e-5 if mode == 1 else 8e-3
    assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref)), np.max(np.abs(got - ref))


@pytest.mark.parametrize("ci,co_", [(32, 32), (16, 32)])
def test_weight_gradient_many_segments_per_cta(ci, co_):
    rng = np.random.default_rng(5 + ci + co_)
    B, H, W = 2, 100, 133     # 400 segments: more than one CTA per SM can hold
    x = co.bf16(rng.standard_normal((B, H, W, ci)).astype(np.float32))
    dy = co.bf16(rng.standard_normal((B, H, W, co_)).astype(np.float32))
    lib, h = fem.solver._Handle.get()
    dw = torch.zeros(co_ * co.kpad(ci), dtype=torch.float32, device="cuda")
    xd, dyd = dev_bf16(x), dev_bf16(dy)
    rc = lib.femb200_conv3x3_weight_grad(h, ws._p(xd), ws._p(dyd), ws._p(dw), None, B, H, W, ci, co_)
    assert rc == 0
    torch.cuda.synchronize()
    _, rdw, _ = co.conv3x3_backward(x, np.zeros((co_, co.kpad(ci))), dy)
    gdw = host(dw).reshape(co_, co.kpad(ci))
    assert np.max(np.abs(gdw - rdw)) <= 1e-5 * np.max(np.abs(rdw))


def test_conv_rejects_misaligned_arrays():
    # the tensor-core kernels move 16 bytes per access: a view two bytes into a buffer is
    # refused before anything is launched
    lib, h = fem.solver._Handle.get()
    B, H, W, ci, co_ = 1, 4, 8, 16, 16
    x = torch.zeros(B * H * W * ci + 8, dtype=torch.bfloat16, device="cuda")
    wb = torch.zeros(co_ * co.kpad(ci), dtype=torch.bfloat16, device="cuda")
    bb = torch.zeros(co_, dtype=torch.float32, device="cuda")
    out = torch.empty(B * H * W * co_, dtype=torch.bfloat16, device="cuda")
    rc = lib.femb200_conv3x3_forward(h, ws._p(x[1:]), ws._p(wb), ws._p(bb), None, ws._p(out), B, H, W, ci, co_, 0)
    assert rc == 1 and b"16-byte aligned" in lib.femb200_last_error(h)
    dw = torch.zeros(co_ * co.kpad(ci), dtype=torch.float32, device="cuda")
    rc = lib.femb200_conv3x3_weight_grad(h, ws._p(x), ws._p(out[1:]), ws._p(dw), None, B, H, W, ci, co_)
    assert rc == 1 and b"16-byte aligned" in lib.femb200_last_error(h)
    rc = lib.femb200_conv3x3_forward(h, ws._p(x), ws._p(wb), ws._p(bb), None, ws._p(out), B, H, W, ci, co_, 0)
    assert rc == 0, lib.femb200_last_error(h)
    torch.cuda.synchronize()


def test_network_gradient_matches_oracle():
    # the whole 6-layer network: forward with BF16 activations, MSE, backward through
    # the ReLU masks; the oracle rounds at the same points
    rng = np.random.default_rng(3)
    net = ws.WarmStartNet(seed=1)
    B, H, W = 2, 9, 17
    x = co.bf16(rng.standard_normal((B, H, W, ws.IN_CH)).astype(np.float32))
    tgt = rng.standard_normal((B, H, W, 3)).astype(np.float32)
    xt = dev_bf16(x)
    net.zero_grad()
    out, acts = net.forward(xt, B, H, W, keep=True)
    npix = B * H * W
    scale = 1.0 / npix
    loss, dy = net.loss_grad(out, torch.as_tensor(tgt.reshape(-1), device="cuda"), npix, scale)
    net.backward(acts, dy, B, H, W)
    torch.cuda.synchronize()
    layers = [(host(L["wb"]).astype(np.float64), host(L["b"]).astype(np.float64), L["relu"]) for L in net.layers]
    # oracle forward with the library's rounding points
    a = [x.astype(np.float64)]
    for w, b, relu in layers:
        y = co.conv3x3(a[-1], w, b)
        a.append(co.bf16(np.maximum(y, 0).astype(np.float32)).astype(np.float64) if relu else y)
    rloss, g = co.mse(a[-1], tgt, 3, scale)
    assert abs(loss - rloss) <= 1e-3 * abs(rloss)
    dyr = co.bf16(g.astype(np.float32)).astype(np.float64)
    grads = [None] * len(layers)
    for li in range(len(layers) - 1, -1, -1):
        w, b, relu = layers[li]
        dx, dw, db = co.conv3x3_backward(a[li], w, dyr)
        grads[li] = (dw, db)
        if li > 0:
            dyr = co.bf16((dx * (a[li] > 0)).astype(np.float32)).astype(np.float64)
    for li, L in enumerate(net.layers):
        gw = host(L["gw"])
        rel = np.linalg.norm(gw - grads[li][0]) / np.linalg.norm(grads[li][0])
        relb = np.linalg.norm(host(L["gb"]) - grads[li][1]) / np.linalg.norm(grads[li][1])
        assert rel < 2e-2 and relb < 2e-2, (li, rel, relb)


def test_adam_matches_oracle():
    rng = np.random.default_rng(4)
    n = 1000
    w, m, v, g = [rng.standard_normal(n).astype(np.float32) for _ in range(4)]
    v = np.abs(v)
    t = [torch.as_tensor(a, device="cuda").contiguous() for a in (w, m, v, g)]
    wb = torch.empty(n, dtype=torch.bfloat16, device="cuda")
    lib, h = fem.solver._Handle.get()
    assert lib.femb200_adam_step(h, ws._p(t[0]), ws._p(t[1]), ws._p(t[2]), ws._p(t[3]), ws._p(wb), n, 1e-3, 0.9, 0.999,
                                 1e-8, 3) == 0
    torch.cuda.synchronize()
    rw, rm, rv = co.adam(w.astype(np.float64), m, v, g, 1e-3, 0.9, 0.999, 1e-8, 3)
    assert np.allclose(host(t[0]), rw, rtol=1e-5, atol=1e-6)
    assert np.allclose(host(t[1]), rm, rtol=1e-5, atol=1e-7)
    assert np.allclose(host(wb), co.bf16(host(t[0])))


def test_training_reduces_the_loss():
    # a smooth synthetic history: the network must learn its extrapolation correction
    H, W = 17, 25
    yy, xx = np.meshgrid(np.linspace(0, 1, H), np.linspace(0, 1, W), indexing="ij")
    F = []
    for t in range(8):
        f = np.stack([np.sin(2 * xx + 0.3 * t), np.cos(3 * yy - 0.2 * t ** 1.5), xx * yy * (1 + 0.1 * t ** 2),
                      np.exp(-xx) * (1 + 0.05 * t)], axis=-1).reshape(-1, 4)
        F.append(torch.as_tensor(f, dtype=torch.float32, device="cuda").contiguous())
    net = ws.WarmStartNet(seed=2, lr=2e-3)
    hist = net.train(F, H, W, epochs=80, batch=3)
    assert hist[-1] < 0.5 * hist[0], (hist[0], hist[-1])


def test_warm_started_time_loop_converges_to_the_plain_solution():
    res = ws.shear_band_warm_start(n=16, nsteps=14, ntrain=8, epochs=40, seed=0)
    later = [r for r in res["rows"] if "learned_iter" in r]
    assert later, "no warm-started steps"
    for r in res["rows"]:
        assert r["plain_converged"]
    for r in later:
        assert r["learned_converged"]
        # both runs stop on the same FP64 test: the warm start changes the path, not the answer
        assert r["learned_vs_plain_rel"] < 1e-6, r


def test_learned_start_saves_iterations_over_the_plain_start():
    # BASELINE's learned-warm-start workload, small: the shear band at 32², trained on
    # the first 14 converged steps and fine-tuned online on every later one. The start
    # from extrapolation + network must take at least 25 % fewer DR iterations than the
    # plain start over the test steps, and (the gain fades a network that does not help)
    # no more than 5 % more than extrapolation alone; both shares are printed.
    res = ws.shear_band_warm_start(n=32, nsteps=34, ntrain=14, epochs=60, seed=0, check_interval=50,
                                   online_steps=2)
    later = [r for r in res["rows"] if "learned_iter" in r]
    assert len(later) == 20
    plain = sum(r["plain_iter"] for r in later)
    extrap = sum(r["extrap_iter"] for r in later)
    learned = sum(r["learned_iter"] for r in later)
    print(f"DR iterations over {len(later)} steps: plain {plain}, extrapolation {extrap}, network {learned} "
          f"(network vs plain {learned / plain:.3f}, vs extrapolation {learned / extrap:.3f})")
    assert all(r["learned_converged"] for r in later)
    assert learned <= 0.75 * plain
    assert learned <= 1.05 * extrap
