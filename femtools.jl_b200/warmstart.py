"""Learned warm start of the dynamic-relaxation time loop (no reference counterpart).

A 6-layer 3×3 convolutional network (32 channels, BF16 weights and activations,
FP32 accumulation; libfemtools_b200's tensor-core kernels for the forward pass, the
data and weight gradients, the loss and Adam) maps the converged fields of the two
previous time steps on the (2n+1)² node grid of a structured Q9/P1-disc mesh —
vx, vy, P and ε̇II per step — to the next step's correction to linear extrapolation
of (vx, vy, P). It is trained on the solver's own converged history; afterwards the
DR solve of each step starts from extrapolation + prediction instead of the previous
step's solution. The plain DR iteration still runs to the same tolerance from that
start, so the network can only change how many iterations a step takes, never the
answer it converges to.

The network's output is multiplied by a gain g ∈ [0, 1]: fitted on held-out training
pairs, then (by default) recalibrated after every solved step by least squares of the
network's predictions against the corrections the solver actually produced over the
last few steps, so that a network that stops matching the dynamics fades to plain
extrapolation instead of adding error.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np
import torch

from . import solver as _solver
from .autodiff import DRCheckpoint

HIDDEN = 32
IN_CH = 16      # 8 used: (vx, vy, P, ε̇II) of two steps
OUT_CH = 16     # 3 used: corrections of vx, vy, P
N_TARGET = 3


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _lib():
    return _solver._Handle.get()


def _check(rc):
    lib, h = _lib()
    _solver._check(lib, h, rc)


class GridMap:
    """Node grid of a structured Q9 mesh (nodes x-fastest): the element owning each
    node and the node's local (ξ, η) in it, for evaluating the P1-disc pressure."""

    def __init__(self, mesh):
        if mesh.dim != 2 or mesh.nv != 9:
            raise ValueError("the warm start works on structured Q9/P1-disc meshes")
        nx, ny = 2 * mesh.nel[0] + 1, 2 * mesh.nel[1] + 1
        if nx * ny != mesh.nnodes:
            raise ValueError("not a structured node grid")
        loc = np.array([(-1, -1), (1, -1), (1, 1), (-1, 1), (0, -1), (1, 0), (0, 1), (-1, 0), (0, 0)], dtype=np.int8)
        elem = np.zeros(mesh.nnodes, dtype=np.int32)
        xi = np.zeros(mesh.nnodes, dtype=np.int8)
        eta = np.zeros(mesh.nnodes, dtype=np.int8)
        nodes = mesh.el2n - 1
        for a in range(9):
            elem[nodes[:, a]] = np.arange(mesh.nels, dtype=np.int32)
            xi[nodes[:, a]] = loc[a, 0]
            eta[nodes[:, a]] = loc[a, 1]
        dev = torch.device("cuda")
        self.nx, self.ny = nx, ny
        self.dx = (mesh.coords[1, 0] - mesh.coords[0, 0])
        self.dy = (mesh.coords[nx, 1] - mesh.coords[0, 1])
        self.elem = torch.as_tensor(elem, device=dev)
        self.xi = torch.as_tensor(xi, device=dev)
        self.eta = torch.as_tensor(eta, device=dev)

    def fields(self, dr):
        """(vx, vy, P, ε̇II) on the node grid, FP32, shape (ny·nx, 4)."""
        lib, h = _lib()
        out = torch.empty(self.nx * self.ny * 4, dtype=torch.float32, device=dr.device)
        _check(lib.femb200_q9_grid_fields(h, C.byref(dr.problem()), _p(self.elem), _p(self.xi), _p(self.eta), self.nx,
                                          self.ny, float(self.dx), float(self.dy), _p(out)))
        return out.view(-1, 4)


class WarmStartNet:
    """The network's parameters (FP32 masters, BF16 copies, data-gradient copies) and
    its training state; every operation runs on libfemtools_b200 kernels."""

    def __init__(self, seed=0, hidden=HIDDEN, depth=6, lr=1e-3):
        dev = torch.device("cuda")
        g = torch.Generator().manual_seed(seed)
        chans = [IN_CH] + [hidden] * (depth - 1) + [OUT_CH]
        self.layers = []
        for i in range(depth):
            ci, co = chans[i], chans[i + 1]
            kp = 9 * ci + 8
            fan_in = 9 * ci
            bound = math.sqrt(6.0 / fan_in) * (0.1 if i == depth - 1 else 1.0)
            w = torch.zeros(co, kp)
            w[:, :9 * ci] = (torch.rand(co, 9 * ci, generator=g) * 2 - 1) * bound
            L = {"ci": ci, "co": co, "relu": i < depth - 1,
                 "w": w.to(dev), "b": torch.zeros(co, device=dev)}
            for k in ("mw", "vw", "gw"):
                L[k] = torch.zeros_like(L["w"])
            for k in ("mb", "vb", "gb"):
                L[k] = torch.zeros_like(L["b"])
            L["wb"] = torch.empty(co, kp, dtype=torch.bfloat16, device=dev)
            L["wT"] = torch.empty(ci, 9 * co + 8, dtype=torch.bfloat16, device=dev)
            self.layers.append(L)
        self.lr = lr
        self.step = 0
        self.field_scale = torch.ones(4, device=dev)
        self.gain = 1.0
        self._sync_bf16()

    def _sync_bf16(self):
        lib, h = _lib()
        for L in self.layers:
            _check(lib.femb200_f32_to_bf16(h, _p(L["w"]), _p(L["wb"]), L["w"].numel()))
            _check(lib.femb200_conv3x3_flip_weights(h, _p(L["wb"]), _p(L["wT"]), L["ci"], L["co"]))

    def forward(self, x, B, H, W, keep=False):
        """x: BF16 NHWC (B, H, W, 16). Returns the FP32 output (B, H, W, 16) and, with
        keep, the BF16 activations of every layer for the backward pass."""
        lib, h = _lib()
        acts = [x]
        cur = x
        for L in self.layers:
            if L["relu"]:
                out = torch.empty(B * H * W * L["co"], dtype=torch.bfloat16, device=x.device)
                mode = 0
            else:
                out = torch.empty(B * H * W * L["co"], dtype=torch.float32, device=x.device)
                mode = 1
            _check(lib.femb200_conv3x3_forward(h, _p(cur), _p(L["wb"]), _p(L["b"]), None, _p(out), B, H, W, L["ci"],
                                               L["co"], mode))
            cur = out
            if keep:
                acts.append(out)
        return cur, acts

    def backward(self, acts, dout, B, H, W):
        """Accumulate parameter gradients for the BF16 output gradient dout."""
        lib, h = _lib()
        dy = dout
        for li in range(len(self.layers) - 1, -1, -1):
            L = self.layers[li]
            _check(lib.femb200_conv3x3_weight_grad(h, _p(acts[li]), _p(dy), _p(L["gw"]), _p(L["gb"]), B, H, W, L["ci"],
                                                   L["co"]))
            if li > 0:
                below = self.layers[li - 1]
                dx = torch.empty(B * H * W * L["ci"], dtype=torch.bfloat16, device=dout.device)
                # data gradient through this layer, masked by the ReLU of the layer below
                _check(lib.femb200_conv3x3_forward(h, _p(dy), _p(L["wT"]), None, _p(acts[li]), _p(dx), B, H, W,
                                                   L["co"], L["ci"], 2))
                dy = dx

    def zero_grad(self):
        for L in self.layers:
            L["gw"].zero_()
            L["gb"].zero_()

    def adam(self, b1=0.9, b2=0.999, eps=1e-8):
        lib, h = _lib()
        self.step += 1
        for L in self.layers:
            _check(lib.femb200_adam_step(h, _p(L["w"]), _p(L["mw"]), _p(L["vw"]), _p(L["gw"]), _p(L["wb"]),
                                         L["w"].numel(), self.lr, b1, b2, eps, self.step))
            _check(lib.femb200_adam_step(h, _p(L["b"]), _p(L["mb"]), _p(L["vb"]), _p(L["gb"]), None, L["b"].numel(),
                                         self.lr, b1, b2, eps, self.step))
            _check(lib.femb200_conv3x3_flip_weights(h, _p(L["wb"]), _p(L["wT"]), L["ci"], L["co"]))

    def loss_grad(self, out, target, npix, scale):
        """scale·Σ (out − target)² over the 3 target channels and its BF16 gradient."""
        lib, h = _lib()
        dy = torch.empty(npix * OUT_CH, dtype=torch.bfloat16, device=out.device)
        loss = C.c_double()
        _check(lib.femb200_mse_loss_grad(h, _p(out), _p(target), N_TARGET, OUT_CH, float(scale), _p(dy), npix,
                                         C.byref(loss)))
        return loss.value, dy

    # ---- data of the time loop ----
    # The fields are scaled by their spread over the training history; the step change
    # F_t − F_{t−1} and the target (the next step's correction to linear
    # extrapolation) by the RMS of the current step change, per field, so that the
    # network predicts a dimensionless correction and its output shrinks with the
    # dynamics of the step it is applied to.
    @staticmethod
    def step_rms(Fp, Fc):
        return (Fc - Fp).pow(2).mean(dim=0).sqrt().clamp_min(1e-30).float()

    def make_input(self, Fp, Fc):
        lib, h = _lib()
        npix = Fp.shape[0]
        X = torch.empty(npix * IN_CH, dtype=torch.bfloat16, device=Fp.device)
        scale = torch.cat([self.field_scale, self.step_rms(Fp, Fc)]).contiguous()
        _check(lib.femb200_net_input(h, _p(Fp), _p(Fc), _p(scale), _p(X), npix))
        return X

    def make_target(self, Fp, Fc, Fn):
        lib, h = _lib()
        npix = Fp.shape[0]
        T = torch.empty(npix * N_TARGET, dtype=torch.float32, device=Fp.device)
        scale = self.step_rms(Fp, Fc)[:N_TARGET].contiguous()
        _check(lib.femb200_net_target(h, _p(Fp), _p(Fc), _p(Fn), _p(scale), _p(T), npix))
        return T

    def output_scale(self, Fp, Fc):
        """Host scales of the network's output channels for the step (Fp, Fc), gain included."""
        return [self.gain * float(x) for x in self.step_rms(Fp, Fc)[:N_TARGET].cpu()]

    def fit_scales(self, F):
        stack = torch.stack(F)                            # steps × npix × 4
        self.field_scale = stack.std(dim=(0, 1)).clamp_min(1e-12).float().contiguous()

    def train(self, F, H, W, epochs=200, batch=8, seed=0):
        """Fit on the history F[0..n−1] of grid fields: inputs (F[t−1], F[t]), targets the
        correction of F[t+1] to linear extrapolation. Returns the loss per epoch."""
        self.fit_scales(F)
        X = [self.make_input(F[t - 1], F[t]) for t in range(1, len(F) - 1)]
        T = [self.make_target(F[t - 1], F[t], F[t + 1]) for t in range(1, len(F) - 1)]
        # the latest pairs are held out to set the output gain
        nval = max(1, len(X) // 5) if len(X) > 2 else 0
        Xv, Tv = X[len(X) - nval:], T[len(T) - nval:]
        X, T = X[:len(X) - nval], T[:len(T) - nval]
        n = len(X)
        npix = H * W
        rng = np.random.default_rng(seed)
        hist = []
        for _ in range(epochs):
            order = rng.permutation(n)
            tot = 0.0
            for s0 in range(0, n, batch):
                idx = order[s0:s0 + batch]
                xb = torch.cat([X[i] for i in idx])
                tb = torch.cat([T[i] for i in idx])
                B = len(idx)
                self.zero_grad()
                out, acts = self.forward(xb, B, H, W, keep=True)
                loss, dy = self.loss_grad(out, tb, B * npix, 1.0 / (n * npix))
                self.backward(acts, dy, B, H, W)
                self.adam()
                tot += loss
            hist.append(tot)
        # gain g ∈ [0, 1] minimising Σ |g·prediction − target|² on the held-out pairs: a
        # network that does not beat extrapolation on unseen steps gets switched off
        num = den = 0.0
        for x, t in zip(Xv, Tv):
            out, _ = self.forward(x, 1, H, W)
            pr = out.view(-1, OUT_CH)[:, :N_TARGET]
            num += float((pr * t.view(-1, N_TARGET)).sum())
            den += float((pr * pr).sum())
        self.gain = min(max(num / den, 0.0), 1.0) if den > 0 else (1.0 if not Xv else 0.0)
        return hist

    def train_online(self, pairs, H, W, steps=2, batch=4):
        """`steps` Adam steps on the newest training pairs (X, T) of the time loop: each
        batch holds the newest pair and up to batch − 1 earlier ones, so the network
        follows the solver's converged history as the dynamics change."""
        if not pairs or steps <= 0:
            return
        npix = H * W
        n = len(pairs)
        for k in range(steps):
            idx = [n - 1] + [n - 2 - ((k * (batch - 1) + j) % max(n - 1, 1)) for j in range(min(batch - 1, n - 1))]
            xb = torch.cat([pairs[i][0] for i in idx])
            tb = torch.cat([pairs[i][1] for i in idx])
            B = len(idx)
            self.zero_grad()
            out, acts = self.forward(xb, B, H, W, keep=True)
            _, dy = self.loss_grad(out, tb, B * npix, 1.0 / (B * npix))
            self.backward(acts, dy, B, H, W)
            self.adam()

    def predict(self, Fp, Fc, H, W):
        out, _ = self.forward(self.make_input(Fp, Fc), 1, H, W)
        return out


def apply_guess(dr, bc_v, vprev, vcur, Pprev, Pcur, out=None, scale=None):
    """v, P of dr ← 2·cur − prev (+ the network's correction `out`, FP32 (npix, 16),
    scaled by `scale`); Dirichlet nodes keep their values."""
    lib, h = _lib()
    vp = (C.c_void_p * 2)(*[C.c_void_p(x.data_ptr()) for x in vprev])
    vc = (C.c_void_p * 2)(*[C.c_void_p(x.data_ptr()) for x in vcur])
    sc = (C.c_float * 3)(*[float(x) for x in scale]) if scale is not None else None
    _check(lib.femb200_apply_warm_start(h, C.byref(dr.problem(bc_v)), vp, vc, _p(Pprev), _p(Pcur), _p(out), OUT_CH,
                                        sc))


def extrapolate_state(dr, bc_v, vprev, vcur, Pprev, Pcur):
    """v, P of dr ← 2·cur − prev (2-D or 3-D); Dirichlet DoFs keep their values."""
    lib, h = _lib()
    z = vcur[0]
    vp = (C.c_void_p * 3)(*[C.c_void_p(x.data_ptr()) for x in (list(vprev) + [z] * 3)[:3]])
    vc = (C.c_void_p * 3)(*[C.c_void_p(x.data_ptr()) for x in (list(vcur) + [z] * 3)[:3]])
    _check(lib.femb200_extrapolate_state(h, C.byref(dr.problem(bc_v)), vp, vc, _p(Pprev), _p(Pcur)))


def shear_band_warm_start(n=256, nsteps=200, ntrain=50, epochs=200, seed=0, tolerance=1e-8, check_interval=100,
                          log=None, online_gain=True, gain_window=5, online_steps=0, replay=8, online_batch=4):
    """The learned-warm-start experiment on the 2-D shear-band time loop.

    Steps 1..ntrain run plain DR (each from the previous step's solution) and record
    the converged fields; the network is then trained on them. For every later step
    the same state is solved three times, each to `tolerance`: plain (from the
    previous solution), linear extrapolation 2·x_t − x_{t−1}, and extrapolation plus
    the network's correction; the trajectory continues with the plain solution, so
    all three see identical histories. With `online_steps` > 0 the network keeps
    training after every solved step: that many Adam steps on the newest `replay`
    pairs of the converged history in batches of `online_batch`, their time charged to
    the network's arm.
    Returns per-step iteration counts and times."""
    from . import configs
    case = configs.shear_band_2d_case(n=n, seed=seed)
    dr = case.device_state()
    bc = case.bc_device()
    gm = GridMap(case.mesh)
    H, W = gm.ny, gm.nx
    kw = dict(dt=case.dt, tolerance=tolerance, check_interval=check_interval, throw_on_failure=False,
              max_iterations=2_000_000, iter_max=2_000_000)
    net = WarmStartNet(seed=seed)
    F = []
    hist_v, hist_P = [], []
    rows = []
    cal = []          # (⟨prediction, realised correction⟩, ⟨prediction, prediction⟩) per solved step
    pending = None
    pairs = []        # (input, target) of the converged history since training, newest last
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    train_loss, train_ms = None, 0.0

    def timed_solve():
        ev0.record()
        st = _solver.solve(dr, bc, **kw)
        ev1.record()
        torch.cuda.synchronize()
        return st, ev0.elapsed_time(ev1)

    for step in range(1, nsteps + 1):
        dr.P0.copy_(dr.P)
        row = {"step": step}
        if step > ntrain and len(F) >= 2:
            ck = DRCheckpoint(dr)
            st, ms = timed_solve()
            row.update(plain_iter=st["iter"], plain_ms=ms, plain_converged=bool(st["converged"]))
            plain = DRCheckpoint(dr)
            # linear extrapolation
            ck.restore(dr)
            ev0.record()
            apply_guess(dr, bc, hist_v[-2], hist_v[-1], hist_P[-2], hist_P[-1])
            st, ms = timed_solve()
            row.update(extrap_iter=st["iter"], extrap_ms=ms)
            # extrapolation + network
            ck.restore(dr)
            e0 = torch.cuda.Event(enable_timing=True)
            e0.record()
            out = net.predict(F[-2], F[-1], H, W)
            scale = net.output_scale(F[-2], F[-1])
            pending = (out.view(-1, OUT_CH)[:, :N_TARGET] * net.step_rms(F[-2], F[-1])[:N_TARGET]).clone() \
                if online_gain else None
            apply_guess(dr, bc, hist_v[-2], hist_v[-1], hist_P[-2], hist_P[-1], out, scale)
            e1 = torch.cuda.Event(enable_timing=True)
            e1.record()
            st, ms = timed_solve()
            row.update(learned_iter=st["iter"], learned_ms=ms + e0.elapsed_time(e1), learned_converged=bool(st["converged"]),
                       infer_ms=e0.elapsed_time(e1))
            ws_v = [x.clone() for x in dr.v]
            plain.restore(dr)
            row["learned_vs_plain_rel"] = float(
                torch.linalg.norm(torch.cat(ws_v) - torch.cat(list(dr.v))) / torch.linalg.norm(torch.cat(list(dr.v))))
        else:
            st, ms = timed_solve()
            row.update(plain_iter=st["iter"], plain_ms=ms, plain_converged=bool(st["converged"]))
        _solver.update_stokes_current_stress(dr, case.dt)
        for c in range(3):
            dr.tau_old[c].copy_(dr.tau[c])
        F.append(gm.fields(dr).clone())
        if online_gain and pending is not None and len(F) >= 3:
            # calibrate the gain on the step just solved: the realised correction to
            # linear extrapolation against the network's (unit-gain) prediction for it
            real = F[-1][:, :N_TARGET] - (2 * F[-2][:, :N_TARGET] - F[-3][:, :N_TARGET])
            cal.append((float((pending * real).sum()), float((pending * pending).sum())))
            num = sum(a for a, _ in cal[-gain_window:])
            den = sum(b for _, b in cal[-gain_window:])
            if den > 0:
                net.gain = min(max(num / den, 0.0), 1.0)
            row["gain"] = net.gain
            pending = None
        if online_steps > 0 and step > ntrain and len(F) >= 3:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            pairs.append((net.make_input(F[-3], F[-2]), net.make_target(F[-3], F[-2], F[-1])))
            pairs = pairs[-replay:]
            net.train_online(pairs, H, W, steps=online_steps, batch=online_batch)
            e1.record()
            torch.cuda.synchronize()
            row["online_train_ms"] = e0.elapsed_time(e1)
            if "learned_ms" in row:
                row["learned_ms"] += row["online_train_ms"]
        hist_v.append([x.clone() for x in dr.v])
        hist_P.append(dr.P.clone())
        if len(hist_v) > 2:
            hist_v.pop(0)
            hist_P.pop(0)
        if step == ntrain:
            t0 = time.perf_counter()
            train_loss = net.train(F, H, W, epochs=epochs, seed=seed)
            torch.cuda.synchronize()
            train_ms = (time.perf_counter() - t0) * 1e3
            F = F[-3:]
        elif step > ntrain:
            F = F[-3:]
        rows.append(row)
        if log:
            log(row)
    return {"rows": rows, "train_loss": train_loss, "train_ms": train_ms, "n": n, "nsteps": nsteps, "ntrain": ntrain,
            "epochs": epochs, "gain": net.gain}
