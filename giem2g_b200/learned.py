"""Learned outer preconditioner for the nested FGMRES (configuration C4 of the build plan).

A 4-level 3-D convolutional U-Net (channels 16, 32, 64, 64) maps an outer Krylov vector v (3 complex field
components, 6 real channels scaled by the RMS of v) together with log10(sigma) and log10(frequency) to a
correction c, and the preconditioner returns z = v + rms(v) * c as its guess of A^-1 v: the contracting
IE operator is the identity plus a contraction, so A^-1 v = v + (correction).  The guess either starts the
inner GMRES cycle (mode 1, x0 = z instead of x0 = v) or is the outer preconditioned vector itself
(mode 2); see giem2g_set_outer_preconditioner.  The solver drops the net for the rest of a solve as soon as
a step through it fails to halve the FP64 Arnoldi misfit, so the plain inner GMRES is always the fallback.

Every convolution (forward, weight gradient, input gradient) runs on this library's kernels: 3x3x3
im2col (bf16), the tcgen05 BF16 GEMM with FP32 accumulation (giem2g_gemm_bf16_tn), and the gather-form
col2im.  Weights and activations enter the GEMMs in BF16; ReLU, nearest upsampling, concatenation, the
loss and Adam are plain PyTorch (device memory and autograd bookkeeping only).

Training pairs (v, e) satisfy A e = v exactly.  The default set comes from the solver's own Krylov
histories (make_pairs_krylov): for each training model and plane-wave source, the outer FGMRES iterates
x_k of a mixed-precision solve (k = 0 .. 6 outer iterations) give the residual r_k = b - A x_k and the error
e_k = x* - x_k against a tight FP64 solution x*, so A e_k = r_k; these are the vectors the outer
preconditioner sees during a solve.  An older set (make_pairs) uses smooth random fields e with v = A e and
the plane-wave solutions.  Models follow the C4 recipe: 64x64x16 cells of 100x100x50 m,
log10 sigma ~ GRF(mean -2, std 0.8, correlation 200-800 m), frequency log-uniform in [1e-2, 1e1] Hz.
"""
from __future__ import annotations

import json
import math
import os
import time

import numpy as np

from . import Giem2gError, IEOperator, _check, gemm_bf16_tn, lib

CH = (16, 32, 64, 64)
CIN = 8  # 6 field channels + log10 sigma + log10 frequency


def _stream_ptr():
    import torch
    return torch.cuda.current_stream().cuda_stream


def _kp(c):
    return ((27 * c + 7) // 8) * 8


def _conv_fn():
    import torch

    class Conv3dTC(torch.autograd.Function):
        """3x3x3 convolution, padding 1, stride 1 or 2, channels-last [N, D, H, W, C] float32 in and out."""

        @staticmethod
        def forward(ctx, x, w, stride):
            N, D, H, W, C = x.shape
            cout, kp = w.shape
            Do, Ho, Wo = (D - 1) // stride + 1, (H - 1) // stride + 1, (W - 1) // stride + 1
            xb = x.to(torch.bfloat16).contiguous()
            cols = torch.empty(N * Do * Ho * Wo, kp, dtype=torch.bfloat16, device=x.device)
            _check(lib().giem2g_im2col3d_bf16(xb.data_ptr(), cols.data_ptr(), N, D, H, W, C, stride, kp, _stream_ptr()),
                   "im2col3d")
            wb = w.to(torch.bfloat16).contiguous()
            y = gemm_bf16_tn(cols, wb)
            ctx.save_for_backward(cols, wb)
            ctx.geom = (N, D, H, W, C, stride, kp)
            return y.view(N, Do, Ho, Wo, cout)

        @staticmethod
        def backward(ctx, dy):
            cols, wb = ctx.saved_tensors
            N, D, H, W, C, stride, kp = ctx.geom
            cout = wb.shape[0]
            dyb = dy.reshape(-1, cout).to(torch.bfloat16).contiguous()
            dw = gemm_bf16_tn(dyb.t().contiguous(), cols.t().contiguous())       # [cout, kp]
            dcols = gemm_bf16_tn(dyb, wb.t().contiguous())                      # [V, kp]
            dx = torch.empty(N, D, H, W, C, dtype=torch.float32, device=dy.device)
            _check(lib().giem2g_col2im3d_f32(dcols.data_ptr(), dx.data_ptr(), N, D, H, W, C, stride, kp,
                                             _stream_ptr()), "col2im3d")
            return dx, dw, None

    return Conv3dTC


_CONV = None


def conv3d(x, w, stride=1):
    global _CONV
    if _CONV is None:
        _CONV = _conv_fn()
    return _CONV.apply(x, w, stride)


def _up(x):
    return x.repeat_interleave(2, dim=1).repeat_interleave(2, dim=2).repeat_interleave(2, dim=3)


class UNet3D:
    """Bias-free 4-level U-Net; weights are [Cout, Kp] matrices over (tap, channel) columns."""

    LAYERS = [  # name, Cin, Cout, stride
        ("in", CIN, CH[0], 1), ("e0", CH[0], CH[0], 1),
        ("d1", CH[0], CH[1], 2), ("e1", CH[1], CH[1], 1),
        ("d2", CH[1], CH[2], 2), ("e2", CH[2], CH[2], 1),
        ("d3", CH[2], CH[3], 2), ("b", CH[3], CH[3], 1),
        ("u2", CH[3] + CH[2], CH[2], 1), ("u1", CH[2] + CH[1], CH[1], 1),
        ("u0", CH[1] + CH[0], CH[0], 1), ("out", CH[0], 8, 1),
    ]

    def __init__(self, device="cuda", seed=0):
        import torch
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.w = {}
        for name, cin, cout, _ in self.LAYERS:
            w = torch.zeros(cout, _kp(cin))
            std = math.sqrt(2.0 / (27 * cin)) * (0.1 if name == "out" else 1.0)
            w[:, :27 * cin] = torch.randn(cout, 27 * cin, generator=g) * std
            self.w[name] = w.to(device).requires_grad_(True)
        self.stride = {name: s for name, _, _, s in self.LAYERS}

    def parameters(self):
        return list(self.w.values())

    def _c(self, name, x, relu=True):
        import torch
        y = conv3d(x, self.w[name], self.stride[name])
        return torch.relu(y) if relu else y

    def __call__(self, x):
        import torch
        e0 = self._c("e0", self._c("in", x))
        e1 = self._c("e1", self._c("d1", e0))
        e2 = self._c("e2", self._c("d2", e1))
        b = self._c("b", self._c("d3", e2))
        u2 = self._c("u2", torch.cat([_up(b), e2], dim=-1))
        u1 = self._c("u1", torch.cat([_up(u2), e1], dim=-1))
        u0 = self._c("u0", torch.cat([_up(u1), e0], dim=-1))
        return self._c("out", u0, relu=False)[..., :6]

    def state(self):
        return {k: v.detach().float().cpu().numpy() for k, v in self.w.items()}

    def load(self, state):
        import torch
        for k in self.w:
            self.w[k] = torch.from_numpy(np.asarray(state[k], np.float32)).to(self.w[k].device).requires_grad_(True)

    def save(self, path):
        np.savez_compressed(path, **{k: v.astype(np.float32) for k, v in self.state().items()})

    @classmethod
    def from_file(cls, path, device="cuda"):
        net = cls(device)
        with np.load(path) as d:
            net.load({k: d[k] for k in d.files})
        return net


# ---- field <-> network tensors -------------------------------------------------------------------
def encode(v, logsig, logf):
    """v: complex [3, Nz, Ny, Nx] (torch); returns ([1, Nz, Ny, Nx, 8] float32 input, rms)."""
    import torch
    rms = torch.sqrt(torch.mean(v.real ** 2 + v.imag ** 2)).clamp_min(1e-300)
    f = (v / rms).to(torch.complex64)
    chans = [f[c].real for c in range(3)] + [f[c].imag for c in range(3)]
    chans += [logsig, torch.full_like(logsig, logf)]
    return torch.stack(chans, dim=-1).unsqueeze(0).float(), rms


def decode(c, rms):
    """c: [1, Nz, Ny, Nx, 6] -> complex [3, Nz, Ny, Nx] scaled by rms."""
    import torch
    c = c[0]
    return torch.complex(c[..., 0:3].permute(3, 0, 1, 2), c[..., 3:6].permute(3, 0, 1, 2)).to(torch.complex128) * rms


def model_features(m, sig_file_order):
    """log10 sigma as [Nz, Ny, Nx] (normalised around -2) and log10 frequency."""
    import torch
    s = np.transpose(np.log10(sig_file_order), (2, 0, 1))  # [Nz, Ny, Nx]
    return torch.from_numpy(((s + 2.0) / 1.0).astype(np.float32)).cuda(), float(np.log10(m.freq) / 2.0)


# ---- training data ----------------------------------------------------------------------------------
def _smooth_field(shape, corr, gen):
    import torch
    nz, ny, nx = shape
    w = torch.randn(3, nz, ny, nx, dtype=torch.complex128, device="cuda", generator=gen)
    kz = torch.fft.fftfreq(nz, device="cuda").view(nz, 1, 1)
    ky = torch.fft.fftfreq(ny, device="cuda").view(1, ny, 1)
    kx = torch.fft.fftfreq(nx, device="cuda").view(1, 1, nx)
    filt = torch.exp(-(kx ** 2 + ky ** 2 + (kz * 2) ** 2) * (2 * math.pi * corr) ** 2 / 2)
    f = torch.fft.ifftn(torch.fft.fftn(w, dim=(1, 2, 3)) * filt, dim=(1, 2, 3))
    return f / torch.sqrt(torch.mean(f.real ** 2 + f.imag ** 2))


def make_pairs(n_models=512, pairs_per_model=3, seed=0, solve_pairs=True, log=print):
    """Exact pairs (input tensor, target correction) on 64x64x16 C4 models."""
    import torch
    from .sources import plane_wave_integral
    from .synthetic import config_c4
    gen = torch.Generator(device="cuda").manual_seed(seed)
    X, Y = [], []
    t0 = time.perf_counter()
    for i in range(n_models):
        m, sig = config_c4(seed=seed * 100003 + i)
        op = IEOperator.from_model(m)
        op.calc_ie_kernel(m.csigma, m.thick, m.omega)
        op.calc_fft_of_ie_kernel()
        op.set_anomaly_sigma(sig, m.freq)
        logsig, logf = model_features(m, sig)
        shape = (m.Nz, m.Ny, m.Nx)
        corrs = torch.rand(pairs_per_model, generator=torch.Generator().manual_seed(i)) * 7 + 1
        es = [_smooth_field(shape, float(c), gen) for c in corrs]
        vs = []
        for e in es:
            v = torch.empty_like(e)
            op.apply_device(e.data_ptr(), v.data_ptr(), 0)
            vs.append(v)
        if solve_pairs:
            b = torch.from_numpy(np.ascontiguousarray(plane_wave_integral(m, i % 2))).cuda()
            e = torch.empty_like(b)
            info = op.solve_device(b.data_ptr(), e.data_ptr(), None, tol=1e-8, precision=0)
            if info.stat == 1:
                # SolveEquation returns E = a chi; the operator acts on chi = E / a with rhs sqrt(Re sb) E0
                rhs = torch.empty_like(b)
                op.apply_device(e.data_ptr(), rhs.data_ptr(), 0)
                es.append(e)
                vs.append(rhs)
        for v, e in zip(vs, es):
            x, rms = encode(v, logsig, logf)
            corr = (e - v) / rms
            y = torch.stack([corr[c].real for c in range(3)] + [corr[c].imag for c in range(3)], dim=-1).float()
            X.append(x[0].to(torch.bfloat16))
            Y.append(y.to(torch.bfloat16))
        op.delete()
        if log and (i + 1) % 64 == 0:
            log(f"pairs: {i + 1}/{n_models} models, {len(X)} pairs, {time.perf_counter() - t0:.1f} s")
    return torch.stack(X), torch.stack(Y)


def _operator_system(m, sig, E0):
    """SolveEquation's system (ie_solver_module.F90:62-80): A chi = rhs with rhs = sqrt(Re sigma_b) E0 and
    E = a chi, a = 2 sqrt(Re sigma_b) / (csiga + conj sigma_b) per cell; returns (a, rhs) on the GPU."""
    import torch
    from .sources import _layer_numbers
    from .synthetic import csiga_from_sigma
    sb = m.csigma[_layer_numbers(m)[1:]]
    sq = np.sqrt(sb.real)
    a = 2.0 * sq[:, None, None] / (csiga_from_sigma(sig, m.freq) + np.conj(sb)[:, None, None])
    rhs = sq[None, :, None, None] * E0
    return torch.from_numpy(a).cuda(), torch.from_numpy(np.ascontiguousarray(rhs)).cuda()


def make_pairs_krylov(n_models=512, max_k=6, seed=0, log=print):
    """Residual/error pairs from the solver's own outer FGMRES histories on C4 models.

    The outer iterate after k steps, x_k, is what a solve with an outer basis of k and one restart cycle
    returns (the same Krylov space as the first k steps of the full solve); x_0 is the solver's start, the
    right-hand side.  r_k = b - A x_k takes one FP64 apply, e_k = x* - x_k uses a tight FP64 solution x*."""
    import torch
    from .sources import plane_wave_integral
    from .synthetic import config_c4
    X, Y = [], []
    t0 = time.perf_counter()
    for i in range(n_models):
        m, sig = config_c4(seed=seed * 100003 + i)
        op = IEOperator.from_model(m)
        op.calc_ie_kernel(m.csigma, m.thick, m.omega)
        op.calc_fft_of_ie_kernel()
        op.set_anomaly_sigma(sig, m.freq)
        logsig, logf = model_features(m, sig)
        E0 = plane_wave_integral(m, i % 2)
        a, rhs = _operator_system(m, sig, E0)
        b = torch.from_numpy(np.ascontiguousarray(E0).ravel()).cuda()
        E = torch.empty_like(b)
        ref = op.solve_device(b.data_ptr(), E.data_ptr(), None, tol=1e-10, precision=0)
        if ref.stat != 1:
            op.delete()
            continue
        xstar = E.view(3, *a.shape) / a
        chis = [rhs]
        for k in range(1, max_k + 1):
            info = op.solve_device(b.data_ptr(), E.data_ptr(), None, tol=1e-14, max_restart=1, outer_buf=k,
                                   precision=1)
            chis.append(E.view(3, *a.shape) / a)
            if info.iterations < k:
                break
        for chi in chis:
            Ax = torch.empty_like(chi)
            op.apply_device(chi.contiguous().data_ptr(), Ax.data_ptr(), 0)
            r = rhs - Ax
            e = xstar - chi
            x, rms = encode(r, logsig, logf)
            corr = (e - r) / rms
            y = torch.stack([corr[c].real for c in range(3)] + [corr[c].imag for c in range(3)], dim=-1).float()
            X.append(x[0].to(torch.bfloat16))
            Y.append(y.to(torch.bfloat16))
        op.delete()
        if log and (i + 1) % 64 == 0:
            log(f"Krylov pairs: {i + 1}/{n_models} models, {len(X)} pairs, {time.perf_counter() - t0:.1f} s")
    return torch.stack(X), torch.stack(Y)


def train(net, X, Y, steps=2000, batch=4, lr=1e-3, seed=0, log=print):
    """Adam on the relative squared error of the correction; returns the loss history."""
    import torch
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, steps)
    g = torch.Generator(device="cpu").manual_seed(seed)
    hist = []
    n = X.shape[0]
    for it in range(steps):
        idx = torch.randint(0, n, (batch,), generator=g)
        x, y = X[idx].float(), Y[idx].float()
        out = net(x)
        loss = ((out - y) ** 2).sum() / (y ** 2).sum().clamp_min(1e-12)
        opt.zero_grad(set_to_none=True)
        loss.backward()
        opt.step()
        sched.step()
        hist.append(float(loss.detach()))
        if log and (it + 1) % 200 == 0:
            log(f"train step {it + 1}/{steps}: loss {np.mean(hist[-200:]):.4f}")
    return hist


def evaluate(net, X, Y, batch=4):
    """Mean relative error of the correction and of the plain guess z = v (correction 0)."""
    import torch
    num, den = 0.0, 0.0
    with torch.no_grad():
        for i in range(0, X.shape[0], batch):
            x, y = X[i:i + batch].float(), Y[i:i + batch].float()
            num += float(((net(x) - y) ** 2).sum())
            den += float((y ** 2).sum())
    return num / max(den, 1e-300)


# ---- the solver hook ------------------------------------------------------------------------------
class _DevView:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<c16", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class LearnedPreconditioner:
    """Outer right preconditioner z = v + rms(v) * net(v, log sigma, log f) for one operator."""

    def __init__(self, net, m, sig_file_order):
        self.net = net
        self.shape = (3, m.Nz, m.Ny, m.Nx)
        self.logsig, self.logf = model_features(m, sig_file_order)
        self.calls = 0

    def __call__(self, d_v, d_z, n, stream):
        import torch
        with torch.cuda.stream(torch.cuda.ExternalStream(int(stream))), torch.no_grad():
            v = torch.as_tensor(_DevView(d_v, n), device="cuda").view(self.shape)
            z = torch.as_tensor(_DevView(d_z, n), device="cuda").view(self.shape)
            x, rms = encode(v, self.logsig, self.logf)
            z.copy_(v + decode(self.net(x), rms))
        self.calls += 1
        return 0

    def attach(self, op, mode=1):
        op.set_outer_preconditioner(mode, self)
        return self


def evaluate_solves(net, models, tol=1e-6, pols=(1, 0), log=print):
    """Outer iterations and device time of mixed-precision solves: plain inner GMRES vs the net as warm
    start of the inner cycle (mode 1) and as the whole outer preconditioner (mode 2)."""
    import torch
    from .sources import plane_wave_integral
    rows = []
    for m, sig in models:
        op = IEOperator.from_model(m)
        op.calc_ie_kernel(m.csigma, m.thick, m.omega)
        op.calc_fft_of_ie_kernel()
        op.set_anomaly_sigma(sig, m.freq)
        pre = LearnedPreconditioner(net, m, sig)
        for p in pols:
            b = torch.from_numpy(np.ascontiguousarray(plane_wave_integral(m, p)).ravel()).cuda()
            y = torch.empty_like(b)
            row = {"grid": [m.Nx, m.Ny, m.Nz], "freq": m.freq, "pol": p}
            for label, mode in (("plain", 0), ("net_warm_start", 1), ("net_only", 2)):
                if mode:
                    pre.attach(op, mode)
                else:
                    op.set_outer_preconditioner(0)
                op.solve_device(b.data_ptr(), y.data_ptr(), None, tol=tol, precision=1)  # warm-up / capture
                info = op.solve_device(b.data_ptr(), y.data_ptr(), None, tol=tol, precision=1)
                row[label] = {"iterations": info.iterations, "stat": info.stat, "be": info.be,
                              "device_ms": info.device_ms, "applies": info.applies_fp64 + info.applies_fp32,
                              "net_steps": info.precond_steps}
            op.set_outer_preconditioner(0)
            rows.append(row)
            if log:
                log(json.dumps(row))
        op.delete()
    return rows


WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "unet3d_c4.npz")


def main(argv=None):
    import argparse
    import torch
    ap = argparse.ArgumentParser(description="train the learned outer preconditioner on C4 models")
    ap.add_argument("--models", type=int, default=512)
    ap.add_argument("--pairs", type=int, default=3, help="smooth-field pairs per model (--data smooth)")
    ap.add_argument("--data", default="krylov", choices=["krylov", "smooth"],
                    help="training pairs: the solver's Krylov histories (default) or smooth random fields")
    ap.add_argument("--max-k", type=int, default=6, help="outer iterates per model (--data krylov)")
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--eval", default=None, help="only evaluate the weights in this file on solves")
    args = ap.parse_args(argv)
    import giem2g_b200 as g2
    from .synthetic import config_c2, config_c4
    g2.set_logger(lambda s: None)
    if args.eval:
        net = UNet3D.from_file(args.eval)
        models = [config_c4(seed=70001 + i) for i in range(4)] + [config_c2(seed=4242)]
        rows = evaluate_solves(net, models)
        print(json.dumps({"eval": rows}))
        return
    t0 = time.perf_counter()
    if args.data == "krylov":
        X, Y = make_pairs_krylov(args.models, args.max_k, seed=1)
    else:
        X, Y = make_pairs(args.models, args.pairs, seed=1)
    t_data = time.perf_counter() - t0
    nval = max(8, X.shape[0] // 16)
    Xv, Yv = X[:nval], Y[:nval]
    Xt, Yt = X[nval:], Y[nval:]
    net = UNet3D()
    base = evaluate(net, Xv, Yv)
    t1 = time.perf_counter()
    hist = train(net, Xt, Yt, steps=args.steps, batch=args.batch, lr=args.lr)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    val = evaluate(net, Xv, Yv)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    net.save(args.out)
    print(json.dumps({"data": args.data, "pairs": int(X.shape[0]), "data_s": t_data, "train_s": t_train, "steps": args.steps,
                      "val_rel_err_untrained": base, "val_rel_err": val, "final_train_loss": float(np.mean(hist[-100:])),
                      "weights": args.out}))


if __name__ == "__main__":
    main()
