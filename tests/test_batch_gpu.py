"""Batched applies and batched (lockstep) solves against the single-instance path and the oracle.

Tolerances: complex64 applies 2e-5 relative to the oracle (as the single apply); FP64 batched solves
reproduce the single solves (same iteration counts and status, solutions within 1e-12); mixed batched
solves keep the single solves' status and reach the FP64 solution within 1e-5.
"""
import numpy as np
import pytest

from giem2g_b200.sources import plane_wave_integral
from giem2g_b200.synthetic import config_small_block, csiga_from_sigma
from tests.helpers import random_sigma, random_spatial_tensor, random_vec, rel, tiny_model

pytestmark = pytest.mark.gpu

TOL32 = 2e-5


def _op_random(g2, m, seed=3):
    symm, asym = random_spatial_tensor(m, seed=seed)
    op = g2.IEOperator.from_model(m)
    op.set_background(m.csigma, m.thick, m.omega)
    op.set_ie_kernel_spatial(symm, asym)
    op.calc_fft_of_ie_kernel()
    sig = random_sigma(m, seed)
    op.set_anomaly_conductivity(csiga_from_sigma(sig, m.freq))
    return op, symm, asym, sig


@pytest.mark.parametrize("shape", [(8, 8, 8), (4, 8, 16), (4, 4, 32), (2, 4, 48), (8, 4, 5)])
def test_pair_apply_matches_oracle(g2lib, orc, shape):
    import torch
    m = tiny_model(*shape)
    op, symm, asym, sig = _op_random(g2lib, m)
    csigb, sqsigb = orc.background_cells(m)
    sh, ah = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, symm, asym)
    csiga = csiga_from_sigma(sig, m.freq)
    vs = [random_vec(m, s) for s in (21, 22, 23)]
    d_in = [torch.from_numpy(v.ravel()).to("cuda", torch.complex64) for v in vs]
    d_out = [torch.empty_like(x) for x in d_in]
    g2lib.apply_device_batch(op, [x.data_ptr() for x in d_in], [y.data_ptr() for y in d_out], 1)
    single = torch.empty_like(d_in[0])
    for v, x, y in zip(vs, d_in, d_out):
        ref = orc.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, v)
        got = y.cpu().numpy().astype(np.complex128).reshape(ref.shape)
        assert rel(got, ref) < TOL32
        op.apply_device(x.data_ptr(), single.data_ptr(), 1)
        torch.cuda.synchronize()
        assert rel(got, single.cpu().numpy().astype(np.complex128).reshape(ref.shape)) < TOL32
    op.check_device_error()
    op.delete()


def test_batch_apply_fp64_equals_single(g2lib):
    import torch
    m = tiny_model(8, 8, 6)
    op, *_ = _op_random(g2lib, m)
    d_in = [torch.from_numpy(random_vec(m, s).ravel()).to("cuda") for s in (1, 2, 3)]
    d_out = [torch.empty_like(x) for x in d_in]
    g2lib.apply_device_batch(op, [x.data_ptr() for x in d_in], [y.data_ptr() for y in d_out], 0)
    for x, y in zip(d_in, d_out):
        ref = torch.empty_like(x)
        op.apply_device(x.data_ptr(), ref.data_ptr(), 0)
        torch.cuda.synchronize()
        assert torch.equal(y, ref)
    op.delete()


def _two_frequency_setup(g2):
    m1, sig = config_small_block()
    m2 = m1.with_freq(10.0)
    ops = []
    for m in (m1, m2):
        op = g2.IEOperator.from_model(m)
        op.calc_ie_kernel(m.csigma, m.thick, m.omega)
        op.calc_fft_of_ie_kernel()
        op.set_anomaly_sigma(sig, m.freq)
        ops.append(op)
    # instances: (1 Hz, EY), (1 Hz, EX), (10 Hz, EY)
    inst = [(ops[0], plane_wave_integral(m1, 1)), (ops[0], plane_wave_integral(m1, 0)),
            (ops[1], plane_wave_integral(m2, 1))]
    return ops, inst


@pytest.mark.parametrize("precision,tol", [(0, 1e-8), (1, 1e-6)])
def test_batched_solve_matches_single(g2lib, precision, tol):
    import torch
    ops, inst = _two_frequency_setup(g2lib)
    d_e = [torch.from_numpy(np.ascontiguousarray(e).ravel()).to("cuda") for _, e in inst]
    d_s = [torch.empty_like(x) for x in d_e]
    single, infos1 = [], []
    for (op, _), x in zip(inst, d_e):
        y = torch.empty_like(x)
        infos1.append(op.solve_device(x.data_ptr(), y.data_ptr(), None, tol=tol, precision=precision))
        single.append(y)
    ref64 = []
    for (op, _), x in zip(inst, d_e):
        y = torch.empty_like(x)
        op.solve_device(x.data_ptr(), y.data_ptr(), None, tol=1e-10, precision=0)
        ref64.append(y)
    b = g2lib.Batch([op for op, _ in inst], precision=precision)
    infos = b.solve_device([x.data_ptr() for x in d_e], [y.data_ptr() for y in d_s], tol=tol)
    torch.cuda.synchronize()
    for i in range(len(inst)):
        assert infos[i].stat == infos1[i].stat == 1
        assert len(infos[i].misfits) == infos[i].iterations
        if precision == 0:
            assert infos[i].iterations == infos1[i].iterations
            assert rel(d_s[i].cpu().numpy(), single[i].cpu().numpy()) < 1e-12
            assert np.allclose(infos[i].misfits, infos1[i].misfits, rtol=1e-10, atol=0)
        else:
            assert abs(infos[i].iterations - infos1[i].iterations) <= 1
            assert infos[i].be < tol
            assert rel(d_s[i].cpu().numpy(), ref64[i].cpu().numpy()) < 1e-5
    # the host-array entry point gives the device result
    outs, infos_h = b.solve([e for _, e in inst], tol=tol)
    for i in range(len(inst)):
        assert infos_h[i].iterations == infos[i].iterations
        assert rel(outs[i].ravel(), d_s[i].cpu().numpy()) < 1e-12
    b.delete()
    for op in ops:
        op.delete()


def test_batched_solve_zero_rhs_instance(g2lib):
    import torch
    ops, inst = _two_frequency_setup(g2lib)
    d_e = [torch.from_numpy(np.ascontiguousarray(inst[0][1]).ravel()).to("cuda"),
           torch.zeros(ops[0].nvec, dtype=torch.complex128, device="cuda")]
    d_s = [torch.full_like(x, 1.0) for x in d_e]
    b = g2lib.Batch([ops[0], ops[0]], precision=1)
    infos = b.solve_device([x.data_ptr() for x in d_e], [y.data_ptr() for y in d_s], tol=1e-6)
    torch.cuda.synchronize()
    assert infos[0].stat == 1 and infos[0].iterations > 0
    assert infos[1].stat == 1 and infos[1].iterations == 0
    assert float(d_s[1].abs().max()) == 0.0
    b.delete()
    for op in ops:
        op.delete()


def test_eight_instance_sweep_batch(g2lib, orc):
    """Four frequencies x two polarisations (8 lockstep instances, the multi-frequency sweep's form) on a
    32x32x32 model whose applies take the fused y-pass: in FP64 every instance reproduces its own single solve
    (iterations, status, solution within 1e-12); in mixed precision every instance converges to outer
    relative residual 1e-6 and lies within 1e-5 of its FP64 solution (tol 1e-10).  One FP64 solution is put
    back through the oracle's apply of the same tensor: its recomputed relative residual stays within 1.5x
    the tolerance."""
    import torch
    from giem2g_b200.synthetic import config_grf
    m0, sig = config_grf(32, 32, 32, seed=9)
    freqs = [0.01, 0.3, 3.0, 30.0]
    ops, inst = [], []
    for f in freqs:
        m = m0.with_freq(f)
        op = g2lib.IEOperator.from_model(m)
        op.calc_ie_kernel(m.csigma, m.thick, m.omega)
        op.calc_fft_of_ie_kernel()
        op.set_anomaly_sigma(sig, m.freq)
        ops.append((m, op))
        for pol in (1, 0):
            inst.append((m, op, plane_wave_integral(m, pol)))
    assert len(inst) == 8
    d_e = [torch.from_numpy(np.ascontiguousarray(e).ravel()).to("cuda") for _, _, e in inst]
    ref64, single64 = [], []
    for (_, op, _), x in zip(inst, d_e):
        y = torch.empty_like(x)
        op.solve_device(x.data_ptr(), y.data_ptr(), None, tol=1e-10, precision=0)
        ref64.append(y)
        y8 = torch.empty_like(x)
        single64.append((op.solve_device(x.data_ptr(), y8.data_ptr(), None, tol=1e-8, precision=0), y8))
    for precision, tol in ((0, 1e-8), (1, 1e-6)):
        d_s = [torch.empty_like(x) for x in d_e]
        b = g2lib.Batch([op for _, op, _ in inst], precision=precision)
        infos = b.solve_device([x.data_ptr() for x in d_e], [y.data_ptr() for y in d_s], tol=tol)
        torch.cuda.synchronize()
        for i, info in enumerate(infos):
            assert info.stat == 1 and info.be < tol, (precision, i, info)
            if precision == 0:
                s_info, s_y = single64[i]
                assert info.iterations == s_info.iterations
                assert rel(d_s[i].cpu().numpy(), s_y.cpu().numpy()) < 1e-12
            else:
                assert rel(d_s[i].cpu().numpy(), ref64[i].cpu().numpy()) < 1e-5, i
        b.delete()
    # one FP64 solution through the oracle's apply (SolveEquation's system A chi = sqrt(Re sigma_b) E0)
    m, op, E0 = inst[2]
    sh, ah = op.get_ie_kernel_spectral()
    csiga = csiga_from_sigma(sig, m.freq)
    csigb, sqsigb = orc.background_cells(m)
    E = single64[2][1].cpu().numpy().reshape(E0.shape)
    a = 2.0 * sqsigb[:, None, None] / (csiga + np.conj(csigb)[:, None, None])
    rhs = sqsigb[None, :, None, None] * E0
    r = orc.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, E / a[None]) - rhs
    assert np.linalg.norm(r) / np.linalg.norm(rhs) < 1.5e-8
    for _, op in ops:
        op.delete()


@pytest.mark.parametrize("max_restart", [50, 2])
def test_batched_restarts_match_single(g2lib, max_restart):
    """Outer basis 3 and inner basis 2 force restart cycles (the host runs one outer step ahead inside a cycle
    and stops at its end); with max_restart = 2 the instances stop unconverged (status -1).  In FP64 every
    batched instance reproduces its single solve: status, iterations, misfit history and solution."""
    import torch
    ops, inst = _two_frequency_setup(g2lib)
    d_e = [torch.from_numpy(np.ascontiguousarray(e).ravel()).to("cuda") for _, e in inst]
    kw = dict(outer_buf=3, inner_buf=2, max_restart=max_restart)
    tol = 1e-10
    single = []
    for (op, _), x in zip(inst, d_e):
        y = torch.empty_like(x)
        single.append((op.solve_device(x.data_ptr(), y.data_ptr(), None, tol=tol, precision=0, **kw), y))
    b = g2lib.Batch([op for op, _ in inst], precision=0, **kw)
    d_s = [torch.empty_like(x) for x in d_e]
    infos = b.solve_device([x.data_ptr() for x in d_e], [y.data_ptr() for y in d_s], tol=tol)
    torch.cuda.synchronize()
    for i, (info1, y1) in enumerate(single):
        assert infos[i].stat == info1.stat
        assert infos[i].iterations == info1.iterations
        assert np.allclose(infos[i].misfits, info1.misfits, rtol=1e-10, atol=0)
        assert rel(d_s[i].cpu().numpy(), y1.cpu().numpy()) < 1e-12
        if max_restart == 2:
            assert infos[i].iterations <= 6                      # two cycles of three outer steps at most
            assert infos[i].stat == 1 or infos[i].iterations == 6
        else:
            assert infos[i].stat == 1
    if max_restart == 50:
        assert max(i.iterations for i in infos) > 3              # the batch went through a restart
    else:
        assert any(i.stat == -1 for i in infos)                   # and one instance stopped unconverged
    b.delete()
    for op in ops:
        op.delete()


@pytest.mark.parametrize("precision,tol", [(0, 1e-8), (1, 1e-6)])
def test_batch_of_two_grid_sizes(g2lib, precision, tol):
    """One batch holding operators of two grid sizes (16x16x8 and 32x32x8, both polarisations each): the
    instances of different vector lengths cannot share a Krylov launch, so the lockstep loop runs them through
    the single-instance forms next to the paired ones.  FP64 reproduces every single solve; mixed precision
    converges and stays within 1e-5 of the FP64 solution."""
    import torch
    from giem2g_b200.synthetic import config_grf
    ops, inst = [], []
    for n, seed in ((16, 11), (32, 12)):
        m, sig = config_grf(n, n, 8, seed=seed)
        op = g2lib.IEOperator.from_model(m)
        op.calc_ie_kernel(m.csigma, m.thick, m.omega)
        op.calc_fft_of_ie_kernel()
        op.set_anomaly_sigma(sig, m.freq)
        ops.append(op)
        for pol in (1, 0):
            inst.append((op, plane_wave_integral(m, pol)))
    d_e = [torch.from_numpy(np.ascontiguousarray(e).ravel()).to("cuda") for _, e in inst]
    single, ref64 = [], []
    for (op, _), x in zip(inst, d_e):
        y = torch.empty_like(x)
        single.append((op.solve_device(x.data_ptr(), y.data_ptr(), None, tol=tol, precision=precision), y))
        z = torch.empty_like(x)
        op.solve_device(x.data_ptr(), z.data_ptr(), None, tol=1e-10, precision=0)
        ref64.append(z)
    b = g2lib.Batch([op for op, _ in inst], precision=precision)
    d_s = [torch.empty_like(x) for x in d_e]
    infos = b.solve_device([x.data_ptr() for x in d_e], [y.data_ptr() for y in d_s], tol=tol)
    torch.cuda.synchronize()
    for i, (info1, y1) in enumerate(single):
        assert infos[i].stat == info1.stat == 1
        if precision == 0:
            assert infos[i].iterations == info1.iterations
            assert rel(d_s[i].cpu().numpy(), y1.cpu().numpy()) < 1e-12
        else:
            assert abs(infos[i].iterations - info1.iterations) <= 1
            assert rel(d_s[i].cpu().numpy(), ref64[i].cpu().numpy()) < 1e-5
    b.delete()
    for op in ops:
        op.delete()
