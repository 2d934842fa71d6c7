"""Receiver continuation on the GPU against the oracle.

Tolerances: the receiver tensor 1e-10 relative per component block on small grids and 1e-9 at Nz = 32
(the GPU sums the same lambda terms as the oracle in another order, through a GEMM); its spectrum 1e-12 against numpy's FFT of the GPU's
own spatial tensor; the fields at the receivers 1e-11 relative to the oracle's FFT route (the same
tensor, FP64 throughout).  At the 128x128x32 benchmark grid the tensor is checked at sampled lags
against the oracle and the fields at sampled receiver cells against direct lag sums over the GPU's
own spatial tensor.
"""
import numpy as np
import pytest

from giem2g_b200.synthetic import IEModel, THREE_LAYER_SIGMA, THREE_LAYER_THICK, config_grf, csiga_from_sigma
from tests.helpers import random_sigma, random_vec, rel, tiny_model

pytestmark = pytest.mark.gpu

RECEIVERS = {  # depth, x_shift, y_shift: surface, inside at a cell border, strictly inside (moved), below
    "depths": [0.0, 73.33333333333333, 100.0, 350.0, 600.0],
    "xs": [0.0, 20.0, -35.0, 0.0, 5.0],
    "ys": [0.0, -10.0, 0.0, 15.0, 5.0],
}


def _rc(g2, m, depths, xs, ys):
    rc = g2.RCOperator.from_model(m, depths, xs, ys)
    rc.calc_rc_kernel(m.csigma, m.thick, m.omega)
    return rc


def _per_block_rel(a, b):
    worst = 0.0
    for c in range(15):
        worst = max(worst, rel(a[..., c, :, :], b[..., c, :, :]))
    return worst


def test_receivers_prepared_like_oracle(g2lib, orc):
    m = tiny_model(4, 4, 4)
    rc = g2lib.RCOperator.from_model(m, RECEIVERS["depths"], RECEIVERS["xs"], RECEIVERS["ys"])
    z, rl, ac = rc.receivers()
    rv = orc.prepare_receivers(m, RECEIVERS["depths"], RECEIVERS["xs"], RECEIVERS["ys"])
    assert np.array_equal(z, rv.zrecv) and np.array_equal(rl, rv.recv_layer) and np.array_equal(ac, rv.anom_cell)
    rc.delete()


def _crossing_model():
    """Anomaly from 400 to 700 m, across the 500 m layer interface."""
    return IEModel(4, 4, 4, 60.0, 60.0, np.array([400.0, 450.0, 500.0, 600.0, 700.0]), THREE_LAYER_SIGMA.copy(),
                   THREE_LAYER_THICK.copy(), 2.0)


@pytest.mark.parametrize("shape", [(4, 4, 3), (8, 4, 5), (4, 8, 2), "crossing"])
def test_rc_tensor_matches_oracle(g2lib, orc, shape):
    m = _crossing_model() if shape == "crossing" else tiny_model(*shape)
    d, xs, ys = RECEIVERS["depths"], RECEIVERS["xs"], RECEIVERS["ys"]
    rc = _rc(g2lib, m, d, xs, ys)
    G = rc.get_kernel()
    rv = orc.prepare_receivers(m, d, xs, ys)
    Go = orc.rc_tensor(m, rv)
    assert _per_block_rel(G, Go) < 1e-10
    # spectrum: unnormalised forward 2-D DFT over the lag plane
    rc.calc_fft_of_rc_kernel()
    Gh = rc.get_kernel()
    assert rel(Gh, np.fft.fft2(G, axes=(0, 1))) < 1e-12
    rc.delete()


@pytest.mark.parametrize("shape", [(4, 4, 3), (8, 8, 4), (4, 4, 40)])
def test_rc_recalculate_matches_oracle(g2lib, orc, shape):
    import torch
    m = tiny_model(*shape, freq=3.0)
    d, xs, ys = RECEIVERS["depths"], RECEIVERS["xs"], RECEIVERS["ys"]
    rc = _rc(g2lib, m, d, xs, ys)
    G = rc.get_kernel()
    rc.calc_fft_of_rc_kernel()
    sig = random_sigma(m, 5)
    csiga = csiga_from_sigma(sig, m.freq)
    rc.set_anomaly_conductivity(csiga)
    E = random_vec(m, 13)
    Ea, Ha = rc.recalculate(E)
    csigb, _ = orc.background_cells(m)
    Eo, Ho = orc.rc_apply(m.Nx, m.Ny, m.Nz, G, csiga, csigb, E)
    assert rel(Ea, Eo) < 1e-11 and rel(Ha, Ho) < 1e-11
    # device entry point: same result
    dE = torch.from_numpy(np.ascontiguousarray(E).ravel()).to("cuda")
    dEa = torch.empty(Ea.size, dtype=torch.complex128, device="cuda")
    dHa = torch.empty_like(dEa)
    rc.recalculate_device(dE.data_ptr(), dEa.data_ptr(), dHa.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(dEa.cpu().numpy().reshape(Ea.shape), Ea)
    assert np.array_equal(dHa.cpu().numpy().reshape(Ha.shape), Ha)
    rc.delete()


def test_rc_zero_field_gives_zero(g2lib):
    m = tiny_model(4, 4, 3)
    rc = _rc(g2lib, m, [0.0], None, None)
    rc.calc_fft_of_rc_kernel()
    rc.set_anomaly_sigma(random_sigma(m, 2), m.freq)
    Ea, Ha = rc.recalculate(np.zeros((3, m.Nz, m.Ny, m.Nx), complex))
    assert not np.any(Ea) and not np.any(Ha)
    rc.delete()


def test_rc_errors_are_reported(g2lib):
    m = tiny_model(4, 4, 3)
    rc = g2lib.RCOperator.from_model(m, [0.0])
    with pytest.raises(g2lib.Giem2gError):
        rc.calc_fft_of_rc_kernel()  # no tensor yet
    with pytest.raises(g2lib.Giem2gError):
        rc.recalculate(np.zeros((3, m.Nz, m.Ny, m.Nx), complex))
    rc.delete()
    with pytest.raises(g2lib.Giem2gError):
        g2lib.RCOperator.from_model(tiny_model(6, 4, 3), [0.0])  # Nx not a power of two


def test_rc_full_grid_sampled(g2lib, orc):
    """128x128x32 (the benchmark grid) with two receivers: tensor at sampled lags against the oracle,
    fields at sampled cells against direct lag sums over the GPU's spatial tensor, and linearity."""
    m, sig = config_grf(128, 128, 32, seed=11)
    d, xs, ys = [0.0, m.z[-1] + 40.0], [0.0, 10.0], [0.0, -10.0]
    rc = _rc(g2lib, m, d, xs, ys)
    G = rc.get_kernel()  # [256, 256, 15, 2, 32]
    rv = orc.prepare_receivers(m, d, xs, ys)
    rng = np.random.default_rng(3)
    ix = np.r_[0, 1, 127, 129, 255, rng.integers(0, 256, 5)]
    iy = np.r_[0, 127, 1, 255, 129, rng.integers(0, 256, 5)]
    Go = orc.rc_tensor_lags(m, rv, ix, iy)
    assert _per_block_rel(G[iy, ix], Go) < 1e-9  # 501-term sums over 32 cells: more round-off than tiny grids
    rc.calc_fft_of_rc_kernel()
    csiga = csiga_from_sigma(sig, m.freq)
    rc.set_anomaly_conductivity(csiga)
    E1, E2 = random_vec(m, 1), random_vec(m, 2)
    Ea1, Ha1 = rc.recalculate(E1)
    Ea2, Ha2 = rc.recalculate(E2)
    Ea3, Ha3 = rc.recalculate(2.0 * E1 - 0.5j * E2)
    assert rel(Ea3, 2.0 * Ea1 - 0.5j * Ea2) < 1e-12 and rel(Ha3, 2.0 * Ha1 - 0.5j * Ha2) < 1e-12
    csigb, _ = orc.background_cells(m)
    j = (csiga - csigb[:, None, None])[None] * E1  # [3, Nz, Ny, Nx]
    Nx, Ny = m.Nx, m.Ny
    for (x, y) in [(0, 0), (127, 127), (64, 3), (5, 100)]:
        gi = G[(y - np.arange(Ny))[:, None] % (2 * Ny), (x - np.arange(Nx))[None, :] % (2 * Nx)]  # [Ny,Nx,15,Nr,Nz]
        jx, jy, jz = (np.transpose(j[c], (1, 2, 0))[:, :, None, :] for c in range(3))  # [Ny,Nx,1,Nz]

        def s(c, u):
            return np.sum(gi[:, :, c] * u, axis=(0, 1, 3))

        ex = s(0, jx) + s(1, jy) + s(2, jz)
        ez = s(5, jx) + s(6, jy) + s(7, jz)
        hy = s(11, jx) - s(8, jy) + s(12, jz)
        got = Ea1[y, x]
        assert rel(got[0], ex) < 1e-11 and rel(got[2], ez) < 1e-11
        assert rel(Ha1[y, x, 1], hy) < 1e-11
    rc.delete()
