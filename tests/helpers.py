"""Shared builders for the parity tests (the oracle is used only as the checker)."""
import numpy as np

from giem2g_b200.synthetic import IEModel, THREE_LAYER_SIGMA, THREE_LAYER_THICK, csiga_from_sigma


def tiny_model(Nx=4, Ny=4, Nz=3, freq=1.0):
    z = np.cumsum(np.r_[0.0, np.linspace(30.0, 70.0, Nz)])
    return IEModel(Nx, Ny, Nz, 100.0, 80.0, z, THREE_LAYER_SIGMA.copy(), THREE_LAYER_THICK.copy(), freq)


def random_sigma(m, seed=0, lo=-3.0, hi=0.0):
    rng = np.random.default_rng(seed)
    return 10.0 ** rng.uniform(lo, hi, size=(m.Ny, m.Nx, m.Nz))


def random_vec(m, seed=1):
    rng = np.random.default_rng(seed)
    shape = (3, m.Nz, m.Ny, m.Nx)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def random_spatial_tensor(m, seed=3, scale=1.0):
    rng = np.random.default_rng(seed)
    P = m.Nz * (m.Nz + 1) // 2
    s = (rng.standard_normal((m.Nx, m.Ny, 4, P)) + 1j * rng.standard_normal((m.Nx, m.Ny, 4, P))) * scale
    a = (rng.standard_normal((m.Nx, m.Ny, 2, m.Nz * m.Nz)) + 1j * rng.standard_normal((m.Nx, m.Ny, 2, m.Nz * m.Nz))) * scale
    # components odd in a direction vanish at lag 0 of that direction (xy: x and y, xz: x, yz: y),
    # as the physical tensor does (calc_ie_tensor_module.F90:328-350 zero those weights); the
    # spectral pairing of the reference relies on it
    s[0, :, 1] = 0
    s[:, 0, 1] = 0
    a[0, :, 0] = 0
    a[:, 0, 1] = 0
    return s, a


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
