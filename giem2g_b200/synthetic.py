"""Seeded synthetic models for the IE solve (no dataset is used).

The reference's own example conductivity file (test/128_128_501.dat) is not in
the checkout, so every workload here is generated: a layered background, an
anomaly grid, a conductivity field and frequencies.  Field order of the
conductivity returned by the generators is the reference's text-file order
(Nz, Nx, Ny) with z fastest, i.e. numpy shape [Ny, Nx, Nz]
(mpi_saveload_module.F90:113-146 reads it with a Fortran list READ).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

MU0 = 4.0 * np.pi * 1e-7                       # const_module.F90:32
EPS0 = 1.0 / (MU0 * 299792458.0 * 299792458.0)  # const_module.F90:33
AIR_CONDUCTIVITY = 1e-12                        # const_module.F90:35


@dataclass
class IEModel:
    """Background + anomaly geometry + frequency, the inputs of CalcIntegralGreenTensor."""
    Nx: int
    Ny: int
    Nz: int
    dx: float
    dy: float
    z: np.ndarray            # Nz+1 cell borders, metres, positive down
    sigma: np.ndarray        # Nl layer conductivities (last = half-space)
    thick: np.ndarray        # Nl-1 layer thicknesses
    freq: float
    displacement_currents: bool = True
    name: str = ""

    @property
    def Nl(self) -> int:
        return len(self.sigma)

    @property
    def omega(self) -> float:
        return self.freq * 2.0 * np.pi

    @property
    def csigma(self) -> np.ndarray:
        """Complex conductivity, index 0 = air (data_types_module.F90:244-259)."""
        w = self.omega
        cs = np.zeros(self.Nl + 1, np.complex128)
        if self.displacement_currents:
            cs[0] = AIR_CONDUCTIVITY - 1j * w * EPS0
            cs[1:] = self.sigma - 1j * w * EPS0
        else:
            cs[0] = 0.0
            cs[1:] = self.sigma
        return cs

    @property
    def dz(self) -> np.ndarray:
        return np.diff(self.z)

    def with_freq(self, freq: float) -> "IEModel":
        return IEModel(self.Nx, self.Ny, self.Nz, self.dx, self.dy, self.z, self.sigma, self.thick, freq,
                       self.displacement_currents, self.name)


def csiga_from_sigma(siga_file_order: np.ndarray, freq: float, displacement_currents: bool = True) -> np.ndarray:
    """SetAnomalySigma (ie_solver_module.F90:116-139): real sigma[Ny,Nx,Nz] -> complex csiga[Nz,Ny,Nx]."""
    w = freq * np.pi * 2.0
    c = np.transpose(siga_file_order, (2, 0, 1)).astype(np.complex128)
    if displacement_currents:
        c = c - 1j * w * EPS0
    return np.ascontiguousarray(c)


THREE_LAYER_SIGMA = np.array([0.01, 0.001, 0.1])   # 0-500 m, 500-2000 m, half-space
THREE_LAYER_THICK = np.array([500.0, 1500.0])


def gaussian_random_field(Nx, Ny, Nz, dx, dy, zc, corr_len, seed):
    """Zero-mean unit-variance field with covariance exp(-r^2/(2 l^2)) on physical coordinates.

    White noise is filtered in the Fourier domain on a grid padded by 2x in x/y
    and then standardised exactly.  z uses the cell centres `zc` (non-uniform
    spacing is handled by a dense Gaussian smoothing matrix along z).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    px, py = 2 * Nx, 2 * Ny
    noise = rng.standard_normal((Nz, py, px))
    kx = np.fft.fftfreq(px, d=dx) * 2 * np.pi
    ky = np.fft.fftfreq(py, d=dy) * 2 * np.pi
    filt = np.exp(-0.25 * corr_len ** 2 * (kx[None, :] ** 2 + ky[:, None] ** 2))  # sqrt of Gaussian spectrum
    f = np.fft.ifft2(np.fft.fft2(noise, axes=(1, 2)) * filt[None], axes=(1, 2)).real[:, :Ny, :Nx]
    dzm = zc[:, None] - zc[None, :]
    S = np.exp(-(dzm ** 2) / (corr_len ** 2))                                   # sqrt-kernel along z
    S /= np.sqrt((S ** 2).sum(axis=1, keepdims=True))
    f = np.tensordot(S, f, axes=(1, 0))
    f = (f - f.mean()) / f.std()
    return f  # [Nz, Ny, Nx]


def _to_file_order(a_zyx: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(np.transpose(a_zyx, (1, 2, 0)))  # [Ny, Nx, Nz]


def config_small_block():
    """32x32x8 cells of 100x100x50 m, 3-layer background, 8x8x4 block at 1 S/m in 0.01 S/m, 1 Hz."""
    Nx = Ny = 32
    Nz = 8
    z = np.arange(Nz + 1) * 50.0
    m = IEModel(Nx, Ny, Nz, 100.0, 100.0, z, THREE_LAYER_SIGMA.copy(), THREE_LAYER_THICK.copy(), 1.0,
                name="block32x32x8")
    sig = np.full((Nz, Ny, Nx), 0.01)
    sig[2:6, 12:20, 12:20] = 1.0
    return m, _to_file_order(sig)


def config_grf(Nx=128, Ny=128, Nz=32, dx=50.0, dy=50.0, dzc=25.0, freq=0.1, mean=-2.0, std=0.7,
               corr_len=400.0, seed=2024):
    """Lognormal conductivity (Gaussian-correlated log10 sigma) over the 3-layer background."""
    z = np.arange(Nz + 1) * dzc
    m = IEModel(Nx, Ny, Nz, dx, dy, z, THREE_LAYER_SIGMA.copy(), THREE_LAYER_THICK.copy(), freq,
                name=f"grf{Nx}x{Ny}x{Nz}")
    zc = 0.5 * (z[1:] + z[:-1])
    g = gaussian_random_field(Nx, Ny, Nz, dx, dy, zc, corr_len, seed)
    sig = 10.0 ** (mean + std * g)
    return m, _to_file_order(sig)


def config_c2(seed=2024):
    return config_grf(128, 128, 32, 50.0, 50.0, 25.0, 0.1, -2.0, 0.7, 400.0, seed)


def config_c4(seed=7, corr_len=None, freq=None):
    rng = np.random.Generator(np.random.PCG64(seed + 1000003))
    if corr_len is None:
        corr_len = float(rng.uniform(200.0, 800.0))
    if freq is None:
        freq = float(10 ** rng.uniform(-2.0, 1.0))
    return config_grf(64, 64, 16, 100.0, 100.0, 50.0, freq, -2.0, 0.8, corr_len, seed)


def config_c5(seed=5):
    m, sig = config_grf(256, 256, 48, 25.0, 25.0, 20.0, 0.01, -2.0, 1.0, 300.0, seed)
    rng = np.random.Generator(np.random.PCG64(seed + 77))
    Nx, Ny, Nz = 256, 256, 48
    x = (np.arange(Nx) + 0.5) * 25.0
    y = (np.arange(Ny) + 0.5) * 25.0
    zc = 0.5 * (m.z[1:] + m.z[:-1])
    s = np.transpose(sig, (2, 0, 1)).copy()
    for _ in range(3):
        cx, cy = rng.uniform(1000, 5400, size=2)
        cz = rng.uniform(200, 760)
        ax, ay = rng.uniform(150, 500, size=2)
        az = rng.uniform(60, 200)
        inside = (((x[None, None, :] - cx) / ax) ** 2 + ((y[None, :, None] - cy) / ay) ** 2
                  + ((zc[:, None, None] - cz) / az) ** 2) <= 1.0
        s[inside] = 1.0
    m.name = "grf256x256x48+ellipsoids"
    return m, _to_file_order(s)
