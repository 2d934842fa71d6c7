"""Plane-wave source: the 1-D background (normal) field of the layered medium.

Restates PlaneWaveIntegral (sources_module.F90:67-101), the cell-averaged field that is the
right-hand side of the IE solve, and PlaneWave (:26-66), the field at receiver depths that the
receiver fields add to the anomalous part, both with the lambda = 0 layered recursion of Calc_APQ
(apq_module.F90:230-312).  The field is constant in x and y.  Host-side numpy: it is a handful of
complex numbers per layer and cell.
"""
from __future__ import annotations

import numpy as np

from .synthetic import MU0

EX, EY = 0, 1


def get_layer(m, z) -> int:
    """GetLayerSingle (data_types_module.F90:214-242): 0 at the surface, -1 in the air."""
    depth = np.r_[0.0, np.cumsum(m.thick)]  # depth[1..Nl-1]
    if abs(z) < 1e-15:
        return 0
    if z < 0:
        return -1
    if m.Nl == 1:
        return 1
    if z > depth[m.Nl - 1]:
        return m.Nl
    l = 1
    while z > depth[l]:
        l += 1
    return l


def _layer_numbers(m) -> np.ndarray:
    """Lnumber(0:Nz) (mpi_saveload_module.F90:99-100)."""
    L = np.zeros(m.Nz + 1, int)
    for i in range(1, m.Nz + 1):
        L[i] = get_layer(m, 0.5 * (m.z[i - 1] + m.z[i]))
    L[0] = get_layer(m, m.z[0] * (1.0 - 1e-7))
    return L


def _apq0(m):
    """Calc_APQ at lambda = 0 (apq_module.F90:230-312): eta, q, depth, A(l,1,1) and the surface factor t1
    of PlaneWave / PlaneWaveIntegral (sources_module.F90:36-42, :78-84)."""
    Nl = m.Nl
    cs = m.csigma
    k2 = 1j * cs * MU0 * m.omega
    thick = np.r_[0.0, m.thick]
    depth = np.r_[0.0, np.cumsum(m.thick)]
    eta = np.zeros(Nl + 1, complex)
    el = np.zeros(Nl + 1, complex)
    for i in range(1, Nl + 1):
        eta[i] = np.sqrt(0.0 - k2[i])
    for i in range(1, Nl):
        el[i] = np.exp(-2 * eta[i] * thick[i])
    p = np.zeros((Nl + 1, 2), complex)
    q = np.zeros((Nl + 1, 2), complex)
    ceta = np.sqrt(0.0 - k2[0]) / eta[1]
    p[1, 0] = (1 - ceta) / (1 + ceta)
    cg = cs[0] / cs[1]
    p[1, 1] = (cg - ceta) / (cg + ceta)
    for i in range(2, Nl + 1):
        w = el[i - 1] * p[i - 1]
        w = (w - 1) / (w + 1)
        a = np.array([eta[i - 1] / eta[i], eta[i - 1] / eta[i] * cs[i] / cs[i - 1]])
        w = w * a
        p[i] = (1 + w) / (1 - w)
    if Nl > 1:
        a = np.array([eta[Nl] / eta[Nl - 1], eta[Nl] / eta[Nl - 1] * cs[Nl - 1] / cs[Nl]])
        q[Nl - 1] = (1 - a) / (1 + a)
        for i in range(Nl - 2, 0, -1):
            w = el[i + 1] * q[i + 1]
            w = (w - 1) / (w + 1)
            a = np.array([eta[i + 1] / eta[i], eta[i + 1] / eta[i] * cs[i] / cs[i + 1]])
            w = w * a
            q[i] = (1 + w) / (1 - w)
    Arr = np.array([1 / eta[i] / (1 - p[i] * q[i] * el[i]) if i else [0, 0] for i in range(Nl + 1)], complex)
    # A(J, I, 1) chain (apq_module.F90:250-264), only column 1 / row 1 is used
    A11 = np.zeros(Nl + 1, complex)  # A(l, 1, 1) = A(1, l, 1)
    for i in range(1, Nl + 1):
        v = Arr[i, 0]
        for j in range(i - 1, 0, -1):
            tmp = depth[j] * (k2[j] - k2[j + 1]) / (eta[j + 1] + eta[j])
            v = v * (1 + p[j + 1, 0]) / (1 + p[j, 0] * el[j]) * np.exp(tmp)
        A11[i] = v
    t1 = 1 + q[1, 0] * np.exp(-depth[1] * eta[1] * 2) if Nl > 1 else 1.0 + 0j
    t1 = A11[1] * t1
    return eta, q, depth, A11, t1


def plane_wave_integral(m, pol: int) -> np.ndarray:
    """E0[3, Nz, Ny, Nx] (Fortran (Nx,Ny,Nz,3)); pol 0 = EX, 1 = EY."""
    Nl = m.Nl
    eta, q, depth, A11, t1 = _apq0(m)
    L = _layer_numbers(m)
    E0 = np.zeros((3, m.Nz, m.Ny, m.Nx), complex)
    for iz in range(1, m.Nz + 1):
        dz = m.z[iz] - m.z[iz - 1]
        l = L[iz]
        e1 = np.exp(-eta[l] * m.z[iz - 1])
        e2 = np.exp(-eta[l] * m.z[iz])
        if l < Nl:
            e3 = q[l, 0] * np.exp(-eta[l] * (2 * depth[l] - m.z[iz - 1]))
            e4 = q[l, 0] * np.exp(-eta[l] * (2 * depth[l] - m.z[iz]))
        else:
            e3 = e4 = 0.0
        G = (e1 - e2 + e4 - e3) * A11[l] / t1
        G = G / dz / eta[l]
        E0[pol, iz - 1] = G
    return E0


def plane_wave_points(m, pol: int, zrecv) -> np.ndarray:
    """PlaneWave (sources_module.F90:26-66): the normal field at receiver depths, F[Nr, 6] with columns
    Ex Ey Ez Hx Hy Hz; pol 0 = EX (Ex, Hy nonzero), 1 = EY (Ey, Hx nonzero)."""
    Nl = m.Nl
    eta, q, depth, A11, t1 = _apq0(m)
    iwm = 1j * MU0 * m.omega
    zr = np.atleast_1d(np.asarray(zrecv, dtype=np.float64))
    F = np.zeros((len(zr), 6), complex)
    for ir, z in enumerate(zr):
        l = max(get_layer(m, z), 1)
        t2 = A11[l] / t1
        e1 = np.exp(-eta[l] * z)
        e2 = q[l, 0] * np.exp(-eta[l] * (2.0 * depth[l] - z)) if l < Nl else 0.0
        g1 = t2 * (e1 + e2)
        g2 = -t2 * (e1 - e2) * eta[l] / iwm
        if pol == EX:
            F[ir, 0], F[ir, 4] = g1, g2
        else:
            F[ir, 1], F[ir, 3] = g1, -g2
    return F
