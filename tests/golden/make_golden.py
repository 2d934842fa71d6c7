"""Generate the small golden fixtures the tests pin against (run from the repository root):

    python tests/golden/make_golden.py

The reference ships no test vectors and cannot be built here, so these fixtures come from the
CPU oracle (oracle/), whose own correctness is pinned by tests/test_oracle.py (dense block-Toeplitz
brute force, independent numpy restatements, analytic plane wave).  They freeze the oracle's output
on an 8x8x4 model that crosses the 500 m layer interface so that later changes to either the oracle
or the GPU path are caught even without recomputing the oracle.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from giem2g_b200.synthetic import IEModel, THREE_LAYER_SIGMA, THREE_LAYER_THICK, csiga_from_sigma  # noqa: E402


def golden_model():
    z = 300.0 + np.arange(5) * 100.0          # 300..700 m: cells 1-2 in layer 1, 3-4 in layer 2
    m = IEModel(8, 8, 4, 120.0, 90.0, z, THREE_LAYER_SIGMA.copy(), THREE_LAYER_THICK.copy(), 2.0)
    rng = np.random.Generator(np.random.PCG64(12345))
    sig = 10.0 ** rng.uniform(-3.0, 0.0, size=(m.Ny, m.Nx, m.Nz))
    return m, sig


def main():
    m, sig = golden_model()
    S, A = oracle.green_tensor(m)
    sh, ah = oracle.tensor_spectrum(m.Nx, m.Ny, m.Nz, S, A)
    csiga = csiga_from_sigma(sig, m.freq)
    csigb, sqsigb = oracle.background_cells(m)
    rng = np.random.Generator(np.random.PCG64(777))
    v = rng.standard_normal((3, m.Nz, m.Ny, m.Nx)) + 1j * rng.standard_normal((3, m.Nz, m.Ny, m.Nx))
    Av = oracle.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, v)
    E0 = oracle.plane_wave(m, 1)
    Es, info, hist = oracle.solve(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, E0, None, 30, 10, 100, 1e-10)
    np.savez_compressed(os.path.join(HERE, "golden_8x8x4.npz"), sigma=sig, symm=S, asym=A, symm_hat=sh,
                        asym_hat=ah, v=v, Av=Av, E0=E0, Esol=Es, misfits=hist,
                        info=np.array([info.iterations, info.stat, info.applies]), be=np.array([info.be]))
    print("wrote golden_8x8x4.npz", info.iterations, info.stat)


if __name__ == "__main__":
    main()
