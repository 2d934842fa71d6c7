"""The GPU Green's tensor end to end at the benchmark's own size (128x128x32, 50x50x25 m cells, the anomaly
crossing the 500 m interface at cell 20, 0.1 Hz).

On some small test models the cross-layer xx/xy/yy entries of the GPU tensor differ from the oracle's by more
than the 1e-10 that every other entry meets (test_green_gpu.py explains why: the reference arithmetic divides
FFT round-off of the VBT weights at lambda < 1e-10 /m by lambda).  These tests measure that difference at this
model and what it does downstream: an
operator built from the ORACLE's spatial tensor (giem2g_set_ie_kernel_spatial) and one built from the GPU's
(giem2g_calc_ie_kernel) apply the same vector and solve both polarisations in FP64 at tol 1e-8.  At this
model the difference is round-off (2e-12 over the cross-layer entries): the apply agrees to 1e-12 and the
FP64 solutions to 1e-10, far below the mixed-precision field error (about 1e-6) the benchmark's method
accepts.  The measured figures are printed (pytest -s).
"""
import numpy as np
import pytest

from giem2g_b200.sources import plane_wave_integral
from giem2g_b200.synthetic import config_c2, csiga_from_sigma
from tests.helpers import random_vec, rel

pytestmark = pytest.mark.gpu

# Measured on a B200 (oracle on 16 host threads): cross-layer entries max |dG| / max|G| 9.9e-15 (xx, yy),
# 9.1e-17 (xy), 2-norm relative 2.0e-12 over those entries; FP64 apply 1.4e-13; FP64 solutions 4.2e-12 (EY)
# and 4.1e-12 (EX), 18 outer iterations each.  At this model the cross-layer entries meet the same 1e-10 as
# every other entry, and the bounds below sit one to two orders of magnitude above the measurement.
CROSS_BOUND = 1e-10   # 2-norm relative over the cross-layer entries of each of xx, xy, yy
APPLY_BOUND = 1e-12
FIELD_BOUND = 1e-10


@pytest.fixture(scope="module")
def two_ops(g2lib, orc):
    m, sig = config_c2(seed=2024)
    S_o, A_o = orc.green_tensor(m, nthreads=0)
    op_g = g2lib.IEOperator.from_model(m)
    op_g.calc_ie_kernel(m.csigma, m.thick, m.omega)
    S_g, A_g = op_g.get_ie_kernel_spatial()
    op_g.calc_fft_of_ie_kernel()
    op_g.set_anomaly_sigma(sig, m.freq)
    op_o = g2lib.IEOperator.from_model(m)
    op_o.set_background(m.csigma, m.thick, m.omega)
    op_o.set_ie_kernel_spatial(S_o, A_o)
    op_o.calc_fft_of_ie_kernel()
    op_o.set_anomaly_sigma(sig, m.freq)
    yield m, sig, op_g, op_o, (S_g, A_g), (S_o, A_o)
    op_g.delete()
    op_o.delete()


def test_c2_cross_layer_deviation(two_ops, orc):
    from tests.test_green_gpu import _cross_layer_mask
    m, sig, op_g, op_o, (S_g, A_g), (S_o, A_o) = two_ops
    cross = _cross_layer_mask(orc.layer_numbers(m), m.Nz)
    assert cross.any()
    worst = []
    for c, name in enumerate(("xx", "xy", "yy")):
        scale = np.abs(S_o[:, :, c]).max()
        dev = np.abs(S_g[:, :, c][..., cross] - S_o[:, :, c][..., cross]).max() / scale
        blk = rel(S_g[:, :, c][..., cross], S_o[:, :, c][..., cross])
        print(f"cross-layer {name}: max |dG| / max|G| = {dev:.3e}, 2-norm rel over the cross-layer entries {blk:.3e}")
        worst.append(blk)
    assert max(worst) < CROSS_BOUND


def test_c2_apply_with_gpu_tensor_vs_oracle_tensor(two_ops, orc):
    """The FP64 apply of the GPU-built operator against the oracle's apply of the oracle-built tensor."""
    m, sig, op_g, op_o, _, (S_o, A_o) = two_ops
    sh_o, ah_o = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, S_o, A_o)
    csiga = csiga_from_sigma(sig, m.freq)
    csigb, sqsigb = orc.background_cells(m)
    v = random_vec(m, 31)
    ref = orc.apply(m.Nx, m.Ny, m.Nz, sh_o, ah_o, csiga, csigb, sqsigb, m.dz, v)
    d_g = rel(op_g.apply_precond(v), ref)
    d_o = rel(op_o.apply_precond(v), ref)
    print(f"apply: GPU tensor vs oracle tensor {d_g:.3e}; oracle-tensor operator on the GPU {d_o:.3e}")
    assert d_o < 1e-12
    assert d_g < APPLY_BOUND


def test_c2_fp64_solutions_with_gpu_tensor_vs_oracle_tensor(two_ops):
    m, sig, op_g, op_o, _, _ = two_ops
    for pol in (1, 0):
        E0 = plane_wave_integral(m, pol)
        Eg, ig = op_g.solve_equation(E0, tol=1e-8, precision=0)
        Eo, io = op_o.solve_equation(E0, tol=1e-8, precision=0)
        assert ig.stat == io.stat == 1
        d = rel(Eg, Eo)
        print(f"pol {'EY' if pol else 'EX'}: ||E_gpu_tensor - E_oracle_tensor|| / ||E|| = {d:.3e} "
              f"(outer iterations {ig.iterations} / {io.iterations})")
        assert d < FIELD_BOUND
