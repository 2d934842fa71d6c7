"""Model of the in-warp slice reduction of the barrier-free contraction (k_contract_wl, csrc/contract.cu).

Lane = zl + ZW*s (+ ZW*SL*vv when the vectors are split over lane groups) holds NR = 2*3*PTS partial sums (re, im of 3 components x PTS points) of row zl over
its j-slice s. log2(SL) halving steps follow: at step b a lane whose bit b of s is set keeps the upper
half of what it still holds and sends the lower half to lane ^ (ZW << b); the other lane does the
opposite. Each adds what it receives to what it keeps. Afterwards lane s holds HR = NR/SL reals starting
at flat index f0(s), and stores them as complex outputs k = (f0 + i) / 2 -> (component k / PTS,
point k % PTS).

The model replays exactly that data movement on random partial sums and checks three things:
* every output is the sum over the SL slices;
* every (component, point) output is stored by exactly one lane of the row;
* the stores cover all outputs.
"""
import numpy as np
import pytest


def _halve(vals, SL, ZW):
    """vals: [32, NR] per-lane partials. Returns per-lane (f0, kept values) after the halving steps."""
    NR = vals.shape[1]
    held = {lane: vals[lane].copy() for lane in range(32)}
    f0 = {lane: 0 for lane in range(32)}
    length, b = NR, 0
    while (1 << b) < SL:
        half = length // 2
        new = {}
        for lane in range(32):
            s = (lane // ZW) % SL
            up = (s >> b) & 1
            partner = lane ^ (ZW << b)
            mine = held[lane]
            theirs = held[partner]
            keep = mine[half:length] if up else mine[:half]
            # the partner sends the half this lane keeps
            recv = theirs[half:length] if up else theirs[:half]
            out = mine.copy()
            out[:half] = keep + recv
            new[lane] = out
            if up:
                f0[lane] += half
        held = new
        length = half
        b += 1
    return {lane: (f0[lane], held[lane][:length]) for lane in range(32)}


# (SL, NP, VS) of the shipped k_contract_wl shapes; VS > 1 splits the NP vectors over lane groups
# (lane = zl + ZW*(s + SL*vv), ZW = 32/(SL*VS)), and a lane of group vv holds the LanePts points of its vectors
SHAPES = [(1, 1, 1), (2, 1, 1), (4, 1, 1), (2, 2, 1), (4, 2, 1), (8, 2, 1), (2, 2, 2), (4, 2, 2)]


def _gp(p, vv, NP, VS):
    """LanePts<NP, VS>::gp: the lane's local point p -> global point slot*NP + vector."""
    npl = NP // VS
    return (p // npl) * NP + vv * npl + p % npl


@pytest.mark.parametrize("SL,NP,VS", SHAPES)
def test_halving_sums_every_output_once(SL, NP, VS):
    ZW = 32 // (SL * VS)
    PL = 4 * NP // VS
    NR = 2 * 3 * PL
    HR = NR // SL
    assert HR % 2 == 0  # whole complex outputs per lane (the kernel's static_assert)
    rng = np.random.default_rng(SL * 10 + NP + 100 * VS)
    vals = rng.standard_normal((32, NR))
    res = _halve(vals, SL, ZW)
    for zl in range(ZW):
        stored = {}
        for vv in range(VS):
            lanes = [zl + ZW * (s + SL * vv) for s in range(SL)]
            total = vals[lanes].sum(axis=0)  # the row's outputs (this lane group's points) over its slices
            for lane in lanes:
                f0, kept = res[lane]
                assert len(kept) == HR
                np.testing.assert_allclose(kept, total[f0:f0 + HR], rtol=1e-12, atol=1e-12)
                for i in range(0, HR, 2):
                    k = (f0 + i) >> 1
                    c, p = divmod(k, PL)
                    key = (c, _gp(p, vv, NP, VS))
                    assert key not in stored
                    stored[key] = (kept[i], kept[i + 1])
                    assert kept[i] == pytest.approx(total[2 * k]) and kept[i + 1] == pytest.approx(total[2 * k + 1])
        # every (component, global point) of the row is stored exactly once across the lane groups
        assert sorted(stored) == [(c, p) for c in range(3) for p in range(4 * NP)]


def test_slices_of_one_lane_group_read_consecutive_j():
    """Interleaved slices: at step jj the SL lanes of one row read j = jj*SL + s, SL consecutive
    spectrum entries; over all steps every j is read once per row."""
    for SL in (1, 2, 4, 8):
        NZ = 32
        seen = []
        for jj in range(NZ // SL):
            js = [jj * SL + s for s in range(SL)]
            assert js == list(range(js[0], js[0] + SL))
            seen += js
        assert sorted(seen) == list(range(NZ))
