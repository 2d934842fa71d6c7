"""Host logic of the tile-shape pin (giem2g_b200.autotune.pin_contraction), the bench's --variants option.

A fake operator stands in for the library: the pin only calls contract_variants, set_contract_variant
and set_fft_lines.
"""
import pytest

from giem2g_b200.autotune import pin_contraction


class FakeOp:
    def __init__(self, counts):
        self.counts = counts  # precision -> number of variants
        self.set = {}
        self.lines = None
        self.lines64 = None

    def contract_variants(self, prec):
        return self.counts[prec]

    def set_contract_variant(self, prec, v):
        self.set[prec] = v

    def set_fft_lines(self, lines, precision=None):
        if precision is None:
            self.lines = lines
            self.lines64 = lines
        else:
            self.lines64 = lines


def test_pin_sets_every_precision_and_the_fft_lines():
    op = FakeOp({0: 11, 1: 24, 2: 16})
    picks = pin_contraction(op, "5,21,14,8")
    assert op.set == {0: 5, 1: 21, 2: 14} and op.lines == 8
    assert picks["0"]["variant"] == 5 and picks["fft_lines"]["lines"] == 8
    assert all(p["pinned"] for p in picks.values())


def test_pin_without_fft_lines_leaves_them_alone():
    op = FakeOp({0: 2, 1: 4, 2: 4})
    pin_contraction(op, "1,3,0")
    assert op.set == {0: 1, 1: 3, 2: 0} and op.lines is None


def test_pin_skips_precisions_with_a_single_shape():
    op = FakeOp({0: 1, 1: 4, 2: 0})
    pin_contraction(op, "0,2,0")
    assert op.set == {1: 2}


def test_pin_second_fft_lines_value_is_complex128s():
    op = FakeOp({0: 11, 1: 24, 2: 16})
    picks = pin_contraction(op, "5,21,14,16,8")
    assert op.lines == 16 and op.lines64 == 8
    assert picks["fft_lines"]["lines"] == 16 and picks["fft_lines64"]["lines"] == 8


@pytest.mark.parametrize("spec", ["5,21", "1,2,3,4,5,6", "x,1,2"])
def test_pin_rejects_malformed_specs(spec):
    with pytest.raises(ValueError):
        pin_contraction(FakeOp({0: 11, 1: 24, 2: 16}), spec)


def test_pin_rejects_out_of_range_variants():
    with pytest.raises(ValueError):
        pin_contraction(FakeOp({0: 11, 1: 24, 2: 16}), "11,0,0")
