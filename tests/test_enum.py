"""Error-pattern order tables (sg_enum.h, built by the library) against the oracle's own
restatement of the reference loops."""
import ctypes as C

import numpy as np
import pytest

from oracle_api import Oracle


def lib_order(sg, ic):
    from sogrand_b200 import _lib

    out = np.zeros(65536, np.uint32)
    n = _lib.load().sg_pattern_order(ic, out.ctypes.data, out.size)
    return out[:n]


@pytest.fixture(scope="module")
def oracle(oracle_paths):
    return Oracle(oracle_paths["libm"])


@pytest.mark.parametrize("ic", [0, 1, 2, 3, 5, 8, 13, 21, 34, 55, 56])
def test_table_equals_oracle_order(sg, oracle, ic):
    a = lib_order(sg, ic)
    b = np.zeros(65536, np.uint32)
    n = oracle.lib.sgo_pattern_order(ic, b, b.size)
    assert n == 65536 and len(a) == 65536
    assert np.array_equal(a, b)


@pytest.mark.parametrize("ic", [0, 4, 30, 56])
def test_table_is_a_permutation(sg, ic):
    a = lib_order(sg, ic) & 0xFFFF
    assert len(np.unique(a)) == 65536
    assert a[0] == 0  # the hard decision first
    assert a[-1] == 0xFFFF  # all ones last


def test_canonical_order_for_large_ic(sg):
    base = lib_order(sg, 56)
    for ic in [57, 64, 100, 333, 1000, 4096, 100000]:
        assert np.array_equal(lib_order(sg, ic), base), ic
    assert not np.array_equal(lib_order(sg, 55), base)


def test_group_starts_follow_logistic_weight(sg):
    # for IC = 0 the first weights hold exactly one pattern each:
    # wt 1 = {pos0}, wt 2 = {pos1}, wt 3 = {pos2, pos0+pos1}
    a = lib_order(sg, 0)
    gs = (a >> 16) & 1
    assert list(a[1:5] & 0xFFFF) == [0b1, 0b10, 0b100, 0b11]
    assert list(gs[1:5]) == [1, 1, 1, 0]
