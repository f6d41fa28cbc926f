"""The box means of the local intensity scale divide by their window length
with a corrected reciprocal product; it must give the IEEE quotient's bits
for every float input (all 2^32, on the GPU) and every window the kernels
instantiate (half-widths 1..6)."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("d", [3.0, 5.0, 7.0, 9.0, 11.0, 13.0])
def test_division_by_window_length_matches_ieee(d):
    from libapr_b200._lib import check, lib

    n, first = C.c_uint64(), C.c_uint32()
    check(lib().aprb_check_division_by_constant(d, C.byref(n), C.byref(first)))
    assert n.value == 0, "first differing input bits 0x%08x" % first.value
