"""CPU test of the Hessenberg least squares the solvers run on the device
(lsq.cu): the same column update and back substitution, compiled for the host
(opem_selftest_lsq), equal the host Givens QR of dense.cpp on seeded problems,
fresh cycles and cycles started from a deflated restart block."""
import ctypes as C

import pytest

from openparem_b200 import _lib


@pytest.mark.parametrize("m,kd,seed", [(12, 4, 1), (30, 0, 2), (100, 30, 3), (60, 20, 4)])
def test_device_least_squares_equals_host_givens(m, kd, seed):
    d = C.c_double(1.0)
    rc = _lib.lib().opem_selftest_lsq(m, kd, seed, C.byref(d))
    assert rc == _lib.OK
    assert d.value < 1e-11, d.value


def test_bad_sizes():
    d = C.c_double(0.0)
    assert _lib.lib().opem_selftest_lsq(1, 0, 1, C.byref(d)) == _lib.ERR_ARG
    assert _lib.lib().opem_selftest_lsq(10, 9, 1, C.byref(d)) == _lib.ERR_ARG
