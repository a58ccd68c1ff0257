"""CPU checks of the port face tables the boundary assembly uploads
(opem_selftest_face_tables): the library's exact tangential mass tables and the
nodal-rule ones (the overlap integrals of ports driven by their own 2D modes)
equal the oracle's, and the nodal rule (MFEM's order-p L2 triangle) integrates
every polynomial of degree <= p exactly."""
import ctypes as C
from math import factorial

import numpy as np
import pytest

from openparem_b200 import _lib
from oracle.fem import basis, nodal_face_tables
from oracle.quadrature import l2_nodal_rule


def _lib_tables(p, nodal):
    ldf = p * (p + 2)
    out = np.zeros(4 * 3 * ldf * ldf)
    rc = _lib.lib().opem_selftest_face_tables(p, nodal, out.ctypes.data_as(C.POINTER(C.c_double)), out.size)
    assert rc == _lib.OK
    return out.reshape(4, 3, ldf, ldf)


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("nodal", [0, 1])
def test_face_tables_match_oracle(p, nodal):
    lib = _lib_tables(p, nodal)
    ora = nodal_face_tables(p) if nodal else basis(p)[4]
    for f in range(4):
        Fh = ora[f][1]   # (2, 2, ldf, ldf)
        ref = np.stack([Fh[0, 0], Fh[1, 1], Fh[0, 1] + Fh[1, 0]])
        assert np.abs(lib[f] - ref).max() <= 1e-11 * np.abs(ref).max(), (p, nodal, f)
    if p > 1 or nodal:
        # the rule is not exact for the degree-2p products: the tables differ
        assert np.abs(_lib_tables(p, 1) - _lib_tables(p, 0)).max() > 1e-8


@pytest.mark.parametrize("p", range(0, 9))
def test_nodal_rule_exact_to_degree_p(p):
    x, w = l2_nodal_rule(p)
    assert len(w) == (p + 1) * (p + 2) // 2
    assert np.all(x > 0) and np.all(x.sum(axis=1) < 1)   # open nodes: inside the triangle
    for a in range(p + 1):
        for b in range(p + 1 - a):
            exact = factorial(a) * factorial(b) / factorial(a + b + 2)
            assert abs(np.sum(w * x[:, 0] ** a * x[:, 1] ** b) - exact) <= 1e-13, (p, a, b)


def test_face_tables_reject_bad_arguments():
    out = np.zeros(10)
    assert _lib.lib().opem_selftest_face_tables(2, 1, out.ctypes.data_as(C.POINTER(C.c_double)), 10) == _lib.ERR_ARG
    assert _lib.lib().opem_selftest_face_tables(9, 0, out.ctypes.data_as(C.POINTER(C.c_double)), 10) == _lib.ERR_ARG
