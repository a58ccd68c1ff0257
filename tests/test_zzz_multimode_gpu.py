"""GPU: ports with several modes (opem_problem_add_port_mode) on the FP64 path:
the empty WR90 section at 16 GHz with TE10 and TE20 on each port solves on the
device to the oracle's 4 x 4 S (|dS| <= 1e-8, solver rtol 1e-12); mixed
precision declines such problems."""
import numpy as np
import pytest

from openparem_b200 import Fem3D, default_opts, _lib
from openparem_b200.fem3d import Context, OpemError
from test_multimode_cpu import two_mode_guide

pytestmark = pytest.mark.gpu


def test_two_mode_ports_match_oracle():
    from oracle import fem
    prob = two_mode_guide()
    F = Fem3D(prob, context=Context(0)).assemble()
    assert F.info()["nports"] == 4
    f = 16e9
    S, Zo, st = F.solve(f, default_opts(rtol=1e-12, restart=200, maxits=6000, h_rtol=1e-13))
    assert st["converged"] == 1
    ref = fem.solve_frequency(fem.Operators(prob), f)
    assert np.abs(S - ref["S"]).max() <= 1e-8, (S, ref["S"])
    assert np.abs(Zo - ref["Z"]).max() <= 1e-8 * np.abs(ref["Z"]).max()
    with pytest.raises(OpemError):
        F.solve(f, default_opts(precision=_lib.PREC_MIXED, rtol=1e-10))
