"""Full-size workloads checked through size-independent properties (the oracle's
direct solve does not fit in seconds at these sizes).

config 3: 40x20x100 hex (480k tets), ND2 (3,108,320 DOF), copper impedance walls with
0.5 um roughness, per-element eps_r ~ lognormal(ln 3, 0.1).  At one frequency:
  * the FP64 solve and the batched mixed solve converge and agree to |dS| <= 1e-6;
  * without forced reciprocity the FP64 S is reciprocal to 1e-4 (|S12 - S21|; the
    discrete S extraction is reciprocal only up to discretisation error, 2.4e-5 here,
    which is why the reference forces it);
  * the lossy guide is passive: every column of S has sum_i |S_ij|^2 <= 1 + 1e-9.
"""
import numpy as np
import pytest

from openparem_b200 import meshgen, Fem3D, default_opts
from openparem_b200 import _lib

pytestmark = pytest.mark.gpu


def test_config3_fullsize_properties():
    prob, freqs = meshgen.config3(nfreq=101)
    F = Fem3D(prob, device=0).assemble()
    assert F.info()["ndofs"] == 3108320
    f = float(freqs[50])   # 10 GHz
    S, _, st = F.solve(f, default_opts(rtol=1e-10, force_reciprocal=0))
    assert st["converged"] == 1
    assert abs(S[0, 1] - S[1, 0]) <= 1e-4
    assert np.all((np.abs(S) ** 2).sum(axis=0) <= 1 + 1e-9)
    Sm, stm = F.sweep([f], default_opts(rtol=1e-10, force_reciprocal=0, precision=_lib.PREC_MIXED, poly_degree=16))
    assert stm[0]["converged"] == 1
    assert np.abs(Sm[0] - S).max() <= 1e-6
