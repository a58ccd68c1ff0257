"""GPU: the reference's adaptive loop (fem3d.adaptive_solve) with the device
step (assembly, solve, ZZ indicator and marking on the device; refinement on the
host)."""
import numpy as np
import pytest

from openparem_b200 import meshgen, default_opts
from openparem_b200.fem3d import Context

pytestmark = pytest.mark.gpu

TIGHT = dict(rtol=1e-12, restart=200, maxits=6000, h_rtol=1e-13)


@pytest.fixture(scope="module")
def ctx():
    return Context(0)


def test_adaptive_loop_on_the_device(ctx):
    """The reference's adaptive loop (fem3d.adaptive_solve) with the device
    step: assembly, solve, ZZ indicator and marking on the device, refinement on
    the host.  WR90 straight, ND2, 10 GHz, three passes marking 10 % of the
    elements (the cut between marked and unmarked errors is 1e-4 relative or
    more, far above the device-oracle indicator difference): the first pass
    equals the oracle's solve of the starting mesh, every pass refines, and the
    phase error of S21 against the exact -beta L falls, as in the oracle-step
    loop on CPU (0.40, 0.30, 0.28 deg)."""
    from oracle import fem
    from openparem_b200.fem3d import adaptive_solve, device_step
    prob = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 50e-3, 6, 3, 15, 2)
    f = 10e9
    S, pf, hist = adaptive_solve(prob, device_step(f, 0.1, default_opts(**TIGHT), ctx), variable="S", rel_tol=1e-12,
                                 iter_max=3)
    assert [h["iteration"] for h in hist] == [1, 2, 3]
    assert hist[2]["tets"] > hist[1]["tets"] > hist[0]["tets"]
    assert hist[1]["relative_error"] > 0 and hist[2]["relative_error"] > 0
    ref = fem.solve_frequency(fem.Operators(prob), f)["S"]
    assert np.abs(hist[0]["S"] - ref).max() <= 1e-8
    k0 = 2 * np.pi * f / 299792458.0
    exact = np.angle(np.exp(-1j * np.sqrt(k0 ** 2 - (np.pi / meshgen.WR_A) ** 2) * 50e-3), deg=True)
    errs = [abs(np.angle(h["S"][1, 0], deg=True) - exact) for h in hist]
    assert errs[2] < errs[0]
