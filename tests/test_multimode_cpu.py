"""Ports with several modes (the reference's ports with several Mode blocks),
oracle side: an empty WR90 section at 16 GHz, where TE10 and TE20 propagate,
with both ports driven by their own 2D modes and TE20 added as a second mode
on each.  S-ports: 1, 2 the ports' TE10, 3, 4 their TE20.  Each mode crosses
the section on its own S-port pair, the modes do not convert into each other,
and the 4 x 4 S is passive; a port absorbs with the gamma of its largest-|gamma|
mode when the other drives (Port::addPortIntegrators, port.cpp:5790-5806).
On this coarse ND2 mesh the largest singular value of S is 1.00044."""
import numpy as np

from openparem_b200 import meshgen
from oracle import fem


def two_mode_guide(order=2):
    a, b = meshgen.WR_A, meshgen.WR_B
    prob = meshgen.waveguide_problem(a, b, 30e-3, 6, 3, 6, order)
    for p in prob["ports"]:
        m = p["mode"]
        o, u, v = (np.asarray(m[k], float) for k in ("origin", "u", "v"))
        p0 = o + 0.25 * a * u          # TE20's field is largest a quarter across
        m.update(kind="FEM2D", nsub=1, order2d=order,
                 extra_modes=[{"index": 1, "vpath": (p0.tolist(), (p0 + b * v).tolist())}])
    return prob


def test_two_mode_ports_oracle():
    prob = two_mode_guide()
    assert fem.sports(prob) == [(0, None), (1, None), (0, prob["ports"][0]["mode"]["extra_modes"][0]),
                                (1, prob["ports"][1]["mode"]["extra_modes"][0])]
    ops = fem.Operators(prob)
    f = 16e9
    r = fem.solve_frequency(ops, f)
    S = r["S"]
    assert S.shape == (4, 4)
    assert abs(S[1, 0]) > 0.99 and abs(S[3, 2]) > 0.99           # each mode crosses on its own pair
    assert np.abs(S[2:, :2]).max() < 0.02                          # no conversion (mesh asymmetry only)
    assert np.linalg.svd(S, compute_uv=False).max() < 1 + 1e-3     # passive to the discretisation (4.4e-4)
    k0 = 2 * np.pi * f / 299792458.0
    for s, kc in ((0, np.pi / meshgen.WR_A), (2, 2 * np.pi / meshgen.WR_A)):
        beta = np.sqrt(k0 ** 2 - kc ** 2)
        assert abs(fem.sport_mode(ops, s, f)["gamma"].imag / beta - 1) < 1e-3
    # the absorbing condition takes TE10's gamma, the larger
    assert fem.robin_gamma(ops, 0, f) == fem.sport_mode(ops, 0, f)["gamma"]
    assert abs(fem.sport_mode(ops, 2, f)["gamma"]) < abs(fem.robin_gamma(ops, 0, f))
