"""GPU parity: the CUDA solve stage (through the C ABI) against the FP64 oracle.

Tolerances
  assembled operators / system matrix: 1e-12 relative to the operator's max entry
  S-parameters:                        |dS| <= 1e-8 with solver rtol 1e-12
  fields:                              1e-7 relative (E) / 1e-6 (H, CG to 1e-12)
"""
import numpy as np
import pytest

from openparem_b200 import meshgen, Fem3D, default_opts, OpemError
from openparem_b200 import _lib

pytestmark = pytest.mark.gpu

TIGHT = dict(rtol=1e-12, restart=200, maxits=6000, h_rtol=1e-13)


def _oracle():
    from oracle import fem
    return fem


CASES = {
    "c1_nd1": lambda: meshgen.config1()[0],
    "slab_nd2": lambda: meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 20e-3, 3, 2, 6, 2,
                                                  slab=(5e-3, 12e-3, 4.4, 0.02)),
    "slab_nd3": lambda: meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 20e-3, 3, 2, 4, 3,
                                                  slab=(5e-3, 12e-3, 2.2, 0.001)),
    "copper_nd2": lambda: meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 20e-3, 3, 2, 5, 2, wall="impedance",
                                                    wall_sigma=5.8e7, wall_Rz=0.5e-6),
    "radcap_nd1": lambda: meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 20e-3, 4, 2, 8, 1, ports=("zmin",),
                                                    radiation_cap=5e-3, cap_nz=2),
    "perelem_nd2": lambda: meshgen.waveguide_problem(
        meshgen.WR_A, meshgen.WR_B, 15e-3, 2, 2, 4, 2,
        per_element_eps=np.random.default_rng(3).lognormal(np.log(3.0), 0.1, size=2 * 2 * 4 * 6)),
}


@pytest.fixture(scope="module")
def ctx():
    from openparem_b200.fem3d import Context
    return Context(0)


@pytest.mark.parametrize("case", list(CASES))
def test_operators_match_oracle(ctx, case):
    fem = _oracle()
    prob = CASES[case]()
    F = Fem3D(prob, context=ctx).assemble()
    ops = fem.Operators(prob)
    for name, ref in [("K", ops.K), ("M_eps", ops.M_eps), ("M1", ops.M1), ("Q_mu", ops.Q_mu),
                      ("M_tand", ops.M_tand)]:
        G = F.operator(name)
        scale = max(abs(ref).max(), 1e-300)
        assert abs(G - ref).max() <= 1e-12 * scale, name
    for f in (8e9, 11.5e9):
        for d in range(F.nports):
            A = F.system_matrix(f, d)
            Aref = fem.assemble_A(ops, f, d)
            assert abs(A - Aref).max() <= 1e-12 * abs(Aref).max()


@pytest.mark.parametrize("case", list(CASES))
def test_s_parameters_match_oracle(ctx, case):
    fem = _oracle()
    prob = CASES[case]()
    F = Fem3D(prob, context=ctx).assemble()
    ops = fem.Operators(prob)
    for f in (9e9, 10.3e9):
        S, Z, st = F.solve(f, default_opts(**TIGHT))
        ref = fem.solve_frequency(ops, f)
        assert st["converged"] == 1
        assert np.abs(S - ref["S"]).max() <= 1e-8, (case, f, S, ref["S"])
        assert np.allclose(Z, ref["Z"], rtol=1e-12)


def test_fields_match_oracle(ctx):
    fem = _oracle()
    prob = CASES["slab_nd2"]()
    F = Fem3D(prob, context=ctx).assemble()
    ops = fem.Operators(prob)
    f = 9.7e9
    F.solve(f, default_opts(**TIGHT))
    ref = fem.solve_frequency(ops, f, return_fields=True)
    for d in range(2):
        e, h = F.fields(d)
        er, hr = ref["fields"][d]
        assert np.linalg.norm(e - er) <= 1e-7 * np.linalg.norm(er)
        assert np.linalg.norm(h - hr) <= 1e-6 * np.linalg.norm(hr)


def test_deterministic(ctx):
    prob = CASES["slab_nd2"]()
    F = Fem3D(prob, context=ctx).assemble()
    S1, _, _ = F.solve(10e9)
    S2, _, _ = F.solve(10e9)
    assert np.array_equal(S1, S2)
    G = Fem3D(prob, context=ctx).assemble()
    assert np.array_equal(F.operator("K").data, G.operator("K").data)


def test_sweep_equals_single(ctx):
    prob = CASES["c1_nd1"]()
    F = Fem3D(prob, context=ctx).assemble()
    fr = np.array([8.5e9, 10e9, 11.5e9])
    Ssw, st = F.sweep(fr)
    for i, f in enumerate(fr):
        S, _, _ = F.solve(f)
        assert np.abs(S - Ssw[i]).max() <= 1e-12


def test_wr90_mesh_nd3_against_oracle(ctx):
    """The reference's WR90 regression mesh at ND3 (the largest GPU order)."""
    fem = _oracle()
    from tests.test_oracle_golden import wr90_problem
    prob = wr90_problem(3)
    F = Fem3D(prob, context=ctx).assemble()
    S, _, st = F.solve(9e9, default_opts(**TIGHT))
    ref = fem.solve_frequency(fem.Operators(prob), 9e9)["S"]
    assert np.abs(S - ref).max() <= 1e-8


def test_not_converged_is_reported(ctx):
    prob = CASES["slab_nd2"]()
    F = Fem3D(prob, context=ctx).assemble()
    with pytest.raises(OpemError) as ei:
        F.solve(10e9, default_opts(maxits=2, restart=2))
    assert ei.value.code == _lib.ERR_NOT_CONVERGED
    S, _, st = F.solve(10e9, default_opts(maxits=2, restart=2), allow_not_converged=True)
    assert st["converged"] == 0 and st["iterations"] <= 4


def test_errors_are_status_codes(ctx):
    prob = CASES["c1_nd1"]()
    F = Fem3D(prob, context=ctx)
    with pytest.raises(OpemError) as ei:
        F.solve(10e9)
    assert ei.value.code == _lib.ERR_STATE
    bad = dict(prob)
    bad["order"] = 4
    with pytest.raises(OpemError) as ei:
        Fem3D(bad, context=ctx)
    assert ei.value.code == _lib.ERR_UNSUPPORTED
    bad = dict(prob)
    tris = np.array(prob["bdr_tris"]).copy()
    tris[0] = [0, 1, int(np.max(prob["tets"]))]
    bad["bdr_tris"] = tris
    with pytest.raises(OpemError) as ei:
        Fem3D(bad, context=ctx)
    assert ei.value.code == _lib.ERR_MESH


def test_deflated_restart_cuts_iterations(ctx):
    """GMRES-DR(m, k) vs plain GMRES(m): same S, fewer iterations on a mesh
    where plain restarting stagnates."""
    prob = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 50e-3, 8, 4, 20, 2, slab=(20e-3, 30e-3, 4.4, 0.02))
    F = Fem3D(prob, context=ctx).assemble()
    S0, _, st0 = F.solve(10e9, default_opts(restart=60, deflate=0, maxits=20000))
    S1, _, st1 = F.solve(10e9, default_opts(restart=60, deflate=20, maxits=20000))
    assert st0["converged"] == 1 and st1["converged"] == 1
    assert np.abs(S0 - S1).max() <= 1e-7
    assert st1["iterations"] < st0["iterations"]


@pytest.mark.parametrize("case", ["c1_nd1", "slab_nd2", "copper_nd2", "radcap_nd1", "slab_nd3", "perelem_nd2"])
def test_mixed_sweep_matches_fp64_and_oracle(ctx, case):
    """Batched FP32-inner / FP64-refinement sweep vs the FP64 solve and the oracle:
    |dS| <= 1e-6 with outer rtol 1e-10."""
    fem = _oracle()
    prob = CASES[case]()
    F = Fem3D(prob, context=ctx).assemble()
    fr = np.linspace(8.5e9, 11.5e9, 5)[[3, 0, 4, 1, 2]]   # unsorted: results come back in caller order
    Sm, st = F.sweep(fr, default_opts(precision=_lib.PREC_MIXED, rtol=1e-10))
    ops = fem.Operators(prob)
    for i, f in enumerate(fr):
        S, _, _ = F.solve(f, default_opts(rtol=1e-12, restart=200))
        assert st[i]["converged"] == 1 and st[i]["rnorm"] <= 1e-10
        assert np.abs(Sm[i] - S).max() <= 1e-6, (case, f)
        assert np.abs(Sm[i] - fem.solve_frequency(ops, f)["S"]).max() <= 1e-6


def test_mixed_single_frequency_entry(ctx):
    prob = CASES["slab_nd2"]()
    F = Fem3D(prob, context=ctx).assemble()
    S1, Z1, st1 = F.solve(9.9e9, default_opts(precision=_lib.PREC_MIXED))
    S0, Z0, _ = F.solve(9.9e9)
    assert np.abs(S1 - S0).max() <= 1e-6 and np.allclose(Z1, Z0)
    assert st1["outer"] >= 1


def test_mesh_error_indicator_matches_oracle(ctx):
    """ZZ error indicator and marking (opem_mesh_errors) on the device against
    oracle/estimate.py applied to the device's own H fields (ND2, lossy slab):
    errors to 1e-7 of the largest, the same marked set."""
    from oracle import fem
    from oracle.estimate import mesh_errors
    prob = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 50e-3, 6, 3, 15, 2, slab=(20e-3, 30e-3, 4.4, 0.02))
    F = Fem3D(prob, context=ctx).assemble()
    S, _, st = F.solve(10e9, default_opts(**TIGHT))
    assert st["converged"] == 1
    err, marked, mx = F.mesh_errors(0.05)
    hs = [F.fields(d)[1] for d in range(2)]
    ref, mref, mxref = mesh_errors(fem.Operators(prob), hs, 0.05)
    assert np.abs(err - ref).max() <= 1e-7 * ref.max()
    assert len(marked) == len(mref) == 81 and abs(mx - mxref) <= 1e-7 * mxref
    assert np.allclose(np.sort(ref[marked]), np.sort(ref[mref]), rtol=1e-6, atol=0)

