"""The reference's regression comparator and results CSV (CPU).

opem_evaluate_test_cases restates process3D (process3D.cpp:105-560).  It is
pinned to the reference itself: for five of its WR90 regression projects
(tests/golden/wr90_regression.json, made by tests/golden/make_wr90_fixture.py)
the reference's own found values are written into a results CSV, the
project's *_test_cases.csv is evaluated against it, and every output line
(status, found value, error, threshold) and the order of the lines equal the
block the reference wrote to regression_results.csv.current.
"""
import json
import os

import numpy as np
import pytest

from openparem_b200.fem3d import evaluate_test_cases, write_results_csv, OpemError

HERE = os.path.dirname(os.path.abspath(__file__))


def _regression():
    with open(os.path.join(HERE, "golden", "wr90_regression.json")) as f:
        return json.load(f)["projects"]


def _found_csv(path, rows):
    """A results CSV (DB format, Hz) holding the reference's found values of the
    evaluation rows: magS(dB) and argS(deg) per (frequency, portOut, portIn)."""
    vals, freqs, nports = {}, [], 1
    for r in rows:
        f, po, pi, var, fn = r[2], int(r[3]), int(r[4]), r[5], r[6]
        found = r[8] if fn == "equal" else r[7]
        nports = max(nports, po, pi)
        if f not in freqs:
            freqs.append(f)
        vals[(f, po, pi, var)] = found
    lines = ["#Touchstone format,DB", "#frequency unit,Hz", f"#number of frequencies,{len(freqs)}",
             f"#number of ports,{nports}"]
    for f in freqs:
        fields = [f]
        for col in range(1, nports + 1):          # driven port outer, as the header orders S(row;col)
            for row in range(1, nports + 1):
                fields.append(vals.get((f, row, col, "magS(dB)"), "0"))
                fields.append(vals.get((f, row, col, "argS(deg)"), "0"))
        lines.append(",".join(fields))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


@pytest.mark.parametrize("project", ["straight", "straight-lossy", "straight-loaded", "shorted", "opened"])
def test_comparator_reproduces_reference_evaluation(tmp_path, project):
    rec = _regression()[project]
    tc = tmp_path / "cases.csv"
    with open(tc, "w") as fh:
        fh.write("# ResultDatabase::save_as_test\n" + "\n".join(",".join(r) for r in rec["test_cases"]) + "\n")
    res = tmp_path / "results.csv"
    _found_csv(res, rec["evaluation"])
    out = tmp_path / "test_results.csv"
    n, npass = evaluate_test_cases(tc, res, out)
    lines = open(out).read().splitlines()
    assert lines[0].startswith("# name,status,frequency")
    expected = [",".join(r) + "," for r in rec["evaluation"]]
    assert n == len(expected) and npass == sum(r[1] == "pass" for r in rec["evaluation"])
    assert lines[1:] == expected


def test_results_csv_round_trip_and_failures(tmp_path):
    """Results written by opem_write_results_csv (RI and DB) evaluate like the
    values they hold; a case outside its tolerance fails."""
    fr = np.array([9e9, 10e9])
    S = np.zeros((2, 2, 2), dtype=complex)
    S[:, 1, 0] = np.exp(1j * np.deg2rad([-20.75, 172.88])) * 0.999
    S[:, 0, 1] = S[:, 1, 0]
    S[:, 0, 0] = S[:, 1, 1] = 1e-6
    tc = tmp_path / "cases.csv"
    with open(tc, "w") as fh:
        fh.write("# ResultDatabase::save_as_test\n"
                 "a,9000000000,argS(deg),2,1,equal,-20.75,1e-9\n"
                 "b,10000000000,argS(deg),1,2,equal,172.9,1e-9   // off by 0.02 deg\n"
                 "c,9000000000,magS(dB),1,1,lessthan,-110\n"
                 "d,10000000000,magS(dB),2,1,greaterthan,-0.01\n")
    for fmt in ("RI", "DB", "MA"):
        res = tmp_path / f"r_{fmt}.csv"
        write_results_csv(res, fr, S, 50.0, fmt, "GHz")
        out = tmp_path / f"o_{fmt}.csv"
        n, npass = evaluate_test_cases(tc, res, out)
        assert (n, npass) == (4, 3)
        rows = {ln.split(",")[0]: ln.split(",") for ln in open(out).read().splitlines()[1:]}
        assert rows["b"][1] == "FAIL" and rows["a"][1] == "pass"
        assert abs(float(rows["c"][7]) - (-120.0)) < 1e-9
    bad = tmp_path / "bad.csv"
    with open(bad, "w") as fh:
        fh.write("x,9e9,argS(deg),2,1,equal,1\n")     # equal without a tolerance
    with pytest.raises(OpemError):
        evaluate_test_cases(bad, tmp_path / "r_DB.csv", tmp_path / "o.csv")


def test_regression_flow_on_the_mu_r_2_guide(tmp_path):
    """The reference's regression flow end to end on its permeability/
    rectangular_waveguide project (mu_r = 2, ND6, no recorded run): the project
    read by the C++ reader, solved by the oracle, written by
    opem_write_results_csv and judged by opem_evaluate_test_cases against the
    project's own test cases (those of its first frequency): all pass."""
    from project_files import reference_project
    from openparem_b200.fem3d import project_problem
    from oracle import fem
    proj, rec = reference_project(str(tmp_path), "permeability-straight")
    prob, fr = project_problem(proj)
    assert np.allclose(prob["mu_r"], [2.0])
    f0 = fr[0]
    S = fem.solve_frequency(fem.Operators(prob), f0)["S"]
    res = tmp_path / "straight_results.csv"
    write_results_csv(res, [f0], S[None], 0.0, "DB", "GHz")
    cases = [r for r in _regression()["permeability-straight"]["test_cases"] if float(r[1]) == f0]
    tc = tmp_path / "cases.csv"
    with open(tc, "w") as fh:
        fh.write("# ResultDatabase::save_as_test\n" + "\n".join(",".join(r) for r in cases) + "\n")
    n, npass = evaluate_test_cases(tc, res, tmp_path / "out.csv")
    assert n == len(cases) == 8 and npass == n


def test_comparator_rejects_antenna_cases_and_missing_files(tmp_path):
    from openparem_b200 import _lib
    tc = tmp_path / "ant.csv"
    with open(tc, "w") as fh:
        fh.write("# PatternDatabase::save_as_test\ng,9e9,gain,1,equal,5,0.1\n")
    res = tmp_path / "r.csv"
    write_results_csv(res, [9e9], np.eye(1)[None].astype(complex) * 0.5, 50.0)
    with pytest.raises(OpemError) as e:
        evaluate_test_cases(tc, res, tmp_path / "o.csv")
    assert e.value.code == _lib.ERR_UNSUPPORTED
    with pytest.raises(OpemError):
        evaluate_test_cases(tmp_path / "missing.csv", res, tmp_path / "o.csv")


def test_regression_flow_on_the_partially_filled_mu_r_guide(tmp_path):
    """The same flow on the reference's permeability/partially_filled_rect_waveguide
    project (a partial fill of eps_r 2.45, mu_r 2, ND6, no recorded run): its
    ports see two materials, so the reader drives them by order-6 modes on the
    unsplit port faces; every test case of the first frequency passes, |S21|
    within +-1e-7 dB of 0 dB among them."""
    from project_files import reference_project
    from openparem_b200.fem3d import project_problem
    from oracle import fem
    proj, rec = reference_project(str(tmp_path), "permeability-partially-filled")
    prob, fr = project_problem(proj)
    assert [(p["mode"]["kind"], p["mode"]["nsub"], p["mode"]["order2d"]) for p in prob["ports"]] == [("FEM2D", 1, 6)] * 2
    f0 = fr[0]
    S = fem.solve_frequency(fem.Operators(prob), f0)["S"]
    res = tmp_path / "part_results.csv"
    write_results_csv(res, [f0], S[None], 0.0, "DB", "GHz")
    cases = [r for r in _regression()["permeability-partially-filled"]["test_cases"] if float(r[1]) == f0]
    tc = tmp_path / "cases.csv"
    with open(tc, "w") as fh:
        fh.write("# ResultDatabase::save_as_test\n" + "\n".join(",".join(r) for r in cases) + "\n")
    n, npass = evaluate_test_cases(tc, res, tmp_path / "out.csv")
    assert n == len(cases) >= 8 and npass == n
