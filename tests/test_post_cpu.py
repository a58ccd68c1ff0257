"""CPU tests of the host-side S-parameter post-processing (renormalisation and
Touchstone output); no GPU is needed for these entry points."""
import numpy as np
import pytest

from openparem_b200.fem3d import renormalize, write_touchstone, OpemError


def _ref_renorm(S, Zo, zref):
    """Restatement of the reference's S2Z / Z2S (results.cpp:455-565) in numpy."""
    n = S.shape[0]
    I = np.eye(n)
    k = np.diag(np.sqrt(Zo))
    Z = k @ (I + S) @ np.linalg.inv(I - S) @ k
    kr = np.diag(np.full(n, np.sqrt(zref + 0j)))
    kri = np.linalg.inv(kr)
    return np.linalg.inv(Z @ kri + kr) @ (Z @ kri - kr)


def _random_s(n, rng):
    A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    return 0.4 * A / np.linalg.norm(A, 2)


@pytest.mark.parametrize("n", [1, 2, 3, 5])
def test_renormalize_matches_reference_formula(n):
    rng = np.random.default_rng(n)
    S = _random_s(n, rng)
    Zo = 400 + 80 * rng.normal(size=n) + 1j * 30 * rng.normal(size=n)
    out = renormalize(S, Zo, 50.0)
    assert np.abs(out - _ref_renorm(S, Zo, 50.0)).max() < 1e-12
    back = renormalize(out, np.full(n, 50.0 + 0j), Zo[0]) if np.allclose(Zo, Zo[0]) else None
    assert back is None or np.abs(back - S).max() < 1e-12


def test_renormalize_identity_and_round_trip():
    rng = np.random.default_rng(7)
    S = _random_s(2, rng)
    z = 377.0 + 12j
    assert np.abs(renormalize(S, [z, z], z) - S).max() < 1e-13
    S50 = renormalize(S, [z, z], 50.0)
    assert np.abs(renormalize(S50, [50.0, 50.0], z) - S).max() < 1e-12
    with pytest.raises(OpemError):
        renormalize(np.eye(2), [50.0, 50.0], 50.0)   # I - S singular


def _parse(path):
    head, rows = [], []
    for ln in open(path):
        ln = ln.rstrip("\n")
        if ln.startswith("!") or not ln.strip():
            head.append(ln)
            continue
        if ln.startswith("#"):
            head.append(ln)
            continue
        rows.append(ln.split("!")[0].split())
    return head, rows


def test_touchstone_two_port_layout(tmp_path):
    rng = np.random.default_rng(1)
    f = np.array([8e9, 9.5e9])
    S = np.stack([_random_s(2, rng) for _ in f])
    p = tmp_path / "t.s2p"
    write_touchstone(p, f, S, 50.0, "RI", "GHz")
    head, rows = _parse(p)
    assert "# GHz S RI R 50" in head
    assert len(rows) == 2
    for q, r in enumerate(rows):
        v = np.array(r, dtype=float)
        assert abs(v[0] - f[q] * 1e-9) < 1e-12
        got = v[1::2] + 1j * v[2::2]
        want = np.array([S[q, 0, 0], S[q, 1, 0], S[q, 0, 1], S[q, 1, 1]])   # column by column
        assert np.abs(got - want).max() < 1e-13


def test_touchstone_many_ports_and_formats(tmp_path):
    rng = np.random.default_rng(2)
    n = 5
    f = np.array([10e9])
    S = _random_s(n, rng)[None]
    p = tmp_path / "t.s5p"
    write_touchstone(p, f, S, 75.0, "DB", "MHz")
    head, rows = _parse(p)
    assert "# MHz S DB R 75" in head
    vals = [float(x) for r in rows for x in r]
    assert abs(vals[0] - 1e4) < 1e-9
    pairs = np.array(vals[1:]).reshape(-1, 2)
    assert pairs.shape[0] == n * n
    want = S[0].ravel()                                                   # row by row
    assert np.abs(pairs[:, 0] - 20 * np.log10(np.abs(want))).max() < 1e-12
    assert np.abs(pairs[:, 1] - np.angle(want, deg=True)).max() < 1e-12
    # at most four pairs per line; two lines per row of 5 entries
    assert len(rows) == 2 * n
    ma = tmp_path / "m.s5p"
    write_touchstone(ma, f, S, 75.0, "MA", "Hz")
    _, rows2 = _parse(ma)
    pairs2 = np.array([float(x) for r in rows2 for x in r][1:]).reshape(-1, 2)
    assert np.abs(pairs2[:, 0] - np.abs(want)).max() < 1e-13
    with pytest.raises(OpemError):
        write_touchstone(tmp_path / "x.s5p", f, S, 75.0, "XY", "GHz")


def _ref_mixed(S, pairs, zref):
    """fem3D::build_Mc_Ms (conversion 1) + Result::SparameterConversion restated in numpy."""
    n = S.shape[0]
    za = np.full(n, zref, dtype=complex)
    zb = za.copy()
    Kv = np.eye(n, dtype=complex)
    Ki = np.eye(n, dtype=complex)
    for p, q in pairs:
        p -= 1; q -= 1
        zb[p], zb[q] = zref / 2, 2 * zref
        Kv[p, p], Kv[p, q], Kv[q, p], Kv[q, q] = 0.5, 0.5, 1, -1
        Ki[p, p], Ki[p, q], Ki[q, p], Ki[q, q] = 1, 1, 0.5, -0.5
    t1 = np.diag(1 / np.sqrt(zb)) @ Kv @ np.diag(np.sqrt(za))
    t2 = np.diag(np.sqrt(zb)) @ Ki @ np.diag(1 / np.sqrt(za))
    Ms, Mc = 0.5 * (t1 + t2), 0.5 * (t1 - t2)
    return (Mc + Ms @ S) @ np.linalg.inv(Ms + Mc @ S), zb


def test_mixed_mode_matches_reference_formula():
    from openparem_b200.fem3d import mixed_mode
    rng = np.random.default_rng(11)
    for n, pairs in ((2, [(1, 2)]), (4, [(1, 2), (3, 4)]), (4, [(2, 4)]), (5, [(1, 3), (4, 5)])):
        S = _random_s(n, rng)
        S = 0.5 * (S + S.T)
        out, zo = mixed_mode(S, pairs, 50.0)
        ref, zb = _ref_mixed(S, pairs, 50.0)
        assert np.abs(out - ref).max() < 1e-12 and np.allclose(zo, zb)


def test_mixed_mode_of_two_uncoupled_lines():
    """Two identical matched 50-ohm thru lines (1->3, 2->4): the common (25 ohm) and
    differential (100 ohm) modes are matched, both carry the thru, no mode conversion."""
    from openparem_b200.fem3d import mixed_mode
    t = 0.8 * np.exp(-0.7j)
    S = np.zeros((4, 4), dtype=complex)
    S[0, 2] = S[2, 0] = S[1, 3] = S[3, 1] = t
    out, zo = mixed_mode(S, [(1, 2), (3, 4)], 50.0)
    assert np.allclose(zo, [25, 100, 25, 100])
    assert abs(out[2, 0] - t) < 1e-14 and abs(out[3, 1] - t) < 1e-14      # Scc21, Sdd21
    assert abs(out[0, 0]) < 1e-14 and abs(out[1, 1]) < 1e-14              # matched modes
    assert abs(out[3, 0]) < 1e-14 and abs(out[2, 1]) < 1e-14              # no conversion
    with pytest.raises(OpemError):
        mixed_mode(S, [(1, 1)], 50.0)


def test_single_ended_identity_maps_renormalise():
    """With Tv = Ti = I the modal to single-ended conversion only changes the
    reference impedance of every S-port from the mode's to zref: it equals the
    reference's renormalisation (S2Z / Z2S) to zref."""
    from openparem_b200.fem3d import single_ended
    rng = np.random.default_rng(13)
    for n in (1, 2, 4):
        S = _random_s(n, rng)
        Zm = 60 + 20 * rng.random(n) + 1j * 5 * rng.normal(size=n)
        out = single_ended(S, Zm, np.eye(n), np.eye(n), 50.0)
        assert np.abs(out - _ref_renorm(S, Zm, 50.0)).max() < 1e-12


def test_single_ended_from_line_voltages_and_currents():
    """Two two-conductor ports (four S-ports): modal waves a_m, b_m = S a_m give
    modal line voltages V = sqrt(Zm)(a + b) and currents I = (a - b)/sqrt(Zm); the
    single-ended ones are Tv^-1 V and Ti^-1 I, whose waves at zref,
    (V/sqrt(zref) +- sqrt(zref) I)/2, must satisfy b_s = S_out a_s for every a_m."""
    from openparem_b200.fem3d import single_ended
    rng = np.random.default_rng(17)
    n = 4
    S = _random_s(n, rng)
    Zm = np.array([30 + 2j, 70 - 3j, 28 + 1j, 75 + 0j])
    Tv = np.zeros((n, n), dtype=complex)
    Ti = np.zeros((n, n), dtype=complex)
    for b in (0, 2):   # one 2 x 2 block per port
        Tv[b:b + 2, b:b + 2] = rng.normal(size=(2, 2)) + 0.1j * rng.normal(size=(2, 2)) + 2 * np.eye(2)
        Ti[b:b + 2, b:b + 2] = rng.normal(size=(2, 2)) + 0.1j * rng.normal(size=(2, 2)) + 2 * np.eye(2)
    zref = 50.0
    out = single_ended(S, Zm, Tv, Ti, zref)
    am = rng.normal(size=(n, 3)) + 1j * rng.normal(size=(n, 3))
    bm = S @ am
    V = np.sqrt(Zm)[:, None] * (am + bm)
    I = (am - bm) / np.sqrt(Zm)[:, None]
    Vs, Is = np.linalg.solve(Tv, V), np.linalg.solve(Ti, I)
    a_s = (Vs / np.sqrt(zref) + np.sqrt(zref) * Is) / 2
    b_s = (Vs / np.sqrt(zref) - np.sqrt(zref) * Is) / 2
    assert np.abs(out @ a_s - b_s).max() < 1e-12
    with pytest.raises(OpemError):
        single_ended(S, Zm, np.zeros((n, n)), Ti, zref)   # Tv singular


def test_touchstone2_layout(tmp_path):
    from openparem_b200.fem3d import write_touchstone2
    rng = np.random.default_rng(5)
    fr = np.array([9e9, 10e9])
    S = np.stack([_random_s(4, rng) for _ in fr])
    path = tmp_path / "mm.s4p"
    write_touchstone2(path, fr, S, 50.0, "RI", "GHz", pairs=[(1, 2), (3, 4)])
    lines = open(path).read().splitlines()
    assert "[Version] 2.0" in lines and "[Number of Ports] 4" in lines and "[Number of Frequencies] 2" in lines
    assert "[Matrix Format] Full" in lines and lines[-1] == "[End]"
    assert "[Mixed-Mode Order] C1,2 D1,2 C3,4 D3,4" in lines
    assert "! S-port comm_net1_net2" in lines and "! S-port diff_net3_net4" in lines
    data = lines[lines.index("[Network Data]") + 1:-1]
    vals = np.array([float(x) for ln in data for x in ln.split("!")[0].split()])
    assert len(vals) == 2 * (1 + 2 * 16)
    assert abs(vals[0] - 9.0) < 1e-12 and abs(vals[1] - S[0, 0, 0].real) < 1e-14
    # two ports: 21_12 order keyword, data column by column as in version 1.1
    write_touchstone2(tmp_path / "a.s2p", fr, S[:, :2, :2], 50.0, "MA", "GHz")
    l2 = open(tmp_path / "a.s2p").read().splitlines()
    assert "[Two-Port Data Order] 21_12" in l2 and not any(x.startswith("[Mixed-Mode") for x in l2)


def _ref_line_maps(I, V):
    """The reference's line calculation (OpenParEM2D fem2D.cpp:1591-1790) restated
    in numpy: per mode, signs of the line currents scaled by the return-current
    rule, a flip when the first entry is negative, Tv = (conj(Ti)^-1)^T."""
    I, V = np.array(I, dtype=complex), np.array(V, dtype=complex)
    n = I.shape[0]
    Ti = np.zeros((n, n), dtype=complex)
    fl = np.zeros(n, dtype=bool)
    for i in range(n):
        sg = np.where(I[i].real >= 0, 1.0, -1.0)
        mc, rc = np.sum(sg * I[i]), np.sum(I[i])
        Ti[i] = sg * 0.5 * (abs(mc) + abs(rc)) / abs(mc)
        if Ti[i, 0].real < 0:
            fl[i] = True
            Ti[i], I[i], V[i] = -Ti[i], -I[i], -V[i]
    Tv = np.linalg.inv(Ti.conj()).T
    return Ti, Tv, fl, np.sum(Ti * I, axis=1), np.sum(Tv * V, axis=1)


def test_port_line_maps_even_odd_pair():
    """Symmetric coupled lines: the even mode (equal line currents c) maps with
    Ti row [1, 1] and the odd mode (c, -c) with [1/2, -1/2]; the odd mode given
    with its first current negative is flipped; the mode currents are 2c and c."""
    from openparem_b200.fem3d import port_line_maps
    c = 0.02 - 0.001j
    I = np.array([[c, c], [-c, c]])
    V = np.array([[3.0 + 0.1j, 3.0 + 0.1j], [-1.2, 1.2]])
    r = port_line_maps(I, V)
    assert np.abs(r["Ti"] - np.array([[1, 1], [0.5, -0.5]])).max() < 1e-15
    assert list(r["flipped"]) == [False, True]
    assert np.abs(r["Im"] - np.array([2 * c, c])).max() < 1e-15
    # Tv = (conj(Ti)^-1)^T: even-mode voltage is the line mean, odd the difference
    assert np.abs(r["Tv"] - np.array([[0.5, 0.5], [1.0, -1.0]])).max() < 1e-15
    assert np.abs(r["Vm"] - np.array([3.0 + 0.1j, 2.4])).max() < 1e-15


@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_port_line_maps_match_reference_rule_and_conserve_power(n):
    """Random mode currents and voltages on n lines: the library's maps equal the
    restated rule, and V_m . conj(I_m) summed over the modes equals the same sum
    over the lines (Tv^T conj(Ti) = I), which the single-ended conversion needs."""
    from openparem_b200.fem3d import port_line_maps
    rng = np.random.default_rng(40 + n)
    while True:   # sign patterns of +-1 can be singular: those raise, tested below
        I = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)) + 2 * np.eye(n)
        if abs(np.linalg.det(np.where(I.real >= 0, 1.0, -1.0))) > 0.5:
            break
        with pytest.raises(OpemError):
            port_line_maps(I)
    V = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    r = port_line_maps(I, V)
    Ti, Tv, fl, Im, Vm = _ref_line_maps(I, V)
    for k, ref in (("Ti", Ti), ("Tv", Tv), ("Im", Im), ("Vm", Vm)):
        assert np.abs(r[k] - ref).max() < 1e-12 * max(1.0, np.abs(ref).max()), k
    assert (r["flipped"] == fl).all()
    assert np.abs(r["Tv"].T @ r["Ti"].conj() - np.eye(n)).max() < 1e-12
    # powers of line voltage/current pairs on the mode basis
    vl, il = rng.normal(size=n) + 1j * rng.normal(size=n), rng.normal(size=n) + 1j * rng.normal(size=n)
    assert abs(np.sum((r["Tv"] @ vl) * np.conj(r["Ti"] @ il)) - np.sum(vl * np.conj(il))) < 1e-12
    with pytest.raises(OpemError):
        port_line_maps(np.zeros((n, n)))   # no net current
