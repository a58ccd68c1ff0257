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
