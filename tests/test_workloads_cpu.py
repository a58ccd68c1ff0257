"""CPU checks of the synthetic workload generators (configs 4 and 5): seeded,
deterministic, and of the stated shapes and sizes."""
import numpy as np

from openparem_b200 import meshgen


def test_config4_sections():
    a = meshgen.config4(seed=0)
    b = meshgen.config4(seed=0)
    assert len(a) == 64
    orders = set()
    for (pa, fa), (pb, fb) in zip(a, b):
        assert np.array_equal(pa["tets"], pb["tets"]) and np.array_equal(fa, fb)
        assert len(fa) == 1 and 8e9 <= fa[0] <= 12e9
        orders.add(pa["order"])
        z = pa["verts"][:, 2]
        L = z.max() - 5e-3                      # guide length without the 5 mm air cap
        assert 10e-3 - 1e-9 <= L <= 60e-3 + 1e-9
        types = sorted(v["type"] for v in pa["boundaries"].values())
        assert types == ["pec", "port", "radiation"] and len(pa["ports"]) == 1
    assert orders == {1, 2}


def test_config5_stream():
    reqs = meshgen.config5(seed=0, count=6, max_dofs=200_000)
    t = [r[0] for r in reqs]
    assert all(t1 > t0 for t0, t1 in zip(t, t[1:]))          # Poisson arrival times increase
    for _, p, f in reqs:
        a = p["verts"][:, 0].max() - p["verts"][:, 0].min()
        assert 20e-3 - 1e-9 <= a <= 24e-3 + 1e-9                 # TE10 the only propagating air mode
        assert 1 <= len(f) <= 4 and np.all((f >= 8e9) & (f <= 12e9))
        assert p["order"] in (1, 2, 3)
        assert 1.0 <= p["eps_r"][1] <= 10.0 and p["tand"][1] == 0.01
        nhex = len(p["tets"]) / 6
        assert nhex * meshgen.DOF_PER_HEX[p["order"]] <= 3 * 200_000
