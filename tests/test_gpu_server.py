"""GPU tests of the serving loop (opem_server_*): requests of different sizes
run overlapped on one GPU and each result is the same as the same request
run alone.

Tolerances
  server vs the same request through the server alone: |dS| <= 1e-12 (the
      kernels are deterministic and read only their own request's data)
  server vs a direct FP64 sweep on the caller's stream: |dS| <= 1e-12
  server vs a direct batched (mixed) sweep: |dS| <= 1e-8 (the server caps the
      batched workspace, which may split the sweep into other batches)
  mixed-precision requests run concurrently vs the same requests alone:
      |dS| <= 1e-8 (same reason)
"""
import numpy as np
import pytest

from openparem_b200 import meshgen, Fem3D, Server, Context, default_opts
from openparem_b200 import _lib

pytestmark = pytest.mark.gpu


def _problems():
    return [
        ("c1_nd1", meshgen.config1()[0], np.array([9.0e9, 10.0e9, 11.0e9])),
        ("slab_nd2", meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 20e-3, 3, 2, 6, 2,
                                               slab=(5e-3, 12e-3, 4.4, 0.02)), np.array([8.5e9, 10.5e9])),
        ("air_nd3", meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 20e-3, 3, 2, 4, 3),
         np.array([9.5e9, 11.5e9, 10.0e9, 8.2e9])),
        ("cap_nd1", meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 20e-3, 4, 2, 8, 1, ports=("zmin",),
                                              radiation_cap=5e-3, cap_nz=2), np.array([10.0e9])),
    ]


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _overlaps(ts):
    for i in range(len(ts)):
        for j in range(i + 1, len(ts)):
            a, b = ts[i], ts[j]
            if a["started"] < b["finished"] and b["started"] < a["finished"]:
                return True
    return False


def test_results_alone_equal_results_in_the_mix(ctx):
    probs = _problems()
    fems = [Fem3D(p, context=ctx) for _, p, _ in probs]   # assembled by their first request
    opts = default_opts(rtol=1e-10)
    srv = Server(0, slots=4)
    try:
        alone = []
        for F, (_, _, fr) in zip(fems, probs):
            S, st, _ = srv.wait(srv.submit(F, fr, opts))
            assert all(s["converged"] == 1 for s in st)
            alone.append(S)
        ids = [srv.submit(F, fr, opts) for F, (_, _, fr) in zip(fems, probs)]
        mix, times = [], []
        for rid in ids:
            S, st, t = srv.wait(rid)
            mix.append(S)
            times.append(t)
        for (name, _, _), a, m in zip(probs, alone, mix):
            assert np.abs(a - m).max() <= 1e-12, name
        assert _overlaps(times), "no two requests ran at the same time"
        assert srv.info()["completed"] == 2 * len(probs)
        # the server's FP64 result equals a direct sweep on the caller's own stream
        for F, (name, _, fr), a in zip(fems, probs, alone):
            S, _ = F.sweep(fr, opts)
            assert np.abs(S - a).max() <= 1e-12, name
    finally:
        srv.close()


def test_concurrent_mixed_requests_equal_alone(ctx):
    """Three mixed-precision (batched sweep) requests of different orders and
    sizes submitted at once, with no budget limit: their run intervals overlap on
    the GPU and each S equals the same request run alone (|dS| <= 1e-8), all
    systems converged."""
    probs = _problems()[:3]
    fems = [Fem3D(p, context=ctx).assemble() for _, p, _ in probs]
    opts = default_opts(rtol=1e-10, precision=_lib.PREC_MIXED, poly_degree=8)
    srv = Server(0, slots=3)
    try:
        alone = []
        for F, (_, _, fr) in zip(fems, probs):
            S, st, _ = srv.wait(srv.submit(F, fr, opts))
            assert all(s["converged"] == 1 for s in st)
            alone.append(S)
        ids = [srv.submit(F, fr, opts) for F, (_, _, fr) in zip(fems, probs)]
        res = [srv.wait(r) for r in ids]
    finally:
        srv.close()
    assert _overlaps([r[2] for r in res]), "no two mixed requests ran at the same time"
    for (name, _, _), a, (S, st, _) in zip(probs, alone, res):
        assert all(s["converged"] == 1 for s in st), name
        assert np.abs(S - a).max() <= 1e-8, name


def test_budget_serialises_and_mixed_requests(ctx):
    probs = _problems()[:3]
    fems = [Fem3D(p, context=ctx).assemble() for _, p, _ in probs]
    opts = default_opts(rtol=1e-10, precision=_lib.PREC_MIXED, poly_degree=8)
    srv = Server(0, slots=3, hbm_budget_bytes=1)   # every request exceeds the budget: one at a time
    try:
        ids = [srv.submit(F, fr, opts) for F, (_, _, fr) in zip(fems, probs)]
        res = [srv.wait(r) for r in ids]
    finally:
        srv.close()
    times = sorted((r[2] for r in res), key=lambda t: t["started"])
    for a, b in zip(times, times[1:]):
        assert b["started"] >= a["finished"]
    for F, (name, _, fr), (S, st, _) in zip(fems, probs, res):
        assert all(s["converged"] == 1 for s in st)
        Sd, _ = F.sweep(fr, opts)
        assert np.abs(S - Sd).max() <= 1e-8, name


def test_wait_timeout_and_bad_requests(ctx):
    F = Fem3D(_problems()[1][1], context=ctx).assemble()
    srv = Server(0, slots=1)
    try:
        rid = srv.submit(F, [10e9], default_opts())
        S, st, t = srv.wait(rid, timeout=120.0)
        assert st[0]["converged"] == 1 and t["finished"] >= t["started"] >= t["submitted"]
        with pytest.raises(Exception):
            srv.submit(F, [-1.0], default_opts())
        with pytest.raises(KeyError):
            srv.wait(12345)
    finally:
        srv.close()


def test_cancel_queued_and_running(ctx):
    """Cancelled requests: a queued one is dropped, a running one stops at its next
    Krylov step; both waits report ERR_CANCELLED and the problems stay usable."""
    from openparem_b200.fem3d import OpemError
    big = Fem3D(meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 50e-3, 12, 6, 30, 2,
                                          slab=(20e-3, 30e-3, 4.4, 0.02)), context=ctx).assemble()
    small = Fem3D(_problems()[0][1], context=ctx).assemble()
    srv = Server(0, slots=1)
    try:
        opts = default_opts(rtol=1e-12, restart=100)
        r_big = srv.submit(big, np.linspace(8e9, 12e9, 6), opts)    # FP64 path, several seconds
        r_small = srv.submit(small, [10e9], opts)                   # queued behind it (one slot)
        srv.cancel(r_small)
        with pytest.raises(OpemError) as e1:
            srv.wait(r_small, timeout=60.0)
        assert e1.value.code == _lib.ERR_CANCELLED
        import time
        t0 = time.time()
        while srv.info()["running"] == 0 and time.time() - t0 < 60:
            time.sleep(0.01)
        srv.cancel(r_big)
        with pytest.raises(OpemError) as e2:
            srv.wait(r_big, timeout=300.0)
        assert e2.value.code == _lib.ERR_CANCELLED
        S, st, _ = srv.wait(srv.submit(small, [10e9], opts))   # the flag is cleared for the next request
        assert st[0]["converged"] == 1
    finally:
        srv.close()


def test_bounded_wait_timeout_selftest(ctx):
    """The device-side bounded wait gives up, reports OPEM_ERR_TIMEOUT through its
    status word, and the context keeps working."""
    L = _lib.lib()
    assert L.opem_selftest_wait_timeout(ctx.h, 1 << 14) == _lib.ERR_TIMEOUT
    F = Fem3D(_problems()[0][1], context=ctx).assemble()
    S, _, st = F.solve(10e9)
    assert st["converged"] == 1
