"""The allocation-free assembly entry point, opem_system_matrix_noalloc.

It exists for callers that cannot allocate device memory when they need the
system matrix: a process whose GPU memory is already owned by another
allocator (a PETSc/Kokkos pool, or a serving process that reserves its whole
HBM budget at start-up), or a latency-critical loop that must not call
cudaMalloc/cudaFree.  Instead of a cudaMalloc'd staging buffer it uses a
static 16 MiB device array, so it is limited to OPEM_NOALLOC_MAX_NNZ nonzeros.

The test goes through the C ABI (ctypes) and compares two calls in a row with
the allocating entry point opem_get_system_matrix, at the 1e-12 relative
tolerance the operator parity tests use.  The cases cover analytic TE ports,
copper walls with a lossy slab, and ports driven by their own 2D mode (the
slab-loaded WR90 project through the project reader), whose propagation
constant comes from the 2D mode solve rather than the TE formula.  This file sorts last so a run that
stops at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from openparem_b200 import meshgen, Fem3D, _lib
from openparem_b200.fem3d import Context

pytestmark = pytest.mark.gpu


def _noalloc(F, freq, d, nnz):
    out = np.full(2 * nnz, np.nan)
    rc = _lib.lib().opem_system_matrix_noalloc(F.h, float(freq), int(d), out.ctypes.data_as(_lib.DP))
    return rc, out[0::2] + 1j * out[1::2]


@pytest.mark.parametrize("case", ["c1_nd1", "slab_nd2_copper", "loaded_2d_mode_ports"])
def test_noalloc_matches_allocating_entry_point(case, tmp_path):
    ctx = Context(0)
    if case == "loaded_2d_mode_ports":
        from openparem_b200.fem3d import project_problem
        from project_files import reference_project
        proj, _ = reference_project(str(tmp_path), "straight-loaded")
        assert [p["mode"]["kind"] for p in project_problem(proj, order=2)[0]["ports"]] == ["FEM2D", "FEM2D"]
        F, _ = Fem3D.from_project(proj, order=2, context=ctx)
        F.assemble()
    else:
        if case == "c1_nd1":
            prob = meshgen.config1()[0]
        else:
            prob = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 20e-3, 3, 2, 6, 2, wall="impedance",
                                             wall_sigma=5.8e7, wall_Rz=0.5e-6, slab=(5e-3, 12e-3, 4.4, 0.02))
        F = Fem3D(prob, context=ctx).assemble()
    nnz = F.info()["nnz"]
    assert nnz <= _lib.NOALLOC_MAX_NNZ
    for freq, d in [(9.3e9, 0), (11.1e9, 1)]:
        ref = F.system_matrix(freq, d).data
        scale = np.abs(ref).max()
        for _ in range(2):   # two calls in a row share the static array
            rc, vals = _noalloc(F, freq, d, nnz)
            assert rc == _lib.OK, _lib.lib().opem_context_last_error(ctx.h)
            assert np.all(np.isfinite(vals))
            assert np.abs(vals - ref).max() <= 1e-12 * scale
    F.close()
    ctx.close()


def test_noalloc_rejects_problems_beyond_its_limit():
    ctx = Context(0)
    prob = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 20e-3, 6, 3, 8, 3)
    F = Fem3D(prob, context=ctx).assemble()
    nnz = F.info()["nnz"]
    assert nnz > _lib.NOALLOC_MAX_NNZ
    out = np.zeros(2 * nnz)   # full size, so even a wrong acceptance could not overrun it
    rc = _lib.lib().opem_system_matrix_noalloc(F.h, 10e9, 0, out.ctypes.data_as(_lib.DP))
    assert rc == _lib.ERR_ARG
    assert b"OPEM_NOALLOC_MAX_NNZ" in _lib.lib().opem_context_last_error(ctx.h)
    F.close()
    ctx.close()
