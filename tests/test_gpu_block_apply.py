"""GPU: the batched vertex-patch block apply (the preconditioner that replaces
the reference's direct PCLU, solveComplexLinearSystem.c:153-161) on the
tensor cores (tcgen05, split TF32 operands, FP32 accumulation in tensor
memory) and on the FP32 FMA pipe, both against an FP64 host product of the
same FP32 blocks and inputs, through the C ABI.

Tolerance: 1e-5 of the largest result for both kernels (FP32 accumulation over
patches of up to 100 DOFs; the split products keep about 22 mantissa bits)."""
import numpy as np
import pytest

from openparem_b200 import meshgen, Fem3D, _lib
from openparem_b200.fem3d import Context

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _check(F, freq, nsys, r0, nd):
    out = np.zeros(5)
    rc = _lib.lib().opem_check_block_apply(F.h, float(freq), nsys, r0, nd, out.ctypes.data_as(_lib.DP), 5)
    assert rc == _lib.OK, _lib.lib().opem_context_last_error(F.ctx.h)
    return out


@pytest.mark.parametrize("nsys,r0,nd", [(26, 0, 13), (26, 13, 13), (8, 0, 8), (1, 0, 1), (32, 0, 32), (20, 3, 17)])
def test_tensor_core_block_apply_nd2(nsys, r0, nd):
    ctx = Context(0)
    prob = meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 20e-3, 4, 2, 8, 2, slab=(5e-3, 12e-3, 4.4, 0.02))
    F = Fem3D(prob, context=ctx).assemble()
    assert F.info()["max_patch"] <= 128
    out = _check(F, 10e9, nsys, r0, nd)
    assert out[4] == 0            # no bounded wait ran out
    assert out[2] in (1, 2)       # the solver's pick (the faster kernel on first use)
    assert 0 <= out[0] <= TOL
    assert out[1] <= TOL
    F.close()
    ctx.close()


def test_tensor_core_block_apply_nd1_and_nd3_fallback():
    ctx = Context(0)
    F1 = Fem3D(meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 20e-3, 3, 2, 6, 1), context=ctx).assemble()
    out = _check(F1, 9e9, 13, 0, 13)
    assert out[4] == 0 and 0 <= out[0] <= TOL and out[1] <= TOL
    F3 = Fem3D(meshgen.waveguide_problem(meshgen.WR_A, meshgen.WR_B, 20e-3, 3, 2, 6, 3), context=ctx).assemble()
    if F3.info()["max_patch"] > 128:
        out = _check(F3, 9e9, 13, 0, 13)
        assert out[0] == -1 and out[2] == 1 and out[1] <= TOL
    F1.close()
    F3.close()
    ctx.close()
