"""CPU checks of the C ABI library: it loads, exports every declared symbol and
reports errors (without a GPU) through status codes instead of crashing."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "opem_b200.h")
LIB = os.path.join(ROOT, "openparem_b200", "libopem_b200.so")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(opem_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        from openparem_b200 import build
        build.build()
    return C.CDLL(LIB)


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ["opem_context_create", "opem_problem_create", "opem_problem_assemble", "opem_solve_frequency",
              "opem_solve_sweep", "opem_get_fields", "opem_get_operator"]:
        assert n in names


def test_every_declared_symbol_is_exported(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_binding_table_matches_header():
    from openparem_b200 import _lib
    bound = sorted(n for n, _, _ in _lib.SIGNATURES)
    assert bound == declared_functions()


def test_default_opts(lib):
    from openparem_b200 import _lib
    L = _lib.lib()
    o = _lib.SolverOpts()
    L.opem_default_opts(C.byref(o))
    assert o.rtol == 1e-10 and o.maxits == 5000 and o.force_reciprocal == 1


def test_null_arguments_rejected(lib):
    from openparem_b200 import _lib
    L = _lib.lib()
    assert L.opem_context_create(0, None) == _lib.ERR_ARG
    assert L.opem_problem_assemble(None) == _lib.ERR_ARG
    assert L.opem_solve_frequency(None, 1e9, None, None, None, None) == _lib.ERR_ARG
    assert L.opem_context_last_error(None) == b"null context"


def test_context_without_device_reports_error():
    """On a machine without a GPU the context call fails with a status code."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from openparem_b200 import _lib
    h = C.c_void_p()
    rc = _lib.lib().opem_context_create(0, C.byref(h))
    assert rc in (_lib.ERR_CUDA, _lib.ERR_ARG)
    assert not h.value


def test_server_without_gpu_reports_status(lib):
    """Server creation on a machine without a usable device fails with a status
    code (no crash), and null arguments are rejected."""
    from openparem_b200 import _lib
    L = _lib.lib()
    h = C.c_void_p()
    assert L.opem_server_create(0, 0, 0, C.byref(h)) == _lib.ERR_ARG
    assert L.opem_server_create(0, 2, 0, None) == _lib.ERR_ARG
    assert L.opem_server_destroy(None) == _lib.ERR_ARG
    assert L.opem_server_wait(None, 1, 0.0, None, None, None) == _lib.ERR_ARG
    rc = L.opem_server_create(0, 2, 0, C.byref(h))
    if rc == _lib.OK:   # a GPU is present after all
        assert L.opem_server_destroy(h) == _lib.OK
    else:
        assert rc in (_lib.ERR_CUDA, _lib.ERR_ARG) and not h

