"""ctypes binding of libopem_b200.so (the C ABI declared in include/opem_b200.h).

The library is built in-tree by ``openparem_b200.build``.  There is no
fallback: if the shared library is missing, importing this module raises.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libopem_b200.so")

OK = 0
ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_STATE, ERR_MESH = -1, -2, -3, -4, -5
ERR_NOT_CONVERGED, ERR_BREAKDOWN, ERR_TIMEOUT, ERR_UNSUPPORTED = -6, -7, -8, -9
ERR_CANCELLED = -10
BDR_PEC, BDR_PMC, BDR_PORT, BDR_IMPEDANCE, BDR_RADIATION = 1, 2, 3, 4, 5
PREC_FP64, PREC_MIXED = 0, 1
NOALLOC_MAX_NNZ = 1 << 20

ERROR_NAMES = {ERR_ARG: "OPEM_ERR_ARG", ERR_CUDA: "OPEM_ERR_CUDA", ERR_NOMEM: "OPEM_ERR_NOMEM",
               ERR_STATE: "OPEM_ERR_STATE", ERR_MESH: "OPEM_ERR_MESH", ERR_NOT_CONVERGED: "OPEM_ERR_NOT_CONVERGED",
               ERR_BREAKDOWN: "OPEM_ERR_BREAKDOWN", ERR_TIMEOUT: "OPEM_ERR_TIMEOUT",
               ERR_UNSUPPORTED: "OPEM_ERR_UNSUPPORTED", ERR_CANCELLED: "OPEM_ERR_CANCELLED"}


class SolverOpts(C.Structure):
    _fields_ = [("rtol", C.c_double), ("maxits", C.c_int), ("restart", C.c_int), ("precision", C.c_int),
                ("poly_degree", C.c_int), ("force_reciprocal", C.c_int), ("h_maxits", C.c_int),
                ("h_rtol", C.c_double), ("deflate", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("outer", C.c_int), ("h_iterations", C.c_int), ("converged", C.c_int),
                ("rnorm", C.c_double), ("seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


P = C.c_void_p
DP = C.POINTER(C.c_double)
I64P = C.POINTER(C.c_int64)
I32P = C.POINTER(C.c_int32)

# (name, restype, argtypes)
SIGNATURES = [
    ("opem_context_create", C.c_int, [C.c_int, C.POINTER(P)]),
    ("opem_context_destroy", C.c_int, [P]),
    ("opem_context_last_error", C.c_char_p, [P]),
    ("opem_default_opts", None, [C.POINTER(SolverOpts)]),
    ("opem_problem_create", C.c_int, [P, C.c_int64, DP, C.c_int64, I64P, I32P, C.c_int64, I64P, I32P, C.c_int,
                                      C.POINTER(P)]),
    ("opem_problem_destroy", C.c_int, [P]),
    ("opem_problem_set_regions", C.c_int, [P, C.c_int, DP, DP, DP, DP]),
    ("opem_problem_set_boundary", C.c_int, [P, C.c_int, C.c_int, DP, C.c_int]),
    ("opem_problem_set_port_te", C.c_int, [P, C.c_int, DP]),
    ("opem_problem_set_port_fem2d", C.c_int, [P, C.c_int, DP, C.c_int, C.c_int]),
    ("opem_problem_set_port_impedance", C.c_int, [P, C.c_int, C.c_int, C.c_int, DP, C.c_int]),
    ("opem_mesh_errors", C.c_int, [P, C.c_double, DP, I64P, C.c_int64, I64P, DP]),
    ("opem_problem_assemble", C.c_int, [P]),
    ("opem_problem_info", C.c_int, [P, I64P, C.c_int]),
    ("opem_solve_frequency", C.c_int, [P, C.c_double, C.POINTER(SolverOpts), DP, DP, C.POINTER(SolveStats)]),
    ("opem_solve_sweep", C.c_int, [P, C.c_int, DP, C.POINTER(SolverOpts), DP, C.POINTER(SolveStats)]),
    ("opem_get_fields", C.c_int, [P, C.c_int, DP, DP]),
    ("opem_get_operator", C.c_int, [P, C.c_int, I64P, I32P, DP]),
    ("opem_get_system_matrix", C.c_int, [P, C.c_double, C.c_int, DP]),
    ("opem_context_launches", C.c_int, [P, I64P]),
    ("opem_profile_kernels", C.c_int, [P, C.c_double, C.c_int, DP, C.c_int]),
    ("opem_profile_batch_kernels", C.c_int, [P, C.c_double, C.c_int, C.c_int, DP, C.c_int]),
    ("opem_check_block_apply", C.c_int, [P, C.c_double, C.c_int, C.c_int, C.c_int, DP, C.c_int]),
    ("opem_server_create", C.c_int, [C.c_int, C.c_int, C.c_int64, C.POINTER(C.c_void_p)]),
    ("opem_server_destroy", C.c_int, [P]),
    ("opem_server_submit", C.c_int, [P, P, C.c_int, DP, P, C.POINTER(C.c_int64)]),
    ("opem_server_wait", C.c_int, [P, C.c_int64, C.c_double, DP, P, DP]),
    ("opem_server_info", C.c_int, [P, I64P, C.c_int]),
    ("opem_server_cancel", C.c_int, [P, C.c_int64]),
    ("opem_selftest_wait_timeout", C.c_int, [P, C.c_int]),
    ("opem_selftest_lsq", C.c_int, [C.c_int, C.c_int, C.c_int, DP]),
    ("opem_selftest_face_tables", C.c_int, [C.c_int, C.c_int, DP, C.c_int64]),
    ("opem_project_load", C.c_int, [P, C.c_char_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_int), DP, C.c_int]),
    ("opem_project_info", C.c_int, [C.c_char_p, C.c_int, I64P, C.c_int, DP, C.c_int, C.c_char_p, C.c_int]),
    ("opem_project_value", C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int]),
    ("opem_project_read", C.c_int, [C.c_char_p, C.c_int, I64P, DP, I64P, I32P, DP, I64P, I32P, I32P, DP, DP, I32P,
                                     DP, C.c_char_p, C.c_int]),
    ("opem_port_mode_2d", C.c_int, [C.c_int64, DP, C.c_int64, I64P, DP, DP, C.c_double, DP, I64P, I64P, DP, DP]),
    ("opem_port_mode_faces", C.c_int, [C.c_int64, DP, C.c_int64, I64P, DP, DP, DP, C.c_int, C.c_int, C.c_double, DP,
                                        C.c_int64, I64P, DP, DP, DP]),
    ("opem_project_port_impedance", C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                               C.POINTER(C.c_int), DP, C.c_int, C.c_char_p, C.c_int]),
    ("opem_port_mode_faces_z", C.c_int, [C.c_int64, DP, C.c_int64, I64P, DP, DP, DP, C.c_int, C.c_int, C.c_double,
                                          C.c_int, C.c_int, DP, C.c_int, C.c_int, DP]),
    ("opem_s_renormalize", C.c_int, [C.c_int, DP, DP, C.c_double, C.c_double, DP]),
    ("opem_write_touchstone", C.c_int, [C.c_char_p, C.c_int, DP, C.c_int, DP, C.c_double, C.c_char_p, C.c_char_p]),
    ("opem_s_mixed_mode", C.c_int, [C.c_int, DP, C.c_int, C.POINTER(C.c_int), C.c_double, DP, DP]),
    ("opem_s_single_ended", C.c_int, [C.c_int, DP, DP, DP, DP, C.c_double, DP, DP]),
    ("opem_problem_add_port_mode", C.c_int, [C.c_void_p, C.c_int, C.c_int, DP, C.c_int, C.c_int, DP, C.c_int,
                                             C.POINTER(C.c_int)]),
    ("opem_port_line_maps", C.c_int, [C.c_int, DP, DP, DP, DP, C.POINTER(C.c_int), DP, DP]),
    ("opem_s_relative_change", C.c_int, [C.c_int, DP, DP, DP]),
    ("opem_refine_mesh", C.c_int, [C.c_int64, DP, C.c_int64, I64P, I32P, C.c_int64, I64P, I32P, C.c_int64, I64P,
                                    I64P, DP, I64P, I32P, I64P, I32P]),
    ("opem_write_results_csv", C.c_int, [C.c_char_p, C.c_int, DP, C.c_int, DP, C.c_double, C.c_char_p, C.c_char_p]),
    ("opem_evaluate_test_cases", C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(C.c_int),
                                            C.POINTER(C.c_int)]),
    ("opem_write_touchstone2", C.c_int, [C.c_char_p, C.c_int, DP, C.c_int, DP, C.c_double, C.c_char_p, C.c_char_p,
                                          C.c_int, C.POINTER(C.c_int)]),
    ("opem_system_matrix_noalloc", C.c_int, [P, C.c_double, C.c_int, DP]),
]


def load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m openparem_b200.build` "
                          "(the solve stage has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = load()
    return _LIB
