"""ctypes declarations of the C ABI in include/doublyexcited.h."""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libdoublyexcited_b200.so"

DE_OK = 0
DE_E_INVALID = 1
DE_E_SIZE = 2
DE_E_CUDA = 3
DE_E_NOMEM = 4
DE_E_UNSUPPORTED = 5
DE_E_CHOLESKY = 6
DE_E_GEVP = 7
DE_E_SVD = 8
DE_E_ORTHO = 9
DE_E_NOT_CONVERGED = 10
DE_E_IO = 11
DE_E_PARSE = 12
DE_E_LAPACK = 13
DE_E_NAN = 14
DE_E_BUSY = 15


class de_complex(ctypes.Structure):
    _fields_ = [("re", ctypes.c_double), ("im", ctypes.c_double)]


class de_params(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int),
        ("delta", ctypes.c_double),
        ("radius", ctypes.c_double),
        ("autodelta", ctypes.c_int),
        ("theta", ctypes.c_double),
        ("charge", ctypes.c_double),
        ("nelec", ctypes.c_int),
        ("nsmall", ctypes.c_int),
        ("tfactor", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("device", ctypes.c_int),
    ]


class de_gmres(ctypes.Structure):
    _fields_ = [
        ("max_inner_iter", ctypes.c_int),
        ("usepetscflag", ctypes.c_int),
        ("tol", ctypes.c_double),
        ("compat_first_column_only", ctypes.c_int),
    ]


class de_stats(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("converged", ctypes.c_int),
        ("matvecs", ctypes.c_int64),
        ("matvecs_reference", ctypes.c_int64),
        ("max_residual", ctypes.c_double),
        ("t_total_s", ctypes.c_double),
        ("t_matvec_s", ctypes.c_double),
        ("t_prec_s", ctypes.c_double),
        ("t_dense_s", ctypes.c_double),
    ]


class de_input(ctypes.Structure):
    _fields_ = [
        ("params", de_params),
        ("gmres", de_gmres),
        ("writevecs", ctypes.c_int),
        ("readvecs", ctypes.c_int),
        ("invecfile", ctypes.c_char * 300),
        ("outvecfile", ctypes.c_char * 300),
        ("numorbs", ctypes.c_int),
        ("singlet", ctypes.c_int),
        ("numskip", ctypes.c_int),
        ("outmodulus", ctypes.c_int),
        ("takerealpart", ctypes.c_int),
        ("hermopt", ctypes.c_int),
        ("cshiftopt", ctypes.c_int),
        ("gplmr_nev", ctypes.c_int),
        ("gplmr_ns", ctypes.c_int),
        ("gplmr_maxit", ctypes.c_int),
        ("gplmr_tol", ctypes.c_double),
        ("gplmr_shift", de_complex),
        ("kdim", ctypes.c_int),
        ("lanblocksize", ctypes.c_int),
        ("check", ctypes.c_int),
        ("lantol", ctypes.c_double),
    ]


class de_run_info(ctypes.Structure):
    _fields_ = [
        ("totget", ctypes.c_int),
        ("nexpects", ctypes.c_int),
        ("e0", de_complex * 16),
        ("expects", de_complex * 16),
        ("shift", de_complex),
        ("stats", de_stats),
    ]


class de_server_opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("workers", ctypes.c_int), ("max_bytes", ctypes.c_int64)]


class de_request(ctypes.Structure):
    _fields_ = [
        ("params", de_params),
        ("sigma", de_complex),
        ("nev", ctypes.c_int),
        ("ns", ctypes.c_int),
        ("maxit", ctypes.c_int),
        ("tol", ctypes.c_double),
        ("gm", de_gmres),
        ("x", ctypes.c_void_p),
        ("e", ctypes.c_void_p),
    ]


class de_result(ctypes.Structure):
    _fields_ = [
        ("id", ctypes.c_uint64),
        ("status", ctypes.c_int),
        ("stats", de_stats),
        ("t_submit_s", ctypes.c_double),
        ("t_start_s", ctypes.c_double),
        ("t_end_s", ctypes.c_double),
        ("footprint_bytes", ctypes.c_int64),
        ("worker", ctypes.c_int),
    ]


class DeError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


P = ctypes.c_void_p
I64 = ctypes.c_int64
INT = ctypes.c_int

# name -> (restype, argtypes); every symbol the header declares.
SIGNATURES = {
    "de_strerror": (ctypes.c_char_p, [INT]),
    "de_last_error": (ctypes.c_char_p, []),
    "de_version": (ctypes.c_char_p, []),
    "de_kernel_launches": (I64, []),
    "de_params_default": (None, [ctypes.POINTER(de_params)]),
    "de_problem_create": (INT, [ctypes.POINTER(de_params), ctypes.POINTER(P)]),
    "de_problem_destroy": (INT, [P]),
    "de_problem_dims": (INT, [P, ctypes.POINTER(INT), ctypes.POINTER(I64), ctypes.POINTER(I64)]),
    "de_set_stream": (INT, [P, P]),
    "de_set_profiling": (INT, [P, INT]),
    "de_profile_read": (INT, [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                              ctypes.POINTER(I64), ctypes.POINTER(I64)]),
    "de_profile_read32": (INT, [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                ctypes.POINTER(I64), ctypes.POINTER(I64)]),
    "de_hammult": (INT, [P, P, P, I64]),
    "de_hammult_d": (INT, [P, P, P, I64]),
    "de_matblock": (INT, [P, P, P, I64, I64, INT]),
    "de_matblock_d": (INT, [P, P, P, I64, I64, INT]),
    "de_matblock32_d": (INT, [P, P, P, I64, I64, INT]),
    "de_dots": (INT, [P, P, P, I64, INT, INT, P, INT]),
    "de_dots_d": (INT, [P, P, P, I64, INT, INT, P, INT]),
    "de_dots_noalloc_d": (INT, [P, P, I64, INT, INT, P, INT, P]),
    "de_get_expects": (INT, [P, P, INT, INT, P]),
    "de_subspace_guess": (INT, [P, INT, INT, INT, de_complex, INT, P, P]),
    "de_subspace_guess_d": (INT, [P, INT, INT, INT, de_complex, INT, P, P]),
    "de_heplus_orbitals": (INT, [INT, P, INT, INT, P, P]),
    "de_run": (INT, [ctypes.POINTER(de_input), INT, P, P, ctypes.POINTER(de_run_info)]),
    "de_gplmr_eig": (INT, [P, P, P, I64, I64, de_complex, INT, INT, INT, ctypes.c_double,
                           ctypes.POINTER(de_gmres), INT, ctypes.POINTER(de_stats)]),
    "de_gplmr_eig_d": (INT, [P, P, P, I64, I64, de_complex, INT, INT, INT, ctypes.c_double,
                             ctypes.POINTER(de_gmres), INT, ctypes.POINTER(de_stats)]),
    "de_input_default": (None, [ctypes.POINTER(de_input)]),
    "de_read_input": (INT, [ctypes.c_char_p, INT, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(de_input)]),
    "de_input_file_arg": (INT, [INT, ctypes.POINTER(ctypes.c_char_p), ctypes.c_char_p, ctypes.c_size_t]),
    "de_write_vectors": (INT, [ctypes.c_char_p, I64, INT, P]),
    "de_read_vectors": (INT, [ctypes.c_char_p, I64, INT, P]),
    "de_vectors_header": (INT, [ctypes.c_char_p, ctypes.POINTER(I64), ctypes.POINTER(INT)]),
    "de_request_footprint": (INT, [ctypes.POINTER(de_request), ctypes.POINTER(I64)]),
    "de_server_create": (INT, [ctypes.POINTER(de_server_opts), ctypes.POINTER(P)]),
    "de_server_submit": (INT, [P, ctypes.POINTER(de_request), ctypes.POINTER(ctypes.c_uint64)]),
    "de_server_wait": (INT, [P, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(de_result)]),
    "de_server_wait_any": (INT, [P, ctypes.c_double, ctypes.POINTER(de_result)]),
    "de_server_now": (ctypes.c_double, [P]),
    "de_server_load": (INT, [P, ctypes.POINTER(INT), ctypes.POINTER(INT), ctypes.POINTER(I64)]),
    "de_server_destroy": (INT, [P]),
    "de_problem_trim": (INT, [P]),
    "de_set_matvec_kernel": (INT, [P, INT]),
    "de_set_matvec_launch": (INT, [P, INT, INT, INT, INT]),
    "de_get_matvec_launch": (INT, [P, INT, INT, P, P]),
    "de_tuning_lookup": (INT, [ctypes.c_char_p, INT, INT, INT, P, P]),
    "de_kinetic_precond_d": (INT, [P, P, P, INT, de_complex]),
    "de_set_gmres_pc": (INT, [P, INT]),
}

_LIB = None


def lib_path() -> str:
    return os.path.join(_HERE, LIB_NAME)


def lib() -> ctypes.CDLL:
    """Load the in-tree library; raises if it has not been built."""
    global _LIB
    if _LIB is None:
        path = lib_path()
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`"
                              " or `make -C doublyexcited_b200/csrc`")
        L = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def check(status: int, where: str) -> None:
    if status != DE_OK:
        msg = lib().de_last_error()
        raise DeError(status, where, msg.decode() if msg else "")
