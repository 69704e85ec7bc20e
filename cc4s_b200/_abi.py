"""ctypes binding of include/cc4s_cc.h (the library's C ABI)."""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIB = os.path.join(HERE, "libcc4s_b200.so")
MAX_HISTORY = 256

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_BAD_SHAPE = 2
ERR_OUT_OF_MEMORY = 3
WARN_NOT_CONVERGED = 4
ERR_DIIS_SINGULAR = 5
ERR_CUDA = 6
ERR_TIMEOUT = 7
ERR_STATE = 8
ERR_NON_FINITE = 9
ERR_UNSUPPORTED = 10

METHODS = {"Ccsd": 0, "Ccd": 1, "Drccd": 2}
PRECISIONS = {"fp64": 0, "split2": 2, "split3": 3}
MIXERS = {"DiisMixer": 0, "LinearMixer": 1}

# Every symbol the header declares.
EXPORTS = [
    "cc4s_cc_default_options", "cc4s_cc_create", "cc4s_cc_set_inputs",
    "cc4s_cc_set_initial_amplitudes", "cc4s_cc_run", "cc4s_cc_get_amplitudes",
    "cc4s_cc_residual", "cc4s_cc_backward", "cc4s_cc_residual_vjp", "cc4s_cc_relaxed_gradient",
    "cc4s_cc_triples_default_options", "cc4s_cc_perturbative_triples",
    "cc4s_cc_fsc_default_options", "cc4s_cc_finite_size_correction", "cc4s_cc_get_stats", "cc4s_cc_energy_noalloc", "cc4s_cc_destroy",
    "cc4s_cc_last_error",
]


class Options(ctypes.Structure):
    _fields_ = [
        ("method", ctypes.c_int), ("precision", ctypes.c_int), ("mixer", ctypes.c_int),
        ("max_residua", ctypes.c_int), ("ratio", ctypes.c_double),
        ("max_iterations", ctypes.c_int), ("energy_convergence", ctypes.c_double),
        ("amplitudes_convergence", ctypes.c_double), ("level_shift", ctypes.c_double),
        ("integrals_slice_size", ctypes.c_int64), ("ppl", ctypes.c_int), ("device", ctypes.c_int),
        ("profile", ctypes.c_int), ("linearized", ctypes.c_int),
        ("adjacent_pairs_exchange", ctypes.c_int), ("precision_refinement", ctypes.c_double),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("correlation", ctypes.c_double), ("direct", ctypes.c_double),
        ("exchange", ctypes.c_double), ("second_order", ctypes.c_double),
        ("correlation_imag", ctypes.c_double),
        ("iterations", ctypes.c_int), ("converged", ctypes.c_int), ("history_len", ctypes.c_int),
        ("energy", ctypes.c_double * MAX_HISTORY), ("delta_energy", ctypes.c_double * MAX_HISTORY),
        ("residuum_norm", ctypes.c_double * MAX_HISTORY), ("seconds", ctypes.c_double * MAX_HISTORY),
        ("flops_per_iteration", ctypes.c_double), ("refined_from", ctypes.c_int),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("gemm_launches", ctypes.c_uint64), ("other_launches", ctypes.c_uint64),
        ("device_bytes", ctypes.c_uint64), ("flops_per_residual", ctypes.c_double),
        ("gemm_seconds", ctypes.c_double), ("gemm_flops", ctypes.c_double),
        ("top_seconds", ctypes.c_double), ("top_flops", ctypes.c_double),
        ("gemm_profiled_launches", ctypes.c_int),
        ("split_seconds", ctypes.c_double), ("split_flops", ctypes.c_double),
        ("split_launches", ctypes.c_int),
    ]


class LambdaResult(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int), ("converged", ctypes.c_int),
        ("residuum_norm", ctypes.c_double), ("prepare_seconds", ctypes.c_double),
        ("vjp_seconds", ctypes.c_double), ("gradient_seconds", ctypes.c_double),
    ]


class TriplesOptions(ctypes.Structure):
    _fields_ = [("block_size", ctypes.c_int64), ("formulation", ctypes.c_int),
                ("cT", ctypes.c_int)]


class TriplesResult(ctypes.Structure):
    _fields_ = [
        ("correlation", ctypes.c_double), ("seconds", ctypes.c_double),
        ("setup_seconds", ctypes.c_double), ("flops", ctypes.c_double),
        ("executed_flops", ctypes.c_double), ("block_size", ctypes.c_int64),
        ("block_triples", ctypes.c_int64), ("phase_seconds", ctypes.c_double * 4),
        ("mp2_energy", ctypes.c_double), ("cr_denominator", ctypes.c_double),
    ]


class FscOptions(ctypes.Structure):
    _fields_ = [("interpolation_grid_size", ctypes.c_int), ("unit_factor", ctypes.c_double)]


class FscResult(ctypes.Structure):
    _fields_ = [
        ("correction", ctypes.c_double), ("uncorrected", ctypes.c_double),
        ("corrected", ctypes.c_double), ("seconds", ctypes.c_double),
        ("box", ctypes.c_int64 * 3),
    ]


_LIBS = {}


def load(path=None):
    """Loads the C-ABI library (the in-tree build unless `path` names another
    build of the same ABI).  Raises if it is missing: there is no fallback."""
    path = os.path.abspath(path or DEFAULT_LIB)
    if path in _LIBS:
        return _LIBS[path]
    if not os.path.exists(path):
        raise RuntimeError(
            "cc4s_b200 CUDA library not found at %s; build it with "
            "`python -m cc4s_b200.build` (there is no CPU fallback)" % path)
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    dp = P(ctypes.c_double)
    lib.cc4s_cc_default_options.argtypes = [P(Options)]
    lib.cc4s_cc_default_options.restype = None
    lib.cc4s_cc_create.argtypes = [P(Options), P(ctypes.c_void_p)]
    lib.cc4s_cc_set_inputs.argtypes = [ctypes.c_void_p, dp, ctypes.c_int64, dp, ctypes.c_int64,
                                       dp, ctypes.c_int64, ctypes.c_int, ctypes.c_int]
    lib.cc4s_cc_set_initial_amplitudes.argtypes = [ctypes.c_void_p, dp, dp]
    lib.cc4s_cc_run.argtypes = [ctypes.c_void_p, P(Result)]
    lib.cc4s_cc_get_amplitudes.argtypes = [ctypes.c_void_p, dp, dp]
    lib.cc4s_cc_residual.argtypes = [ctypes.c_void_p, dp, dp, dp, dp]
    lib.cc4s_cc_get_stats.argtypes = [ctypes.c_void_p, P(Stats)]
    lib.cc4s_cc_backward.argtypes = [ctypes.c_void_p, dp, dp]
    lib.cc4s_cc_residual_vjp.argtypes = [ctypes.c_void_p, dp, dp, dp, dp, dp, dp, dp]
    lib.cc4s_cc_relaxed_gradient.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, dp,
                                             P(LambdaResult)]
    lib.cc4s_cc_triples_default_options.argtypes = [P(TriplesOptions)]
    lib.cc4s_cc_perturbative_triples.argtypes = [ctypes.c_void_p, P(TriplesOptions),
                                                 P(TriplesResult)]
    lib.cc4s_cc_fsc_default_options.argtypes = [P(FscOptions)]
    lib.cc4s_cc_finite_size_correction.argtypes = [ctypes.c_void_p, dp, ctypes.c_int64, dp, dp, dp,
                                                   P(FscOptions), dp, P(FscResult)]
    lib.cc4s_cc_energy_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                           ctypes.c_void_p, ctypes.c_void_p]
    lib.cc4s_cc_destroy.argtypes = [ctypes.c_void_p]
    lib.cc4s_cc_last_error.argtypes = [ctypes.c_void_p]
    lib.cc4s_cc_last_error.restype = ctypes.c_char_p
    for name in EXPORTS[1:-1]:
        getattr(lib, name).restype = ctypes.c_int
    lib.cc4s_cc_triples_default_options.restype = None
    lib.cc4s_cc_fsc_default_options.restype = None
    _LIBS[path] = lib
    return lib


def ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def as_f64(a):
    """Contiguous float64 buffer in the reference's column-major layout."""
    a = np.asarray(a)
    if np.iscomplexobj(a):
        a = np.asfortranarray(a, dtype=np.complex128)
        return a.reshape(-1, order="F").view(np.float64)
    return np.asfortranarray(a, dtype=np.float64).reshape(-1, order="F")
