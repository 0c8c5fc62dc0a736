"""ctypes binding of the C ABI in include/torchannel_b200.h.

Loads the in-tree ``_tc_b200.so`` (built by ``torchannel_b200.build``).  There
is no fallback: if the library is missing or fails to load, import raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# TORCHANNEL_B200_LIB selects another build of the library (the
# bounds-checked _tc_b200_check.so); default: the in-tree _tc_b200.so
LIB_PATH = os.environ.get("TORCHANNEL_B200_LIB") or os.path.join(HERE, "_tc_b200.so")
CHECKED_LIB_PATH = os.path.join(HERE, "_tc_b200_check.so")

TC_OK, TC_ERR_ARG, TC_ERR_SIZE, TC_ERR_CUDA, TC_ERR_WORKSPACE, TC_ERR_STATE, TC_ERR_NONFINITE = range(7)
TC_FP64, TC_MIXED = 0, 1
TC_TOP_NOSLIP, TC_TOP_FREESLIP = 0, 1
TC_RHS_SEPARATE, TC_RHS_FUSED = 0, 1
TC_IMEX, TC_AB2, TC_FE = 0, 1, 2
PHASES = ["rhs", "cn", "fftx", "ffty", "tri", "iffty", "ifftx", "proj", "fin"]

_dp = ctypes.POINTER(ctypes.c_double)


class GridDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("Lx", ctypes.c_double), ("Ly", ctypes.c_double), ("Lz", ctypes.c_double),
                ("nu", ctypes.c_double), ("U_bulk", ctypes.c_double),
                ("top_wall", ctypes.c_int), ("precision", ctypes.c_int), ("rhs_path", ctypes.c_int),
                ("dz_f", _dp), ("dz_c", _dp)]


# (name, restype, argtypes) for every entry point declared in the header
_V = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
SIGNATURES = [
    ("tc_version", ctypes.c_char_p, []),
    ("tc_last_error", ctypes.c_char_p, []),
    ("tc_workspace_bytes", _I, [ctypes.POINTER(GridDesc), ctypes.POINTER(ctypes.c_size_t)]),
    ("tc_create", _I, [ctypes.POINTER(GridDesc), _V, ctypes.c_size_t, ctypes.POINTER(_V)]),
    ("tc_destroy", _I, [_V]),
    ("tc_set_state", _I, [_V, _V, _V, _V, _D, _V]),
    ("tc_get_state", _I, [_V, _V, _V, _V, _V, _V]),
    ("tc_get_history", _I, [_V, _V, _V, _V, _V]),
    ("tc_set_history", _I, [_V, _V, _V, _V, _V]),
    ("tc_step", _I, [_V, _I, _D, _I, _V]),
    ("tc_use_graphs", _I, [_V, _I]),
    ("tc_use_fused_poisson", _I, [_V, _I]),
    ("tc_use_fp32_poisson", _I, [_V, _I, _I]),
    ("tc_use_tma_rhs", _I, [_V, _I]),
    ("tc_use_bulk_ffty", _I, [_V, _I]),
    ("tc_bounds_error", _I, [ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    ("tc_project_initial", _I, [_V, _V]),
    ("tc_scalars", _I, [_V, ctypes.POINTER(_V)]),
    ("tc_set_forcing", _I, [_V, _D, _V]),
    ("tc_bulk_velocity", _I, [_V, _dp, _V]),
    ("tc_cfl", _I, [_V, _dp, _V]),
    ("tc_diagnostics", _I, [_V, _dp, _V]),
    ("tc_divergence", _I, [_V, _V, _V]),
    ("tc_explicit_rhs", _I, [_V, _I, _V, _V, _V, _V]),
    ("tc_implicit_diffusion", _I, [_V, _D, _V]),
    ("tc_poisson_solve", _I, [_V, _V, _V, _V]),
    ("tc_poisson_solve_noalloc", _I, [_I, _I, _I, _D, _D, _V, _V, _V, _V, _V]),
    ("tc_project", _I, [_V, _V, _D, _V]),
    ("tc_stats_init", _I, [_V, _dp, _D, _D, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    ("tc_stats_accumulate", _I, [_V, _V]),
    ("tc_stats_read", _I, [_V, _dp, _dp, ctypes.POINTER(_I)]),
    ("tc_stats_write", _I, [_V, _dp, _dp, _I]),
    ("tc_timing_enable", _I, [_V, _I]),
    ("tc_timing_read", _I, [_V, _dp, ctypes.POINTER(_I)]),
    ("tc_error", _I, [_V, ctypes.POINTER(_I)]),
    ("tc_adjoint_scratch_bytes", _I, [_V, ctypes.POINTER(ctypes.c_size_t)]),
    ("tc_set_body_force", _I, [_V, _V, _V, _V]),
    ("tc_internal_doubles", _I, [_V, ctypes.POINTER(ctypes.c_size_t)]),
    ("tc_save_internal", _I, [_V, _V, ctypes.POINTER(_I), _V]),
    ("tc_load_internal", _I, [_V, _V, _I, _V]),
    ("tc_kinetic_energy", _I, [_V, _D, _V, _V, _V]),
    ("tc_adjoint_ke_seed", _I, [_V, _D, _V, _V, _V, _V, _V, _V, _V]),
    ("tc_adjoint_rhs", _I, [_V, _V, _V, _V, _V, _V, _V, _V, _V, _V, _V]),
    ("tc_adjoint_cn", _I, [_V, _D, _V, _V, _V, _V, _V]),
    ("tc_adjoint_project", _I, [_V, _V, _V, _V, _V, _V]),
    ("tc_adjoint_step", _I, [_V, _D, _I] + [_V] * 15),
    ("tc_set_ke_accumulator", _I, [_V, _V, _V, _V]),
    ("tc_set_state_tape", _I, [_V, _V, _I, _V]),
    ("tc_set_cn_chunk", _I, [_V, _I]),
    ("tc_batch_table_bytes", _I, [_I, _I, ctypes.POINTER(ctypes.c_size_t)]),
    ("tc_batch_create", _I, [ctypes.POINTER(_V), _I, _V, ctypes.c_size_t, ctypes.POINTER(_V)]),
    ("tc_batch_destroy", _I, [_V]),
    ("tc_batch_set_shape", _I, [_V, _I, _I]),
    ("tc_batch_use_graphs", _I, [_V, _I]),
    ("tc_batch_step", _I, [_V, _I, _dp, _I, _V]),
    ("tc_batch_info", _I, [_V, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)]),
]


def load(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(f"torchannel_b200 CUDA library not built: {path} (run python -m torchannel_b200.build)")
    lib = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = load()
    return _lib


class TCError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"torchannel_b200 error {code}: {msg}")
        self.code = code


def check(rc):
    if rc != TC_OK:
        raise TCError(rc, lib().tc_last_error().decode())
    return rc
