"""ctypes binding of libwmles_cuda.so (declarations in include/wmles_cuda.h).

The library is loaded from this package directory (built by ``python -m
wmles_jax_b200.build``).  There is no fallback: a missing or stale library raises.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwmles_cuda.so")
ABI_VERSION = 1
MAX_BLOCKS = 96

c_int_p = C.POINTER(C.c_int)
c_double_p = C.POINTER(C.c_double)


class WmGas(C.Structure):
    _fields_ = [("gamma", C.c_double), ("R", C.c_double), ("Pr", C.c_double), ("Pr_t", C.c_double),
                ("mu_ref", C.c_double), ("T_ref", C.c_double), ("S_suth", C.c_double)]


class WmBlock(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("ng", C.c_int), ("metrics", c_double_p)]


class WmWall(C.Structure):
    _fields_ = [("block", C.c_int), ("axis", C.c_int), ("side", C.c_int), ("n_match", C.c_int),
                ("isothermal", C.c_int), ("T_wall", C.c_double), ("kappa", C.c_double), ("B", C.c_double),
                ("n_iter", C.c_int), ("geom", c_double_p)]


class WmGhostProgram(C.Structure):
    _fields_ = [("count", C.c_int), ("dst", c_int_p), ("src", c_int_p), ("ops", c_int_p),
                ("nops", C.c_int), ("op_code", c_int_p), ("op_nrm", c_double_p)]


class WmInflow(C.Structure):
    _fields_ = [("block", C.c_int), ("n_modes", C.c_int), ("n_tab", C.c_int), ("modes", c_double_p),
                ("table", c_double_p), ("U_inf", C.c_double), ("L", C.c_double), ("rho_inf", C.c_double),
                ("p_inf", C.c_double)]


class WmSponge(C.Structure):
    _fields_ = [("enabled", C.c_int), ("x_start_l", C.c_double), ("x_end_l", C.c_double),
                ("strength", C.c_double), ("U_inf", C.c_double), ("L", C.c_double)]


class WmCaseDesc(C.Structure):
    _fields_ = [("gas", WmGas), ("scheme", C.c_int), ("kep_order", C.c_int), ("limiter", C.c_int),
                ("th0", C.c_double), ("th1", C.c_double), ("sgs", C.c_int), ("sgs_coeff", C.c_double),
                ("cfl", C.c_double), ("precision", C.c_int), ("cmf_dir", C.c_int), ("cmf_target", C.c_double),
                ("cmf_volume", C.c_double), ("nblocks", C.c_int), ("blocks", C.POINTER(WmBlock)),
                ("nwalls", C.c_int), ("walls", C.POINTER(WmWall)), ("nbc", C.c_int), ("bc_table", c_double_p),
                ("ghost_rhs", WmGhostProgram), ("ghost_all", WmGhostProgram), ("inflow", C.POINTER(WmInflow)),
                ("sponge", WmSponge), ("tile", C.c_int), ("chunk", C.c_int)]


PP = C.POINTER(c_double_p)

# entry point -> (restype, argtypes); exactly the functions declared in include/wmles_cuda.h
SIGNATURES = {
    "wm_version": (C.c_int, []),
    "wm_last_error": (C.c_char_p, []),
    "wm_case_create": (C.c_int, [C.POINTER(WmCaseDesc), C.POINTER(C.c_void_p)]),
    "wm_case_destroy": (None, [C.c_void_p]),
    "wm_apply_bcs": (C.c_int, [C.c_void_p, PP, C.c_double, C.c_void_p]),
    "wm_rhs": (C.c_int, [C.c_void_p, PP, PP, C.c_double, C.c_void_p]),
    "wm_max_dt": (C.c_int, [C.c_void_p, PP, c_double_p, C.c_void_p]),
    "wm_advance": (C.c_int, [C.c_void_p, PP, PP, c_double_p, C.c_double, C.c_void_p]),
    "wm_step": (C.c_int, [C.c_void_p, PP, PP, c_double_p, C.c_double, C.c_void_p]),
    "wm_step_fused": (C.c_int, [C.c_void_p, PP, PP, c_double_p, c_double_p, C.c_double, C.c_void_p]),
    "wm_max_dt_noalloc": (C.c_int, [C.c_int, c_int_p, PP, PP, C.POINTER(WmGas), C.c_double, c_double_p,
                                    C.c_void_p]),
    "wm_case_status": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint), C.c_int, C.c_void_p]),
    "wm_check": (C.c_int, [C.c_void_p, C.c_void_p]),
    "wm_wall_stats": (C.c_int, [C.c_void_p, PP, PP, C.c_void_p]),
    "wm_plane_stats": (C.c_int, [C.c_void_p, C.c_int, c_double_p, c_double_p, C.c_void_p]),
    "wm_derived_fields": (C.c_int, [C.c_void_p, PP, PP, C.c_void_p]),
    "wm_block_geometry": (C.c_int, [c_double_p, c_int_p, c_double_p, c_double_p, PP, PP, c_double_p,
                                    C.c_void_p]),
    "wm_batch_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "wm_batch_destroy": (None, [C.c_void_p]),
    "wm_batch_step": (C.c_int, [C.c_void_p, PP, PP, PP, PP, c_double_p, C.c_void_p]),
    "wm_batch_status": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "wm_batch_info": (C.c_int, [C.c_void_p, c_int_p, c_int_p, C.POINTER(C.c_longlong)]),
    "wm_profile_enable": (C.c_int, [C.c_void_p, C.c_int]),
    "wm_profile_read": (C.c_int, [C.c_void_p, C.c_int, c_double_p, C.POINTER(C.c_longlong)]),
}
KIND_STAGE, KIND_GHOST, KIND_WALL, KIND_DT, KIND_SOURCE = range(5)
# case status bits (WM_ST_*)
ST_NONFINITE, ST_RHO, ST_PRESSURE, ST_DT, ST_WALL = 1, 2, 4, 8, 16
ST_FATAL = ST_NONFINITE | ST_RHO | ST_PRESSURE | ST_DT
ST_NAMES = {ST_NONFINITE: "non-finite state", ST_RHO: "non-positive density", ST_PRESSURE: "non-positive pressure",
            ST_DT: "non-finite or non-positive time step", ST_WALL: "wall-model Newton not settled"}


def status_names(bits):
    """Names of the WM_ST_* bits set in ``bits``."""
    return [name for bit, name in ST_NAMES.items() if bits & bit]


class NonFiniteStateError(RuntimeError):
    """A case's state stopped being a flow state (a WM_ST_FATAL bit of its status word)."""
NDERIVED = 11

_lib = None


def load(path=LIB_PATH):
    """Load the library (once) and bind the signatures; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libwmles_cuda.so not found at {path}: build it with "
                           f"`python -m wmles_jax_b200.build` (the cuda backend has no fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    v = lib.wm_version()
    if v != ABI_VERSION:
        raise RuntimeError(f"libwmles_cuda.so ABI version {v}, expected {ABI_VERSION}: rebuild it")
    _lib = lib
    return lib


def check(status, what):
    if status != 0:
        msg = _lib.wm_last_error().decode(errors="replace") if _lib is not None else ""
        exc = ValueError if status in (-1, -4) else NonFiniteStateError if status == -3 else RuntimeError
        raise exc(f"{what} failed (status {status}): {msg}")


def ptr_array(ptrs):
    """(double*)[] from integer device addresses."""
    arr = (c_double_p * len(ptrs))()
    for i, p in enumerate(ptrs):
        arr[i] = C.cast(C.c_void_p(int(p)), c_double_p)
    return arr


def as_int_p(a):
    return a.ctypes.data_as(c_int_p)


def as_double_p(a):
    return a.ctypes.data_as(c_double_p)
