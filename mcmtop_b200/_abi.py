"""ctypes view of include/mcm_gpu.h (the C ABI of libmcm_gpu.so).

The structures mirror the C declarations field for field.  Loading fails with
an exception when the library has not been built: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmcm_gpu.so")

MCM_OK = 0
MCM_ENBR_OVERFLOW = 1
MCM_EGHOST_OVERFLOW = 2
MCM_ECOMPLEX_C = 3
MCM_ECAP_NOCONV = 4
MCM_ETIMEOUT = 5
MCM_ECUDA = 6
MCM_ENOMEM = 7
MCM_EINVAL = 8
MCM_EUNSUPPORTED = 9
MCM_EGRID_OVERFLOW = 10
MCM_EGHOST_LAYER = 11
MCM_EGRID_TOO_LARGE = 12

PREC_FP64_EXACT = 0
PREC_FP64 = 1
PREC_MIXED = 2
MAX_MATERIALS = 16


class Material(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("eos", C.c_int), ("visc_type", C.c_int),
        ("rho", C.c_double), ("g", C.c_double), ("av_l", C.c_double), ("av_q", C.c_double),
        ("mass", C.c_double), ("h", C.c_double), ("rho_min", C.c_double), ("rho_max", C.c_double),
        ("strinput", C.c_double * 48), ("eosinput", C.c_double * 24),
        ("k_cont", C.c_double), ("n_cont", C.c_double),
    ]


class Config(C.Structure):
    _fields_ = [
        ("ndim", C.c_int), ("disctype", C.c_int), ("tcrit_opt", C.c_int), ("contacttype", C.c_int),
        ("h_opt", C.c_int), ("veloc_opt", C.c_int), ("krtype", C.c_int), ("drelax", C.c_int),
        ("drelax_scale", C.c_double), ("boundary", C.c_int), ("boundary_code", C.c_int * 6),
        ("boundary_x", C.c_double * 6), ("baseaccel", C.c_int), ("base_a", C.c_double * 3),
        ("tssf", C.c_double), ("hmax", C.c_double), ("precision", C.c_int), ("nbr_stride", C.c_int),
        ("reorder_interval", C.c_int), ("block_size", C.c_int), ("nbr_skin", C.c_double),
        ("compensated_sums", C.c_int),
    ]


_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)


class Fields(C.Structure):
    _fields_ = [
        ("x", _DP), ("v", _DP), ("a", _DP),
        ("mass", _DP), ("h", _DP), ("hold", _DP), ("rho", _DP), ("rhoold", _DP), ("e", _DP), ("p", _DP),
        ("c", _DP), ("vabs", _DP),
        ("efps", _DP), ("pcut", _DP), ("p_cut", _DP), ("fail", _DP), ("mindist", _DP), ("critts", _DP),
        ("tracerod", _DP),
        ("etry", _DP), ("einc", _DP), ("capa", _DP),
        ("sigma", _DP), ("s", _DP), ("q", _DP), ("qold", _DP), ("alfa", _DP), ("rod", _DP), ("spin", _DP),
        ("mat", _IP), ("dispbc", _IP), ("nnbr", _IP), ("g_nnbr", _IP), ("ptype", _IP),
        ("h0", _DP), ("repulsion", _DP),
    ]


class Time(C.Structure):
    _fields_ = [("dt", C.c_double), ("dtold", C.c_double), ("ptime", C.c_double), ("endtime", C.c_double)]


class Tuning(C.Structure):
    _fields_ = [("search_threads", C.c_int), ("pair_threads", C.c_int), ("pair_blocks_per_sm", C.c_int),
                ("nbr_stride", C.c_int), ("search_kind", C.c_int), ("pair_kind", C.c_int),
                ("adj_kind", C.c_int), ("ms_per_step", C.c_double)]


# per-particle width of every field in Fields (doubles or ints)
FIELD_WIDTH = {
    "x": 3, "v": 3, "a": 3, "repulsion": 3, "sigma": 9, "s": 9, "q": 9, "qold": 9, "alfa": 9, "rod": 9, "spin": 9,
}
DOUBLE_FIELDS = [f for f, t in Fields._fields_ if t is _DP]
INT_FIELDS = [f for f, t in Fields._fields_ if t is _IP]

_lib = None


def load() -> C.CDLL:
    """Loads libmcm_gpu.so; raises if it is missing (build it with mcmtop_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m mcmtop_b200.build` (no CPU fallback exists)")
    lib = C.CDLL(LIB_PATH)
    H = C.c_void_p
    sig = {
        "mcm_gpu_abi_version": ([], C.c_int),
        "mcm_gpu_set_device": ([C.c_int], C.c_int),
        "mcm_gpu_strerror": ([C.c_int], C.c_char_p),
        "mcm_gpu_last_error": ([H], C.c_char_p),
        "mcm_gpu_material_from_deck": ([C.POINTER(Material)], C.c_int),
        "mcm_gpu_create": ([C.POINTER(Config), C.POINTER(Material), C.c_int, C.c_int, C.POINTER(H)], C.c_int),
        "mcm_gpu_destroy": ([H], C.c_int),
        "mcm_gpu_upload": ([H, C.POINTER(Fields), _DP], C.c_int),
        "mcm_gpu_initialise": ([H, C.POINTER(Fields), C.c_int, C.c_int, C.c_int, C.c_double, C.POINTER(Time)], C.c_int),
        "mcm_gpu_download": ([H, C.POINTER(Fields)], C.c_int),
        "mcm_gpu_step_a": ([H, C.c_double, _DP], C.c_int),
        "mcm_gpu_step_b": ([H, _DP], C.c_int),
        "mcm_gpu_step_c": ([H, C.c_double, C.c_double, _DP], C.c_int),
        "mcm_gpu_run": ([H, C.c_int, C.POINTER(Time), _IP], C.c_int),
        "mcm_gpu_neighbours": ([H, _IP, _IP, _IP, _IP, _IP, _IP], C.c_int),
        "mcm_gpu_ghosts": ([H, _IP, _IP, _DP, _DP, C.c_int], C.c_int),
        "mcm_gpu_contacts": ([H, _IP, _IP, _IP, _IP, _IP, _IP], C.c_int),
        "mcm_gpu_contact_forces": ([H, _DP], C.c_int),
        "mcm_gpu_grid": ([H, _IP, _DP, _DP], C.c_int),
        "mcm_gpu_energies": ([H, _DP], C.c_int),
        "mcm_gpu_stats": ([H, _DP, _IP, _IP, _IP], C.c_int),
        "mcm_gpu_skin_builds": ([H, C.POINTER(C.c_longlong)], C.c_int),
        "mcm_gpu_set_diagnostics": ([H, C.c_int], C.c_int),
        "mcm_gpu_calctotale_noalloc": ([C.c_void_p] * 5 + [C.c_int, C.c_int, C.c_void_p, C.c_void_p], C.c_int),
        "mcm_gpu_profile": ([H, C.c_int], C.c_int),
        "mcm_gpu_profile_report": ([H, C.c_int, C.c_char_p, C.c_int, _DP, _IP], C.c_int),
        "mcm_gpu_kernel_launches": ([H], C.c_longlong),
        "mcm_gpu_timer": ([H, C.c_int, _DP], C.c_int),
        "mcm_gpu_adjoint_forward": ([H, C.c_int, _DP, C.c_int], C.c_int),
        "mcm_gpu_adjoint_backward": ([H, _DP, _DP, _DP, _DP, _DP], C.c_int),
        "mcm_gpu_set_tuning": ([H, C.POINTER(Tuning)], C.c_int),
        "mcm_gpu_get_tuning": ([H, C.POINTER(Tuning)], C.c_int),
        "mcm_gpu_autotune": ([H, C.c_int, C.POINTER(Tuning)], C.c_int),
        "mcm_gpu_batch_create": ([C.POINTER(H), C.c_int, C.c_int, C.POINTER(H)], C.c_int),
        "mcm_gpu_batch_run": ([H, C.c_int, C.POINTER(Time), _IP], C.c_int),
        "mcm_gpu_batch_autotune": ([H, C.c_int, _IP, _DP], C.c_int),
        "mcm_gpu_batch_destroy": ([H], C.c_int),
        "mcm_gpu_batch_adjoint_forward": ([H, C.c_int, C.POINTER(_DP), C.c_int], C.c_int),
        "mcm_gpu_batch_adjoint_backward": ([H, C.POINTER(_DP), C.POINTER(_DP), C.POINTER(_DP), C.POINTER(_DP),
                                            C.POINTER(_DP)], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    """Names declared in include/mcm_gpu.h (for the load/export test)."""
    import re

    hdr = os.path.join(_HERE, "..", "include", "mcm_gpu.h")
    with open(hdr) as fh:
        text = fh.read()
    return sorted(set(re.findall(r"\b(mcm_gpu_[a-z_]+)\s*\(", text)))


class MCMError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        lib = load()
        msg = lib.mcm_gpu_strerror(code).decode()
        super().__init__(f"{where}: {msg} (status {code}){': ' + detail if detail else ''}")


def check(code: int, where: str, handle=None) -> None:
    if code != MCM_OK:
        detail = ""
        if handle is not None:
            detail = load().mcm_gpu_last_error(handle).decode()
        raise MCMError(code, where, detail)
