"""ctypes bindings of the C ABI in include/nuosc_b200.h.

Loads the in-tree nuosc_b200/libnuosc_b200.so.  There is no fallback: if the
library is missing or fails to load, importing the package raises.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnuosc_b200.so")

OK, ERR_INVALID, ERR_CUDA, ERR_OOM, ERR_NUMERIC, ERR_TIMEOUT, ERR_UNSUPPORTED = range(7)
FP64, FP32 = 0, 1
REG_STAT, REG_RHS, REG_PRE, REG_COR = 0, 1, 2, 3
LAYOUT_COMPACT, LAYOUT_GHOSTED = 0, 1
KERNEL_AUTO, KERNEL_DIRECT, KERNEL_XMARCH, KERNEL_XTMA = 0, 1, 2, 3
FIELDS = ["ee", "mm", "emr", "emi", "bee", "bmm", "bemr", "bemi",
          "P1", "P2", "P3", "P1b", "P2b", "P3b", "dP", "dPb"]


class NuoscError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("nuosc error %d: %s" % (code, msg))
        self.code = code


class Params(C.Structure):
    _fields_ = [("px", C.c_int), ("pz", C.c_int), ("nv", C.c_int), ("nphi", C.c_int),
                ("gx", C.c_int), ("gz", C.c_int),
                ("x0", C.c_double), ("x1", C.c_double), ("z0", C.c_double), ("z1", C.c_double),
                ("dx", C.c_double), ("dz", C.c_double), ("cfl", C.c_double), ("ko", C.c_double),
                ("precision", C.c_int), ("device", C.c_int)]


class Geometry(C.Structure):
    _fields_ = [("nx", C.c_int), ("nz", C.c_int), ("nv", C.c_int), ("nv_stride", C.c_int),
                ("gx", C.c_int), ("gz", C.c_int), ("precision", C.c_int),
                ("dt", C.c_double), ("ds_L", C.c_double), ("phy_time", C.c_double),
                ("x0", C.c_double), ("x1", C.c_double), ("z0", C.c_double), ("z1", C.c_double),
                ("dx", C.c_double), ("dz", C.c_double), ("n_nue0", C.c_double * 2),
                ("device_bytes", C.c_size_t)]


class Halo(C.Structure):
    """nuosc_halo: the 32 halo pieces of one slab for one RK stage."""
    _fields_ = [("send_lo", C.c_void_p * 8), ("send_hi", C.c_void_p * 8), ("recv_lo", C.c_void_p * 8),
                ("recv_hi", C.c_void_p * 8), ("bytes", C.c_size_t), ("left", C.c_int), ("right", C.c_int)]


class Diag(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("phy_time", "maxdP", "surv", "survb", "avgP", "avgPb", "aM0", "Lex", "ELNe")] + \
               [("nonfinite", C.c_longlong), ("I1", C.c_double), ("I2", C.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class BatchInfo(C.Structure):
    _fields_ = [("n", C.c_int), ("tz", C.c_int), ("ctas", C.c_int), ("tiles", C.c_longlong),
                ("cells", C.c_longlong), ("cell_velocities", C.c_longlong), ("device_bytes", C.c_size_t),
                ("graph_launches", C.c_longlong), ("kernel_launches", C.c_longlong)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class BatchRecord(C.Structure):
    _fields_ = [("member", C.c_int), ("reserved", C.c_int), ("step", C.c_longlong), ("phy_time", C.c_double),
                ("q", C.c_double * 12)]


_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)

_SIGS = {
    "nuosc_velocity_quadrature": [_I, _DP, _DP, _DP, _DP, _IP],
    "nuosc_create": [C.POINTER(Params), C.POINTER(_P)],
    "nuosc_destroy": [_P],
    "nuosc_set_mu": [_P, _D],
    "nuosc_set_pmo": [_P, _D],
    "nuosc_set_renorm": [_P, _I],
    "nuosc_set_kernel": [_P, _I],
    "nuosc_set_tile": [_P, _I, _I],
    "nuosc_get_tile": [_P, _IP, _IP],
    "nuosc_set_time": [_P, _D],
    "nuosc_get_geometry": [_P, C.POINTER(Geometry)],
    "nuosc_get_velocities": [_P, _DP, _DP, _DP, _DP],
    "nuosc_get_spectra": [_P, _DP, _DP],
    "nuosc_set_spectra": [_P, _DP, _DP, _D, _D],
    "nuosc_fill_init": [_P, _I, _D, _D, _D, _D, _D, _D, _D, C.c_uint64],
    "nuosc_set_state": [_P, _I, _I, _DP, _I],
    "nuosc_get_state": [_P, _I, _I, _DP, _I],
    "nuosc_update_periodic_boundary": [_P, _I],
    "nuosc_calrhs": [_P, _I, _I],
    "nuosc_vectorize": [_P, _I, _I, _D, _I],
    "nuosc_vectorize2": [_P, _I, _I, _D, _I, _I],
    "nuosc_step_rk4": [_P, _I],
    "nuosc_analysis": [_P, C.POINTER(Diag)],
    "nuosc_open_analysis_file": [_P, C.c_char_p],
    "nuosc_add_snapshot_at_v": [_P, _IP, _I, C.c_char_p, _I, _IP, _I],
    "nuosc_add_snapshot_at_xv": [_P, _IP, _I, C.c_char_p, _I, _IP, _I, _IP, _I],
    "nuosc_check_snapshot": [_P, _I],
    "nuosc_gather": [_P, _I, _IP, _I, _IP, _I, _DP],
    "nuosc_synchronize": [_P],
    "nuosc_create_slab": [C.POINTER(Params), _I, C.POINTER(_P)],
    "nuosc_get_slab": [_P, _IP, _IP, _IP, _IP],
    "nuosc_stage": [_P, _I],
    "nuosc_halo_info": [_P, _I, C.POINTER(Halo)],
    "nuosc_halo_exchange_local": [C.POINTER(_P), _I, _I],
    "nuosc_analysis_sums": [_P, _DP],
    "nuosc_diag_from_sums": [_P, _DP, C.POINTER(Diag)],
    "nuosc_set_n_nue0": [_P, C.c_double, C.c_double],
    "nuosc_save_checkpoint": [_P, C.c_char_p],
    "nuosc_load_checkpoint": [_P, C.c_char_p],
    "nuosc_set_moment_sum": [_P, _I],
    "nuosc_get_moment_sum": [_P, _IP],
    "nuosc_moment_error": [_P, _DP],
    "nuosc_set_profiling": [_P, _I],
    "nuosc_get_profile": [_P, _DP, C.POINTER(C.c_longlong), _I],
    "nuosc_batch_create": [C.POINTER(_P), _I, C.POINTER(_P)],
    "nuosc_batch_step": [_P, _I],
    "nuosc_batch_synchronize": [_P],
    "nuosc_batch_get_info": [_P, C.POINTER(BatchInfo)],
    "nuosc_batch_destroy": [_P],
    "nuosc_batch_step_stream": [_P, _I, _I, _P, _I, _IP],
    "nuosc_batch_record_diag": [_P, C.POINTER(BatchRecord), C.POINTER(Diag)],
    "nuosc_batch_set_halt": [_P, _I],
    "nuosc_batch_halted": [_P, _IP, _I],
    "nuosc_release_cached_memory": [_I],
    "nuosc_selftest_wait_timeout": [_I, C.c_uint, C.POINTER(C.c_double)],
    "nuosc_selftest_overdeclare_tx": [_P, C.c_uint],
}
PROF_KINDS = ["stage_s1", "stage_s2", "stage_s4", "calrhs", "moments", "moment_finalize", "stage_s3"]

_lib = None


def lib():
    """The loaded C library (raises if the build is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("nuosc_b200: %s is missing; build it with `python nuosc_b200/build.py`" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.nuosc_last_error.restype = C.c_char_p
        L.nuosc_last_error.argtypes = []
        L.nuosc_stream.restype = _P
        L.nuosc_stream.argtypes = [_P]
        L.nuosc_kernel_launches.restype = C.c_longlong
        L.nuosc_kernel_launches.argtypes = [_P]
        L.nuosc_batch_stream.restype = _P
        L.nuosc_batch_stream.argtypes = [_P]
        L.nuosc_step_count.restype = C.c_longlong
        L.nuosc_step_count.argtypes = [_P]
        L.nuosc_host_alloc.restype = _P
        L.nuosc_host_alloc.argtypes = [C.c_size_t]
        L.nuosc_host_free.restype = None
        L.nuosc_host_free.argtypes = [_P]
        _lib = L
    return _lib


def check(rc):
    if rc != OK:
        raise NuoscError(rc, lib().nuosc_last_error().decode(errors="replace"))
    return rc
