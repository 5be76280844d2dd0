"""ctypes binding of libfdcuda.so (include/fdcuda.h, include/fdhost.h).

The library is built in-tree (fractodactyl_b200/build.py). Loading fails loudly when it
is missing: there is no CPU stand-in for the CUDA route.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfdcuda.so")

# fdc_status
OK, DECLINED, INVALID, DEVICE_ERROR, TIMEOUT, NO_DEVICE = range(6)
STATUS_NAMES = {0: "OK", 1: "DECLINED", 2: "INVALID", 3: "DEVICE_ERROR", 4: "TIMEOUT", 5: "NO_DEVICE"}
# fdc_job flags
DERIVATIVE, BLA, SHIFT, F32, DEVICE_OUT, SERIES = 1, 2, 4, 8, 16, 32


class Job(C.Structure):
    _fields_ = [
        ("orbit", C.c_int32),
        ("tier", C.c_int32),
        ("nx", C.c_uint32),
        ("ny", C.c_uint32),
        ("ss", C.c_uint32),
        ("flags", C.c_uint32),
        ("c_re", C.c_double),
        ("c_im", C.c_double),
        ("h_m", C.c_double),
        ("h_e", C.c_int64),
        ("cos_rot", C.c_double),
        ("sin_rot", C.c_double),
        ("max_iter", C.c_uint64),
        ("escape_radius", C.c_double),
        ("nucleus_period", C.c_int64),
        ("mask", C.c_void_p),
        ("offsets", C.c_void_p),
        ("first_row", C.c_uint32),
        ("rows", C.c_uint32),
        ("deadline_ms", C.c_double),
        ("first_col", C.c_uint32),
        ("cols", C.c_uint32),
    ]


class SeriesInfo(C.Structure):  # fdh_series (include/fdhost.h)
    _fields_ = [
        ("n", C.c_uint64),
        ("points", C.c_uint64),
        ("built_steps", C.c_uint64),
        ("coefficient_pairs", C.c_uint64),
        ("order", C.c_uint32),
        ("growth_count", C.c_uint32),
        ("rho", C.c_double),
        ("state_bound", C.c_double),
        ("derivative_bound", C.c_double),
        ("shift_px", C.c_double),
        ("stop", C.c_char * 16),
    ]


class BoundOut(C.Structure):  # fdc_bound_out
    _fields_ = [("bound", C.c_void_p), ("ez", C.c_void_p), ("ed", C.c_void_p)]


class Stripe(C.Structure):  # fdc_stripe
    _fields_ = [("window", C.c_uint32), ("freq", C.c_double)]


class Out(C.Structure):
    _fields_ = [(name, C.c_void_p) for name in ("cls", "n", "nu", "de", "normal", "z", "dz", "dexp", "status")]


class Counters(C.Structure):
    _fields_ = [
        ("samples", C.c_uint64),
        ("iterations", C.c_uint64),
        ("blocks", C.c_uint64),
        ("skipped", C.c_uint64),
        ("fallback_samples", C.c_uint64),
        ("closed_form_samples", C.c_uint64),
        ("shift", C.c_double),
        ("kernel_ms", C.c_double),
        ("launches", C.c_uint32),
    ]


class Plane(C.Structure):
    _fields_ = [
        ("c_re", C.c_double),
        ("c_im", C.c_double),
        ("h_m", C.c_double),
        ("h_e", C.c_int64),
        ("tier", C.c_int32),
        ("bits", C.c_uint64),
        ("cos_rot", C.c_double),
        ("sin_rot", C.c_double),
    ]


class Tuning(C.Structure):
    _fields_ = [("defer", C.c_uint32), ("blocks_per_sm", C.c_uint32), ("tile_w", C.c_uint32), ("order", C.c_uint32)]


ORDER_ROWS, ORDER_CENTRE = 1, 2  # FDC_ORDER_*


DEFAULT_DEFER = 0  # FDC_DEFAULT_DEFER: each kernel variant's measured default

# Every symbol the headers declare, for the export check.
FDC_SYMBOLS = ["fdc_abi_version", "fdc_open", "fdc_close", "fdc_last_error", "fdc_upload_orbit", "fdc_free_orbit",
               "fdc_upload_bla", "fdc_build_bla", "fdc_upload_series", "fdc_upload_error_radius", "fdc_render_bounded", "fdc_render_stripe", "fdc_render", "fdc_batch_create", "fdc_batch_run", "fdc_batch_free",
               "fdc_render_noalloc", "fdc_set_tuning", "fdc_get_tuning"]
FDH_SYMBOLS = ["fdh_last_error", "fdh_plane_new", "fdh_orbit_fixed", "fdh_orbit_fixed_threads", "fdh_orbit_f64",
               "fdh_nucleus_period",
               "fdh_bla_build", "fdh_bla_build_into", "fdh_guarded_bla_build", "fdh_external_escape_ok", "fdh_series_build", "fdh_error_radius", "fdh_dc_bound", "fdh_encode", "fdh_location"]

_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            "libfdcuda.so is not built (run `python -m fractodactyl_b200.build`); the CUDA route has no fallback")
    L = C.CDLL(LIB_PATH)
    P, D, U32, U64, I32, I64 = C.c_void_p, C.c_double, C.c_uint32, C.c_uint64, C.c_int32, C.c_int64
    L.fdc_abi_version.restype = C.c_int
    L.fdc_open.argtypes = [C.c_int, C.POINTER(P)]
    L.fdc_close.argtypes = [P]
    L.fdc_last_error.restype = C.c_char_p
    L.fdc_last_error.argtypes = [P]
    L.fdc_upload_orbit.argtypes = [P, P, P, U64, U32, C.POINTER(I32)]
    L.fdc_free_orbit.argtypes = [P, I32]
    L.fdc_upload_bla.argtypes = [P, I32, P, P, U32, D, D, I64]
    L.fdc_build_bla.argtypes = [P, I32, D, D, I64, C.POINTER(U32), P]
    L.fdc_upload_series.argtypes = [P, I32, U64, U64, D, P, U32]
    L.fdc_render.argtypes = [P, C.POINTER(Job), C.POINTER(Out), C.POINTER(Counters)]
    L.fdc_render_bounded.argtypes = [P, C.POINTER(Job), C.POINTER(Out), C.POINTER(BoundOut), C.POINTER(Counters)]
    L.fdc_render_stripe.argtypes = [P, C.POINTER(Job), C.POINTER(Out), C.POINTER(Stripe), P, C.POINTER(Counters)]
    L.fdc_upload_error_radius.argtypes = [P, I32, P, U64]
    L.fdc_batch_create.argtypes = [P, P, P, U32, C.POINTER(P)]
    L.fdc_batch_run.argtypes = [P, P, C.POINTER(Counters), P]
    L.fdc_batch_free.argtypes = [P, P]
    L.fdc_set_tuning.argtypes = [P, C.POINTER(Tuning)]
    L.fdc_get_tuning.argtypes = [P, C.POINTER(Tuning)]
    L.fdc_render_noalloc.argtypes = [C.c_int, P, U64, C.POINTER(Job), C.POINTER(Out), P, C.POINTER(Counters), P,
                                     C.c_char_p, C.c_size_t]
    L.fdh_last_error.restype = C.c_char_p
    L.fdh_plane_new.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, D, U32, U32, C.POINTER(Plane)]
    L.fdh_orbit_fixed.restype = I64
    L.fdh_orbit_fixed.argtypes = [C.c_char_p, C.c_char_p, U64, U64, P, P, U64]
    L.fdh_orbit_fixed_threads.restype = I64
    L.fdh_orbit_fixed_threads.argtypes = [C.c_char_p, C.c_char_p, U64, U64, P, P, U64, C.c_int]
    L.fdh_orbit_f64.restype = I64
    L.fdh_orbit_f64.argtypes = [D, D, U64, D, P, P, U64]
    L.fdh_nucleus_period.restype = I64
    L.fdh_nucleus_period.argtypes = [P, P, U64]
    L.fdh_bla_build.argtypes = [P, P, U64, D, D, I64, C.c_int, P, P, C.POINTER(U32), C.POINTER(U64)]
    L.fdh_error_radius.restype = C.c_int
    L.fdh_error_radius.argtypes = [P, P, U64, I64, D, D, P]
    L.fdh_series_build.restype = C.c_int
    L.fdh_series_build.argtypes = [P, P, U64, D, D, U64, U64, C.POINTER(SeriesInfo), P, U32]
    L.fdh_bla_build_into.restype = C.c_int
    L.fdh_bla_build_into.argtypes = [P, P, U64, D, D, I64, C.c_int, P, U64, P, U32, C.POINTER(U32), C.POINTER(U64)]
    L.fdh_guarded_bla_build.restype = C.c_int
    L.fdh_guarded_bla_build.argtypes = [P, P, P, U64, D, D, P, U64, P, U32, C.POINTER(U32), C.POINTER(U64)]
    L.fdh_external_escape_ok.restype = C.c_int
    L.fdh_external_escape_ok.argtypes = [U64, D, D, D, D, I64, D, D, D, I64]
    L.fdh_encode.argtypes = [C.POINTER(Plane), U32, U64, P, P, P, P, P, P, P, P, C.c_int]
    L.fdh_dc_bound.argtypes = [C.POINTER(Plane), I32, U32, U32, C.POINTER(D), C.POINTER(I64)]
    L.fdh_location.argtypes = [C.c_char_p, C.c_char_p, D, D, U64, U64, C.c_char_p, C.c_char_p, C.c_size_t,
                               C.POINTER(U64), C.POINTER(D)]
    _lib = L
    return L


def host_error():
    return lib().fdh_last_error().decode()
