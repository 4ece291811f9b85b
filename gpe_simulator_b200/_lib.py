"""ctypes binding of ``libgpe_ssf.so`` (the C ABI in ``include/gpe_ssf.h``).

There is no fallback: importing a compute entry point without the built
library raises ``RuntimeError``.
"""

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libgpe_ssf.so"

GPE_OK, GPE_ERR_ARG, GPE_ERR_UNSUPPORTED, GPE_ERR_CUDA, GPE_ERR_OOM, GPE_ERR_NONFINITE, GPE_ERR_TIMEOUT = range(7)
C64, C128 = 0, 1
IMAGINARY, REAL = 0, 1
V_NONE, V_REAL64, V_CPLX128 = 0, 1, 2

_dp = ctypes.POINTER(ctypes.c_double)
_llp = ctypes.POINTER(ctypes.c_longlong)
_vp = ctypes.c_void_p


class Desc(ctypes.Structure):
    """``gpe_desc`` (field order and types must match include/gpe_ssf.h)."""
    _fields_ = [
        ("n", ctypes.c_int), ("dtype", ctypes.c_int), ("kind", ctypes.c_int),
        ("beta", ctypes.c_double), ("dt", ctypes.c_double), ("kinetic_coeff", ctypes.c_double),
        ("x_array", _dp), ("k_array", _dp),
        ("static_x", _dp), ("static_x_len", ctypes.c_int),
        ("static_y", _dp), ("static_y_len", ctypes.c_int),
        ("static_z", _dp), ("static_z_len", ctypes.c_int),
        ("static_g", _dp), ("static_g_len", ctypes.c_int),
        ("dynamic_g", _dp), ("dynamic_g_len", ctypes.c_int),
        ("k_cut_enabled", ctypes.c_int), ("k_cut", ctypes.c_double),
        ("beam_enabled", ctypes.c_int),
        ("beam_amp", ctypes.c_double), ("beam_width", ctypes.c_double),
        ("beam_radius", ctypes.c_double), ("beam_omega", ctypes.c_double),
        ("beam_t_ramp", ctypes.c_double),
        ("nk_bins", ctypes.c_int),
        ("local_fp64", ctypes.c_int),
        ("generic_only", ctypes.c_int),
        ("exact_local", ctypes.c_int),
    ]


# name -> (argtypes)
SIGNATURES = {
    "gpe_version": [],
    "gpe_last_error": [ctypes.c_char_p, ctypes.c_size_t],
    "gpe_plan_create": [ctypes.POINTER(Desc), ctypes.POINTER(_vp)],
    "gpe_plan_destroy": [_vp],
    "gpe_plan_info": [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
    "gpe_set_static_potential": [_vp, _vp, ctypes.c_int, _vp],
    "gpe_step": [_vp, _vp, ctypes.c_int, ctypes.c_longlong, _vp],
    "gpe_step_at": [_vp, _vp, ctypes.c_double, _vp],
    "gpe_halfstep": [_vp, _vp, ctypes.c_double, _vp],
    "gpe_fft3d": [_vp, _vp, _vp, ctypes.c_int, _vp],
    "gpe_normalise": [_vp, _vp, _vp],
    "gpe_norm": [_vp, _vp, _dp, _vp],
    "gpe_kinetic_energy": [_vp, _vp, _dp, _vp],
    "gpe_nk_extraction": [_vp, _vp, _dp, _llp, _vp],
    "gpe_diagnostics": [_vp, _vp, ctypes.c_double, _dp, _dp, _llp, _vp],
    "gpe_status": [_vp, ctypes.POINTER(ctypes.c_int), _vp],
    "gpe_angular_momentum": [_vp, _vp, _dp, _vp],
    "gpe_projections": [_vp, _vp, ctypes.c_uint, _dp, _vp],
    "gpe_launch_count": [_vp, _llp],
    "gpe_profile": [_vp, ctypes.c_int],
    "gpe_profile_read": [_vp, _dp, _llp],
    "gpe_batch_create": [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(_vp)],
    "gpe_batch_destroy": [_vp],
    "gpe_batch_add": [_vp, ctypes.POINTER(Desc), ctypes.POINTER(ctypes.c_int)],
    "gpe_batch_remove": [_vp, ctypes.c_int],
    "gpe_batch_bind": [_vp, ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_int), _vp],
    "gpe_batch_step": [_vp, ctypes.c_int, _vp],
    "gpe_batch_diagnostics": [_vp, _dp, _vp],
    "gpe_batch_run": [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_longlong, _vp, _vp, _dp, _dp, _vp],
    "gpe_batch_set_step": [_vp, ctypes.c_int, ctypes.c_longlong],
    "gpe_batch_get_step": [_vp, ctypes.c_int, _llp],
    "gpe_batch_launch_count": [_vp, _llp],
    "gpe_normalise_noalloc": [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _vp],
}

_lib = None


def load():
    """Load the library once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH.name} is not built; run gpe_simulator_b200.build.build() "
                           "(python -c 'import __graft_entry__ as g; g.build()')")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    _lib = lib
    return lib


class GpeError(RuntimeError):
    """A non-OK status from the C ABI."""

    def __init__(self, code, message):
        super().__init__(f"[gpe status {code}] {message}")
        self.code = code


def last_error():
    lib = load()
    buf = ctypes.create_string_buffer(1024)
    lib.gpe_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(code):
    """Map a status code to the exception the reference would raise."""
    if code == GPE_OK:
        return
    msg = last_error()
    if code == GPE_ERR_ARG:
        raise ValueError(msg)
    if code == GPE_ERR_OOM:
        raise MemoryError(msg)
    raise GpeError(code, msg)
