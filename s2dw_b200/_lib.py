"""ctypes binding of libs2dw_cuda.so (the C ABI declared in include/s2dw_cuda.h).

The library is loaded from this package directory.  There is no fallback: if
the shared library is missing or fails to load, every call raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libs2dw_cuda.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_llp = ctypes.POINTER(ctypes.c_longlong)
_vp = ctypes.c_void_p
_i, _d = ctypes.c_int, ctypes.c_double

# name -> (restype, argtypes); every symbol the header declares
SIGNATURES = {
    "s2dwc_version": (ctypes.c_char_p, []),
    "s2dwc_init": (_i, []),
    "s2dwc_finalize": (_i, []),
    "s2dwc_error_string": (ctypes.c_char_p, [_i]),
    "s2dwc_last_error_message": (ctypes.c_char_p, []),
    "s2dwc_assimilate_int": (_i, [_d, _ip]),
    "s2dwc_comp_jmax": (_i, [_i, _d]),
    "s2dwc_band_limits": (_i, [_i, _i, _d, _ip, _ip]),
    "s2dwc_wav_scale_size": (ctypes.c_longlong, [_i, _i, _i, _d]),
    "s2dwc_init_kernels": (_i, [_dp, _dp, _ip, _i, _i, _d]),
    "s2dwc_init_directionality": (_i, [_dp, _i, _i]),
    "s2dwc_admiss": (_i, [_dp, _dp, _dp, _i, _i, _ip]),
    "s2dwc_analysis_flm2wav": (_i, [_dp, _dp, _dp, _dp, _dp, _i, _i, _i, _i, _d]),
    "s2dwc_analysis_flm2wav_dynamic": (_i, [ctypes.POINTER(_dp), _dp, _dp, _dp, _dp, _i, _i, _i, _i, _d]),
    "s2dwc_synthesis_wav2flm": (_i, [_dp, _dp, _dp, _dp, _dp, _dp, _i, _i, _i, _i, _d]),
    "s2dwc_synthesis_wav2flm_dynamic": (_i, [_dp, ctypes.POINTER(_dp), _dp, _dp, _dp, _dp, _i, _i, _i, _i, _d]),
    "s2dwc_plan_create": (_i, [ctypes.POINTER(_vp), _i, _i, _d, _i, _i, _i]),
    "s2dwc_plan_destroy": (_i, [_vp]),
    "s2dwc_plan_footprint": (_i, [_i, _i, _d, _i, _i, _llp]),
    "s2dwc_set_plan_memory_limit": (_i, [ctypes.c_longlong]),
    "s2dwc_plan_set_tables": (_i, [_vp, _dp, _dp, _dp, _i]),
    "s2dwc_plan_wav_offsets": (_i, [_vp, _llp]),
    "s2dwc_plan_workspace_bytes": (ctypes.c_longlong, [_vp]),
    "s2dwc_plan_analysis": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "s2dwc_plan_synthesis": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "s2dwc_plan_analysis_noalloc": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "s2dwc_plan_analysis_batch": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "s2dwc_plan_synthesis_batch": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "s2dwc_plan_check": (_i, [_vp]),
    "s2dwc_plan_set_wait_limit": (_i, [_vp, ctypes.c_longlong]),
    "s2dwc_plan_set_priority": (_i, [_vp, _i]),
    "s2dwc_plan_set_split_min_batch": (_i, [_vp, _i]),
    "s2dwc_plan_reserve": (_i, [_vp, _i, _vp]),
    "s2dwc_plan_stat_moments": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "s2dwc_stat_moments": (_i, [ctypes.POINTER(_dp), _i, _i, _i, _d, _dp, _dp, _dp, _dp, ctypes.POINTER(_dp),
                                _dp, _dp]),
    "s2dwc_plan_launch_count": (_i, [_vp, _ip, _ip]),
    "s2dwc_plan_set_timing": (_i, [_vp, _i]),
    "s2dwc_plan_timing": (_i, [_vp, _i, _llp, _dp]),
    "s2dwc_plan_timing_reset": (_i, [_vp]),
    "s2dwc_fileio_fits_wav_write_dynamic": (_i, [ctypes.POINTER(_dp), _dp, _i, _i, _i, _i, _d, ctypes.c_char_p,
                                                 ctypes.c_char_p]),
    "s2dwc_fileio_fits_wav_write_static": (_i, [_dp, _dp, _i, _i, _i, _i, _d, ctypes.c_char_p, ctypes.c_char_p]),
    "s2dwc_fileio_fits_wav_read_header": (_i, [ctypes.c_char_p, _ip, _ip, _ip, _ip, _dp]),
    "s2dwc_fileio_fits_wav_read_dynamic": (_i, [ctypes.POINTER(_dp), _dp, _i, _i, _i, _i, ctypes.c_char_p]),
    "s2dwc_fileio_fits_wav_read_static": (_i, [_dp, _dp, _i, _i, _i, _i, ctypes.c_char_p]),
    "s2dwc_fileio_matlab_wav_write_dynamic": (_i, [ctypes.POINTER(_dp), _dp, _i, _i, _i, _i, _d, ctypes.c_char_p,
                                                   ctypes.c_char_p]),
    "s2dwc_fileio_matlab_wav_write_static": (_i, [_dp, _dp, _i, _i, _i, _i, _d, ctypes.c_char_p, ctypes.c_char_p]),
    "s2dwc_fileio_matlab_wav_read_header": (_i, [ctypes.c_char_p, _ip, _ip, _ip, _ip, _dp]),
    "s2dwc_fileio_matlab_wav_read_dynamic": (_i, [ctypes.POINTER(_dp), _dp, _i, _i, _i, _i, ctypes.c_char_p]),
    "s2dwc_fileio_matlab_wav_read_static": (_i, [_dp, _dp, _i, _i, _i, _i, ctypes.c_char_p]),
}

KERNEL_KINDS = ["lwalk", "mwalk", "ana_beta", "ana_alpha", "syn_alpha", "syn_beta", "other"]

_lib = None


class S2DWError(RuntimeError):
    """An S2DW status code (the reference's S2DW_ERROR_* numbering)."""

    def __init__(self, code, message):
        self.code = code
        super().__init__(f"S2DW_ERROR {code}: {message}")


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with `python -m s2dw_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code):
    """Raise S2DWError for a non-zero status."""
    if code != 0:
        L = lib()
        detail = L.s2dwc_last_error_message().decode(errors="replace")
        base = L.s2dwc_error_string(code).decode()
        raise S2DWError(code, f"{base}: {detail}" if detail else base)
    return code
