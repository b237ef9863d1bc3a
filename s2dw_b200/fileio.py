"""Python mirror of the reference's s2dw_fileio_mod (src/mod/s2dw_fileio_mod.f90):
FITS and Matlab wavelet coefficient files, through the C ABI
(s2dwc_fileio_*).  Names, argument order and outputs follow the reference's
generic procedures; the static or dynamic form is chosen from the type of
`wav` (one (J+1, 2B-1, 2B, N) array, or a list of per-scale arrays).

    s2dw_fileio_fits_wav_write(wav, scoeff, J, B, N, bl_scoeff, alpha, filename, comment=None)
    s2dw_fileio_fits_wav_read(filename, dynamic=True) -> (wav, scoeff, J, B, N, bl_scoeff, alpha)
    s2dw_fileio_matlab_wav_write(...), s2dw_fileio_matlab_wav_read(...)  (same)

Errors raise S2DWError with the reference's S2DW_ERROR_* code
(S2DW_ERROR_FILEIO = 14 for missing or existing files and malformed ones).
"""
import ctypes

import numpy as np

from ._lib import S2DWError, check, lib
from .core import _dp, _f64, _p, wav_scale_shape

__all__ = [
    "s2dw_fileio_fits_wav_write",
    "s2dw_fileio_fits_wav_read",
    "s2dw_fileio_matlab_wav_write",
    "s2dw_fileio_matlab_wav_read",
]


def _enc(s):
    return None if s is None else str(s).encode()


def _write(kind, wav, scoeff, J, B, N, bl_scoeff, alpha, filename, comment):
    sc = _f64(scoeff, (bl_scoeff, bl_scoeff), True)
    if isinstance(wav, (list, tuple)):
        if len(wav) != J + 1:
            raise S2DWError(8, f"wav has {len(wav)} scales, expected J+1={J + 1}")
        ws = [_f64(wav[j], wav_scale_shape(j, B, N, alpha)) for j in range(J + 1)]
        ptrs = (_dp * (J + 1))(*[_p(w) for w in ws])
        f = getattr(lib(), f"s2dwc_fileio_{kind}_wav_write_dynamic")
        check(f(ptrs, _p(sc), int(J), int(B), int(N), int(bl_scoeff), float(alpha), _enc(filename), _enc(comment)))
    else:
        w = _f64(wav, (J + 1, 2 * B - 1, 2 * B, N))
        f = getattr(lib(), f"s2dwc_fileio_{kind}_wav_write_static")
        check(f(_p(w), _p(sc), int(J), int(B), int(N), int(bl_scoeff), float(alpha), _enc(filename), _enc(comment)))


def _read(kind, filename, dynamic):
    J, B, N, bs = (ctypes.c_int(0) for _ in range(4))
    alpha = ctypes.c_double(0.0)
    L = lib()
    check(getattr(L, f"s2dwc_fileio_{kind}_wav_read_header")(_enc(filename), ctypes.byref(J), ctypes.byref(B),
                                                             ctypes.byref(N), ctypes.byref(bs), ctypes.byref(alpha)))
    J, B, N, bs, alpha = J.value, B.value, N.value, bs.value, alpha.value
    sc = np.zeros((bs, bs), dtype=np.complex128, order="F")
    if dynamic:
        wav = [np.zeros(wav_scale_shape(j, B, N, alpha), order="F") for j in range(J + 1)]
        ptrs = (_dp * (J + 1))(*[_p(w) for w in wav])
        check(getattr(L, f"s2dwc_fileio_{kind}_wav_read_dynamic")(ptrs, _p(sc), J, B, N, bs, _enc(filename)))
    else:
        wav = np.zeros((J + 1, 2 * B - 1, 2 * B, N), order="F")
        check(getattr(L, f"s2dwc_fileio_{kind}_wav_read_static")(_p(wav), _p(sc), J, B, N, bs, _enc(filename)))
    return wav, sc, J, B, N, bs, alpha


def s2dw_fileio_fits_wav_write(wav, scoeff, J, B, N, bl_scoeff, alpha, filename, comment=None):
    """s2dw_fileio_fits_wav_write_{static,dynamic} (fileio:796-926, :956-1079)."""
    _write("fits", wav, scoeff, J, B, N, bl_scoeff, alpha, filename, comment)


def s2dw_fileio_fits_wav_read(filename, dynamic=True):
    """s2dw_fileio_fits_wav_read_{dynamic,static} (fileio:1286-1435, :1109-1253):
    (wav, scoeff, J, B, N, bl_scoeff, alpha)."""
    return _read("fits", filename, dynamic)


def s2dw_fileio_matlab_wav_write(wav, scoeff, J, B, N, bl_scoeff, alpha, filename, comment=None):
    """s2dw_fileio_matlab_wav_write_{static,dynamic} (fileio:102-268, :298-436):
    writes filename (.m) and <base>_scoeff.dat, <base>_wcoeff.dat."""
    _write("matlab", wav, scoeff, J, B, N, bl_scoeff, alpha, filename, comment)


def s2dw_fileio_matlab_wav_read(filename, dynamic=True):
    """s2dw_fileio_matlab_wav_read_{dynamic,static} (fileio:637-763, :473-601)."""
    return _read("matlab", filename, dynamic)
