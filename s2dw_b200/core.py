"""Python mirror of the reference's public module s2dw_core_mod
(src/mod/s2dw_core_mod.f90:29-39), backed by libs2dw_cuda.

Every function keeps the reference's name, argument meaning and array layout
(numpy arrays in Fortran order, first index fastest).  Where the Fortran
routine has intent(out) arguments, the Python function returns them.  Where
the reference prints an error and halts (s2dw_error_mod.f90:127-191), these
functions raise S2DWError with the same status code.
"""
import ctypes

import numpy as np

from ._lib import S2DWError, check, lib

_dp = ctypes.POINTER(ctypes.c_double)

__all__ = [
    "S2DWError",
    "s2dw_core_init_kernels",
    "s2dw_core_init_directionality",
    "s2dw_core_comp_Jmax",
    "s2dw_core_admiss",
    "s2dw_core_analysis_flm2wav",
    "s2dw_core_analysis_flm2wav_dynamic",
    "s2dw_core_synthesis_wav2flm",
    "s2dw_core_synthesis_wav2flm_dynamic",
    "s2dw_core_free_wavdyn",
    "s2dw_core_assimilate_int",
    "band_limits",
    "wav_scale_shape",
]


def _p(a):
    return a.ctypes.data_as(_dp)


def _f64(a, shape=None, complex_=False):
    dt = np.complex128 if complex_ else np.float64
    a = np.asfortranarray(np.asarray(a, dtype=dt))
    if shape is not None and a.shape != tuple(shape):
        raise S2DWError(8, f"array shape {a.shape} != expected {tuple(shape)}")
    return a


def s2dw_core_assimilate_int(x):
    """s2dw_core_assimilate_int (s2dw_core_mod.f90:1398): (assimilated, y)."""
    y = ctypes.c_int(0)
    ok = lib().s2dwc_assimilate_int(float(x), ctypes.byref(y))
    return bool(ok), y.value


def s2dw_core_comp_Jmax(B, alpha):
    """s2dw_core_comp_Jmax (s2dw_core_mod.f90:1365)."""
    return lib().s2dwc_comp_jmax(int(B), float(alpha))


def band_limits(jj, B, alpha):
    """(bl_hi, bl_lo) of scale jj (s2dw_core_mod.f90:372-381)."""
    hi, lo = ctypes.c_int(0), ctypes.c_int(0)
    check(lib().s2dwc_band_limits(int(jj), int(B), float(alpha), ctypes.byref(hi), ctypes.byref(lo)))
    return hi.value, lo.value


def wav_scale_shape(jj, B, N, alpha):
    """Shape (2bl-1, 2bl, N) of wavdyn(jj)%coeff (s2dw_core_mod.f90:746)."""
    hi, _ = band_limits(jj, B, alpha)
    return (2 * hi - 1, 2 * hi, N)


def s2dw_core_init_kernels(J, B, alpha):
    """s2dw_core_init_kernels (s2dw_core_mod.f90:97): (K_gamma, Phi2, bl_scoeff)."""
    K = np.zeros((J + 1, B), order="F")
    Phi2 = np.zeros(B)
    bs = ctypes.c_int(0)
    check(lib().s2dwc_init_kernels(_p(K), _p(Phi2), ctypes.byref(bs), int(J), int(B), float(alpha)))
    return K, Phi2, bs.value


def s2dw_core_init_directionality(B, N):
    """s2dw_core_init_directionality (s2dw_core_mod.f90:219): Slm (B, N)."""
    S = np.zeros((B, N), dtype=np.complex128, order="F")
    check(lib().s2dwc_init_directionality(_p(S), int(B), int(N)))
    return S


def s2dw_core_admiss(K_gamma, Phi2, B, J):
    """s2dw_core_admiss (s2dw_core_mod.f90:285): (admiss, pass)."""
    K = _f64(K_gamma, (J + 1, B))
    P = _f64(Phi2, (B,))
    a = np.zeros(B)
    ok = ctypes.c_int(0)
    check(lib().s2dwc_admiss(_p(a), _p(K), _p(P), int(B), int(J), ctypes.byref(ok)))
    return a, bool(ok.value)


def s2dw_core_analysis_flm2wav(flm, K_gamma, Slm, J, B, N, bl_scoeff, alpha, wav=None):
    """s2dw_core_analysis_flm2wav (s2dw_core_mod.f90:342): (wav, scoeff).

    wav has the static shape (J+1, 2B-1, 2B, N).  As in the reference, only
    each scale's region a<2bl-1, b<2bl is written; pass `wav` to keep the
    rest of an existing array."""
    f = _f64(flm, (B, B), True)
    K = _f64(K_gamma, (J + 1, B))
    S = _f64(Slm, (B, N), True)
    if wav is None:
        wav = np.zeros((J + 1, 2 * B - 1, 2 * B, N), order="F")
    elif wav.shape != (J + 1, 2 * B - 1, 2 * B, N) or not wav.flags["F_CONTIGUOUS"]:
        raise S2DWError(8, "wav must be a Fortran-ordered (J+1, 2B-1, 2B, N) float64 array")
    sc = np.zeros((max(bl_scoeff, 0), max(bl_scoeff, 0)), dtype=np.complex128, order="F")
    check(lib().s2dwc_analysis_flm2wav(_p(wav), _p(sc), _p(f), _p(K), _p(S), int(J), int(B), int(N),
                                       int(bl_scoeff), float(alpha)))
    return wav, sc


def s2dw_core_analysis_flm2wav_dynamic(flm, K_gamma, Slm, J, B, N, bl_scoeff, alpha):
    """s2dw_core_analysis_flm2wav_dynamic (s2dw_core_mod.f90:572):
    (wavdyn, scoeff) with wavdyn[jj] of shape (2bl-1, 2bl, N)."""
    f = _f64(flm, (B, B), True)
    K = _f64(K_gamma, (J + 1, B))
    S = _f64(Slm, (B, N), True)
    wavdyn = [np.zeros(wav_scale_shape(j, B, N, alpha), order="F") for j in range(J + 1)]
    ptrs = (_dp * (J + 1))(*[_p(w) for w in wavdyn])
    sc = np.zeros((max(bl_scoeff, 0), max(bl_scoeff, 0)), dtype=np.complex128, order="F")
    check(lib().s2dwc_analysis_flm2wav_dynamic(ptrs, _p(sc), _p(f), _p(K), _p(S), int(J), int(B), int(N),
                                               int(bl_scoeff), float(alpha)))
    return wavdyn, sc


def s2dw_core_synthesis_wav2flm(wav, scoeff, K_gamma, Phi2, Slm, J, B, N, bl_scoeff, alpha):
    """s2dw_core_synthesis_wav2flm (s2dw_core_mod.f90:816): flm (B, B)."""
    w = _f64(wav, (J + 1, 2 * B - 1, 2 * B, N))
    sc = _f64(scoeff, (bl_scoeff, bl_scoeff), True)
    K = _f64(K_gamma, (J + 1, B))
    P = _f64(Phi2, (B,))
    S = _f64(Slm, (B, N), True)
    flm = np.zeros((B, B), dtype=np.complex128, order="F")
    check(lib().s2dwc_synthesis_wav2flm(_p(flm), _p(w), _p(sc), _p(K), _p(P), _p(S), int(J), int(B), int(N),
                                        int(bl_scoeff), float(alpha)))
    return flm


def s2dw_core_synthesis_wav2flm_dynamic(wavdyn, scoeff, K_gamma, Phi2, Slm, J, B, N, bl_scoeff, alpha):
    """s2dw_core_synthesis_wav2flm_dynamic (s2dw_core_mod.f90:1060): flm.

    Like the reference, the per-scale arrays are consumed: `wavdyn` is
    emptied after the call (s2dw_core_mod.f90:1130, :1264)."""
    if len(wavdyn) != J + 1:
        raise S2DWError(8, f"wavdyn has {len(wavdyn)} scales, expected J+1={J + 1}")
    ws = [_f64(wavdyn[j], wav_scale_shape(j, B, N, alpha)) for j in range(J + 1)]
    ptrs = (_dp * (J + 1))(*[_p(w) for w in ws])
    sc = _f64(scoeff, (bl_scoeff, bl_scoeff), True)
    K = _f64(K_gamma, (J + 1, B))
    P = _f64(Phi2, (B,))
    S = _f64(Slm, (B, N), True)
    flm = np.zeros((B, B), dtype=np.complex128, order="F")
    check(lib().s2dwc_synthesis_wav2flm_dynamic(_p(flm), ptrs, _p(sc), _p(K), _p(P), _p(S), int(J), int(B),
                                                int(N), int(bl_scoeff), float(alpha)))
    if isinstance(wavdyn, list):
        wavdyn.clear()
    return flm


def s2dw_core_free_wavdyn(wavdyn):
    """s2dw_core_free_wavdyn (s2dw_core_mod.f90:1289)."""
    if isinstance(wavdyn, list):
        wavdyn.clear()


def s2dw_stat_moments(wavdyn, J, B, N, alpha, wavdyn_mask=None, higher=True):
    """s2dw_stat_moments (src/mod/s2dw_stat_mod.f90:81-275) through
    s2dwc_stat_moments: returns (mean, var, skew, kur, five, six) arrays of
    J+1 values (five and six None when `higher` is False) and the status, 0 or
    S2DW_ERROR_ARTH_WARNING (6, a scale with zero variance: its higher
    moments are zero).  With a mask the coefficient arrays are masked in
    place, as in the reference (they must then be float64 Fortran-order
    arrays).  Fewer than two unmasked samples raises S2DWError (code 8)."""
    ws = []
    for j in range(J + 1):
        w = wavdyn[j]
        if wavdyn_mask is not None and not (isinstance(w, np.ndarray) and w.dtype == np.float64
                                            and w.flags.f_contiguous):
            raise ValueError("with a mask, wavdyn arrays are masked in place: pass float64 Fortran-order arrays")
        ws.append(_f64(w, wav_scale_shape(j, B, N, alpha)))
    ptrs = (_dp * (J + 1))(*[_p(w) for w in ws])
    mk = None
    if wavdyn_mask is not None:
        ms = [_f64(m, wav_scale_shape(j, B, N, alpha)) for j, m in enumerate(wavdyn_mask)]
        mk = (_dp * (J + 1))(*[_p(m) for m in ms])
    out = [np.zeros(J + 1) for _ in range(6)]
    st = lib().s2dwc_stat_moments(ptrs, int(J), int(B), int(N), float(alpha), _p(out[0]), _p(out[1]), _p(out[2]),
                                  _p(out[3]), mk, _p(out[4]) if higher else None,
                                  _p(out[5]) if higher else None)
    if st not in (0, 6):
        check(st)
    if not higher:
        out[4] = out[5] = None
    return tuple(out), st
