"""ctypes front end of the CPU restatement in s2dw_oracle.c.

TEST INFRASTRUCTURE ONLY: the parity oracle and the CPU baseline.  Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module; the s2dw_b200 package never does.

Parity unpinned: the reference (Fortran 90 + FFTW) cannot be compiled on
this machine and ships no golden vectors, so this restatement is pinned by
known-answer tests instead (see tests/test_oracle.py).

Arrays use the reference's Fortran layouts (numpy order='F'):
  flm (B, B) complex128, K_gamma (J+1, B), Phi2 (B,), Slm (B, N) complex128,
  per-scale wavelet arrays (2bl-1, 2bl, N), static wav (J+1, 2B-1, 2B, N).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libs2dw_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build():
    """Compile the oracle shared library with its Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        L.orc_assimilate_int.argtypes = [ctypes.c_double, _ip]
        L.orc_comp_jmax.argtypes = [ctypes.c_int, ctypes.c_double]
        L.orc_params_valid.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.orc_band_limits.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, _ip, _ip]
        L.orc_quad_weights.argtypes = [ctypes.c_double, ctypes.c_int]
        L.orc_quad_weights.restype = ctypes.c_double
        L.orc_init_kernels.argtypes = [_dp, _dp, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.orc_init_directionality.argtypes = [_dp, ctypes.c_int, ctypes.c_int]
        L.orc_admiss.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_int]
        L.orc_dl_beta_operator.argtypes = [_dp, ctypes.c_double, ctypes.c_int]
        L.orc_dl_edge_ld.argtypes = [_dp, ctypes.c_int]
        L.orc_set_dl_method.argtypes = [ctypes.c_int]
        L.orc_analysis_scale.argtypes = [ctypes.c_int, _dp, ctypes.c_size_t, ctypes.c_size_t,
                                         ctypes.c_size_t, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_double, _dp, _dp, _dp]
        L.orc_synthesis_scale.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_size_t, ctypes.c_size_t,
                                          ctypes.c_size_t, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_double, _dp, _dp]
        L.orc_analysis_dynamic.argtypes = [ctypes.POINTER(_dp), _dp, _dp, _dp, _dp, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.orc_analysis_static.argtypes = [_dp, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.orc_synthesis_dynamic.argtypes = [_dp, ctypes.POINTER(_dp), _dp, _dp, _dp, _dp,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_double]
        L.orc_synthesis_static.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.orc_ran2_reset.argtypes = []
        L.orc_test_gen_flm.argtypes = [ctypes.c_int, _dp, ctypes.c_int32]
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_set_num_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.flags["F_CONTIGUOUS"] or a.ndim <= 1, "arrays must be Fortran-ordered"
    return a.ctypes.data_as(_dp)


def _check(status, what):
    if status != 0:
        raise RuntimeError(f"oracle {what} failed with S2DW error code {status}")


def num_threads():
    return lib().orc_num_threads()


def set_num_threads(n):
    lib().orc_set_num_threads(int(n))


def assimilate_int(x):
    y = ctypes.c_int(0)
    ok = lib().orc_assimilate_int(float(x), ctypes.byref(y))
    return bool(ok), y.value


def comp_jmax(B, alpha):
    return lib().orc_comp_jmax(int(B), float(alpha))


def params_valid(J, B, alpha, N=-1):
    return bool(lib().orc_params_valid(int(J), int(B), float(alpha), int(N)))


def band_limits(jj, B, alpha):
    hi, lo = ctypes.c_int(0), ctypes.c_int(0)
    lib().orc_band_limits(int(jj), int(B), float(alpha), ctypes.byref(hi), ctypes.byref(lo))
    return hi.value, lo.value


def quad_weights(theta, B):
    return lib().orc_quad_weights(float(theta), int(B))


def init_kernels(J, B, alpha):
    K = np.zeros((J + 1, B), order="F")
    Phi2 = np.zeros(B)
    bs = ctypes.c_int(0)
    _check(lib().orc_init_kernels(_p(K), _p(Phi2), ctypes.byref(bs), J, B, float(alpha)),
           "init_kernels")
    return K, Phi2, bs.value


def init_directionality(B, N):
    S = np.zeros((B, N), dtype=np.complex128, order="F")
    _check(lib().orc_init_directionality(_p(S), B, N), "init_directionality")
    return S


def admiss(K, Phi2, B, J):
    a = np.zeros(B)
    ok = lib().orc_admiss(_p(a), _p(K), _p(Phi2), B, J)
    return a, bool(ok)


def dl_plane(l, beta=np.pi / 2):
    """d^l(beta) as an array D[i+l, k+l] = dl(i, k), i, k in [-l, l]."""
    D = np.zeros((2 * l + 1, 2 * l + 1), order="F")
    lib().orc_dl_beta_operator(_p(D), float(beta), int(l))
    return D


def dl_plane_accurate(l):
    """d^l(pi/2) from the long-double edge recurrence (a diagnostic, not the
    reference's algorithm), laid out as dl_plane."""
    D = np.zeros((2 * l + 1, 2 * l + 1), order="F")
    lib().orc_dl_edge_ld(_p(D), int(l))
    return D


def set_dl_method(m):
    """0: the reference's Turok-Bucher planes (default); 1: the accurate
    long-double planes of dl_plane_accurate, to measure how much of a
    difference at large l is the reference's own d-plane error."""
    lib().orc_set_dl_method(int(m))


def analysis_scale(jj, flm, K, S, J, B, N, alpha, debug=False):
    """One scale of the analysis; returns coeff (2bl-1, 2bl, N) and, when
    debug is set, the intermediates Tmmm, Tmmg, Tmbg."""
    hi, _ = band_limits(jj, B, alpha)
    out = np.zeros((2 * hi - 1, 2 * hi, N), order="F")
    dbg = [None, None, None]
    if debug:
        dbg = [np.zeros((hi, hi, 2 * N - 1), dtype=np.complex128, order="F"),
               np.zeros((hi, hi, N), dtype=np.complex128, order="F"),
               np.zeros((hi, 2 * hi, N), dtype=np.complex128, order="F")]
    n = 2 * hi - 1
    _check(lib().orc_analysis_scale(jj, _p(out), 1, n, n * 2 * hi, _p(flm), _p(K), _p(S), J, B, N,
                                    float(alpha), *[_p(d) for d in dbg]), "analysis_scale")
    return (out, *dbg) if debug else out


def analysis_dynamic(flm, K, S, J, B, N, bl_scoeff, alpha):
    """s2dw_core_analysis_flm2wav_dynamic: returns ([coeff_j], scoeff)."""
    wav = []
    for jj in range(J + 1):
        hi, _ = band_limits(jj, B, alpha)
        wav.append(np.zeros((2 * hi - 1, 2 * hi, N), order="F"))
    ptrs = (_dp * (J + 1))(*[_p(w) for w in wav])
    sc = np.zeros((bl_scoeff, bl_scoeff), dtype=np.complex128, order="F")
    _check(lib().orc_analysis_dynamic(ptrs, _p(sc), _p(flm), _p(K), _p(S), J, B, N, bl_scoeff,
                                      float(alpha)), "analysis_dynamic")
    return wav, sc


def analysis_static(flm, K, S, J, B, N, bl_scoeff, alpha):
    """s2dw_core_analysis_flm2wav: returns (wav (J+1,2B-1,2B,N), scoeff).
    Entries outside each scale's a<2bl-1, b<2bl region stay zero."""
    wav = np.zeros((J + 1, 2 * B - 1, 2 * B, N), order="F")
    sc = np.zeros((bl_scoeff, bl_scoeff), dtype=np.complex128, order="F")
    _check(lib().orc_analysis_static(_p(wav), _p(sc), _p(flm), _p(K), _p(S), J, B, N, bl_scoeff,
                                     float(alpha)), "analysis_static")
    return wav, sc


def synthesis_dynamic(wav, scoeff, K, Phi2, S, J, B, N, bl_scoeff, alpha):
    if len(wav) != J + 1:
        raise ValueError(f"oracle synthesis_dynamic: {len(wav)} scales given, J+1 = {J + 1} expected")
    flm = np.zeros((B, B), dtype=np.complex128, order="F")
    wav = [np.asfortranarray(w) for w in wav]
    ptrs = (_dp * (J + 1))(*[_p(w) for w in wav])
    _check(lib().orc_synthesis_dynamic(_p(flm), ptrs, _p(np.asfortranarray(scoeff)), _p(K), _p(Phi2),
                                       _p(S), J, B, N, bl_scoeff, float(alpha)), "synthesis_dynamic")
    return flm


def synthesis_static(wav, scoeff, K, Phi2, S, J, B, N, bl_scoeff, alpha):
    flm = np.zeros((B, B), dtype=np.complex128, order="F")
    _check(lib().orc_synthesis_static(_p(flm), _p(np.asfortranarray(wav)),
                                      _p(np.asfortranarray(scoeff)), _p(K), _p(Phi2), _p(S), J, B, N,
                                      bl_scoeff, float(alpha)), "synthesis_static")
    return flm


def synthesis_scale_debug(jj, coeff, K, S, J, B, N, alpha):
    """One scale of the synthesis from zero; returns (flm contribution,
    V after the alpha FFT, V after the beta sum and fold)."""
    hi, _ = band_limits(jj, B, alpha)
    flm = np.zeros((B, B), dtype=np.complex128, order="F")
    V = np.zeros((hi, 2 * hi, N), dtype=np.complex128, order="F")
    Vm = np.zeros((hi, 2 * hi, N), dtype=np.complex128, order="F")
    n = 2 * hi - 1
    coeff = np.asfortranarray(coeff)
    _check(lib().orc_synthesis_scale(jj, _p(flm), _p(coeff), 1, n, n * 2 * hi, _p(K), _p(S), J, B,
                                     N, float(alpha), _p(V), _p(Vm)), "synthesis_scale")
    return flm, V, Vm


def test_gen_flm(L, seed=1):
    """s2dw_test_gen_flm with the reference's ran2_dp stream (fresh state)."""
    lib().orc_ran2_reset()
    flm = np.zeros((L + 1, L + 1), dtype=np.complex128, order="F")
    lib().orc_test_gen_flm(int(L), _p(flm), int(seed))
    return flm


def stat_moments(wavdyn, J, B, N, alpha, mask=None, higher=True):
    """s2dw_stat_moments on copies of the per-scale arrays: returns (status,
    moments) with moments a (J+1, 6) array of mean, var, skew, kur, five, six
    (five and six zero when higher is False) and the masked coefficients
    (the reference masks wavdyn in place)."""
    ws = [np.array(w, dtype=np.float64, order="F", copy=True) for w in wavdyn]
    ptrs = (_dp * (J + 1))(*[_p(w) for w in ws])
    mk = None
    if mask is not None:
        ms = [np.asfortranarray(m, dtype=np.float64) for m in mask]
        mk = (_dp * (J + 1))(*[_p(m) for m in ms])
    out = np.zeros((6, J + 1))
    L = lib()
    L.orc_stat_moments.restype = ctypes.c_int
    L.orc_stat_moments.argtypes = [ctypes.POINTER(_dp), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                   _dp, _dp, _dp, _dp, ctypes.POINTER(_dp), _dp, _dp]
    rows = [out[i].ctypes.data_as(_dp) for i in range(6)]
    st = L.orc_stat_moments(ptrs, J, B, N, float(alpha), rows[0], rows[1], rows[2], rows[3], mk,
                            rows[4] if higher else None, rows[5] if higher else None)
    return st, out.T.copy(), ws
