"""Pins the oracle's stage conventions without the oracle's own machinery.

The oracle restates the reference loop by loop: Turok-Bucher planes of
d^l(pi/2), the contraction over l, a gamma DFT, naive beta sums with the
2cos / 2i sin kernels, and FFTW-convention c2r / r2c transforms.  This file
evaluates the same transforms a second way, by direct sums at the sample
points with the Wigner d-functions at the sample angles themselves (the
Wigner sum formula, in 80-bit long double), with no FFT, no beta sum and no
d(pi/2) plane.  The two agree only if every convention of the staged form
(FFT signs and normalisation, the Hermitian completion of the c2r, the beta
grid, the eta kernels, the +-n phases, the m' fold, the quadrature weights)
is the one the direct form implies.

Direct forms, derived from s2dw_core_mod.f90 with the identity
sum_{m'=-l..l} d^l_{m'm}(pi/2) d^l_{m'n}(pi/2) e^{i m' beta} = i^{m-n} d^l_{mn}(beta)
(checked below), for one scale j with band limits (bl_lo, bl):

analysis (:625-768):
  X_m(b, g) = sum_{l in (bl_lo, bl), l >= m} sum_{n: N+n odd, |n| <= min(N-1, l)}
              s(l, m, n) d^l_{mn}(beta_b) e^{i n gamma_g},
  s = conj(K_j(l) S(l, n)) f(l, m) for n >= 0, (-1)^n K_j(l) S(l, -n) f(l, m) for n < 0,
  w(a, b, g) = Re X_0 + 2 Re sum_{m=1}^{bl-1} X_m e^{i m alpha_a}
  -- for a real signal and a real wavelet this is the rotated-wavelet inner
  product sum_{lmn} f_lm Psi*_ln D^{l*}_{mn}(alpha, beta, gamma) with
  D = e^{-i m alpha} d^l_{mn}(beta) e^{-i n gamma};

synthesis (:1104-1261):
  flm(l, m) = sum_j sum_{n >= 0, N+n odd, n <= min(N-1, l)} c_n (2l+1)/(8 pi^2) K_j(l) S(l, n)
              (4 pi^2 / N)/(2bl-1) sum_{a,b,g} w_j(a, b, g) q_bl(beta_b) e^{-i m alpha_a}
              e^{-i n gamma_g} d^l_{mn}(beta_b)
            + Phi2(l) scoeff(l, m) for l, m < bl_scoeff,
  c_0 = 1, c_n = 2, q_bl the reference's quadrature weights (:1436-1450);

with alpha_a = 2 pi a/(2bl-1), beta_b = pi (2b+1)/(4 bl), gamma_g = pi g/N.
"""
import math

import mpmath as mp
import numpy as np
import pytest

from oracle import oracle as O

LD = np.longdouble
PI = LD("3.14159265358979323846264338327950288")


def _ld(x):
    """An mpmath number as a long double, through its decimal string."""
    return LD(mp.nstr(x, 30, strip_zeros=False))


_COEF = {}


def _wigner_terms(l, a, b):
    """Terms (coefficient, power of cos(beta/2), power of sin(beta/2)) of
    the Wigner sum formula for d^l_{ab}(beta), first index a."""
    key = (l, a, b)
    if key not in _COEF:
        mp.mp.dps = 40
        f = math.factorial
        num = mp.sqrt(mp.mpf(f(l + a) * f(l - a) * f(l + b) * f(l - b)))
        terms = []
        for k in range(max(0, b - a), min(l + b, l - a) + 1):
            den = f(l + b - k) * f(k) * f(a - b + k) * f(l - a - k)
            terms.append(((-1) ** (a - b + k) * _ld(num / den), 2 * l + b - a - 2 * k, a - b + 2 * k))
        _COEF[key] = terms
    return _COEF[key]


def wigner_d(l, a, b, beta):
    """d^l_{ab}(beta) for an array of beta, in long double."""
    c, s = np.cos(beta / 2), np.sin(beta / 2)
    out = np.zeros_like(beta)
    for co, p, q in _wigner_terms(l, a, b):
        out += co * c ** p * s ** q
    return out


def test_factorisation_identity():
    """sum_{m'} d^l_{m'm}(pi/2) d^l_{m'n}(pi/2) e^{i m' beta} = i^{m-n} d^l_{mn}(beta),
    in 30-digit arithmetic (the identity the direct forms rest on)."""
    mp.mp.dps = 30

    def d_mp(l, a, b, beta):
        c, s = mp.cos(beta / 2), mp.sin(beta / 2)
        f = mp.factorial
        tot = mp.mpf(0)
        for k in range(max(0, b - a), min(l + b, l - a) + 1):
            tot += ((-1) ** (a - b + k) * mp.sqrt(f(l + a) * f(l - a) * f(l + b) * f(l - b))
                    / (f(l + b - k) * f(k) * f(a - b + k) * f(l - a - k))
                    * c ** (2 * l + b - a - 2 * k) * s ** (a - b + 2 * k))
        return tot

    for l, m, n, beta in [(4, 1, 2, 0.7), (5, 3, -1, 2.9), (6, 0, 3, 1.1), (7, -2, 5, 0.05), (3, 3, 3, 1.5)]:
        beta = mp.mpf(beta)
        lhs = mp.fsum(d_mp(l, mm, m, mp.pi / 2) * d_mp(l, mm, n, mp.pi / 2) * mp.expj(mm * beta)
                      for mm in range(-l, l + 1))
        rhs = mp.mpc(0, 1) ** (m - n) * d_mp(l, m, n, beta)
        assert abs(lhs - rhs) < mp.mpf(10) ** -25


def test_long_double_wigner_against_mpmath():
    mp.mp.dps = 30
    beta = np.array([0.1, 1.3, 2.8], dtype=LD)
    for l, a, b in [(15, 3, -2), (15, 15, 0), (12, -7, 7), (20, 1, 1)]:
        got = wigner_d(l, a, b, beta)
        for i, bt in enumerate(beta):
            f = math.factorial
            c, s = mp.cos(mp.mpf(float(bt)) / 2), mp.sin(mp.mpf(float(bt)) / 2)
            ref = mp.fsum((-1) ** (a - b + k) * mp.sqrt(f(l + a) * f(l - a) * f(l + b) * f(l - b))
                          / (f(l + b - k) * f(k) * f(a - b + k) * f(l - a - k))
                          * c ** (2 * l + b - a - 2 * k) * s ** (a - b + 2 * k)
                          for k in range(max(0, b - a), min(l + b, l - a) + 1))
            assert abs(float(got[i]) - float(ref)) < 1e-15


def _grids(bl, N):
    a = np.arange(2 * bl - 1)
    b = np.arange(2 * bl)
    g = np.arange(N)
    alpha = 2 * PI * a.astype(LD) / (2 * bl - 1)
    beta = PI * (2 * b.astype(LD) + 1) / (4 * bl)
    gamma = PI * g.astype(LD) / N
    return alpha, beta, gamma


def _nset(N, l, signed):
    k = min(N - 1, l)
    lo = -k if signed else 0
    return [n for n in range(lo, k + 1) if (N + n) % 2]


def direct_analysis_scale(j, flm, K, S, B, N, alpha_):
    bl, blo = O.band_limits(j, B, alpha_)
    al, be, ga = _grids(bl, N)
    X = np.zeros((bl, 2 * bl, N), dtype=np.clongdouble)
    for l in range(blo + 1, bl):
        for n in _nset(N, l, True):
            ph = np.cos(n * ga) + 1j * np.sin(n * ga)  # e^{i n gamma_g}
            kap = K[j, l] * S[l, -n] * (-1) ** n if n < 0 else np.conj(K[j, l] * S[l, n])
            for m in range(0, l + 1):
                sv = kap * flm[l, m]
                X[m] += sv * wigner_d(l, m, n, be)[:, None] * ph[None, :]
    # c2r of length 2bl-1: Re X_0 + 2 Re sum_{m>=1} X_m e^{i m alpha_a}
    m = np.arange(bl)
    E = np.cos(np.outer(al, m)) + 1j * np.sin(np.outer(al, m))  # (a, m)
    wgt = np.where(m == 0, 1, 2).astype(LD)
    Xr = X.copy()
    Xr[0] = Xr[0].real
    w = np.einsum("am,mbg->abg", E * wgt[None, :], Xr).real
    return w.astype(np.float64)


def quad_weight(theta, bl):
    k = np.arange(bl, dtype=LD)
    return (LD(2) / bl) * np.sin(theta) * np.sum(np.sin((2 * k + 1) * theta) / (2 * k + 1))


def direct_synthesis(wav, sc, K, Phi2, S, J, B, N, bs, alpha_):
    flm = np.zeros((B, B), dtype=np.clongdouble)
    for j in range(J + 1):
        bl, blo = O.band_limits(j, B, alpha_)
        if blo + 1 >= bl:
            continue
        al, be, ga = _grids(bl, N)
        q = np.array([quad_weight(t, bl) for t in be], dtype=LD)
        m_ = np.arange(bl)
        Em = np.cos(np.outer(m_, al)) - 1j * np.sin(np.outer(m_, al))  # e^{-i m alpha_a}, (m, a)
        W = np.asarray(wav[j], dtype=LD)
        Y = np.einsum("ma,abg->mbg", Em, W) * (LD(4) * PI ** 2 / N) / (2 * bl - 1)
        for n in _nset(N, bl - 1, False):
            eg = np.cos(n * ga) - 1j * np.sin(n * ga)
            Z = np.einsum("mbg,g->mb", Y, eg) * q[None, :]  # (m, b)
            for l in range(max(blo + 1, n), bl):
                fac = (1 if n == 0 else 2) * LD(2 * l + 1) / (8 * PI ** 2) * K[j, l] * S[l, n]
                for m in range(0, l + 1):
                    flm[l, m] += fac * np.sum(Z[m] * wigner_d(l, m, n, be))
    for l in range(bs):
        for m in range(bs):
            flm[l, m] += Phi2[l] * sc[l, m]
    return flm.astype(np.complex128)


CASES = [(8, 3, 2.0, None), (16, 4, 2.0, None), (12, 3, 3.0, None), (16, 2, 2.0, 2), (10, 1, 1.5, None)]


def _setup(B, N, alpha_, J):
    if J is None:
        J = O.comp_jmax(B, alpha_)
    K, P, bs = O.init_kernels(J, B, alpha_)
    S = O.init_directionality(B, N)
    return J, K, P, bs, S


def _flm(B, seed):
    rng = np.random.default_rng(seed)
    f = np.zeros((B, B), dtype=np.complex128, order="F")
    for l in range(B):
        f[l, 0] = rng.standard_normal()
        f[l, 1:l + 1] = rng.standard_normal(l) + 1j * rng.standard_normal(l)
    return f


@pytest.mark.parametrize("B,N,alpha_,J", CASES)
def test_oracle_analysis_equals_direct_sum(B, N, alpha_, J):
    J, K, P, bs, S = _setup(B, N, alpha_, J)
    flm = _flm(B, seed=B * 10 + N)
    wav, _ = O.analysis_dynamic(flm, K, S, J, B, N, bs, alpha_)
    for j in range(J + 1):
        ref = direct_analysis_scale(j, flm, K, S, B, N, alpha_)
        scale = np.abs(ref).max()
        if scale == 0:
            assert np.abs(wav[j]).max() == 0
            continue
        err = np.abs(wav[j] - ref).max() / scale
        assert err < 2e-14, f"scale {j}: max|w_oracle - w_direct|/max|w| = {err:.2e}"


@pytest.mark.parametrize("B,N,alpha_,J", CASES)
def test_oracle_synthesis_equals_direct_sum(B, N, alpha_, J):
    """On random (not band-limit-consistent) coefficients, so that the
    synthesis is pinned as an operator and not only through a round trip."""
    J, K, P, bs, S = _setup(B, N, alpha_, J)
    rng = np.random.default_rng(B + N)
    wav = []
    for j in range(J + 1):
        bl, _ = O.band_limits(j, B, alpha_)
        wav.append(np.asfortranarray(rng.standard_normal((2 * bl - 1, 2 * bl, N))))
    sc = np.asfortranarray(rng.standard_normal((bs, bs)) + 1j * rng.standard_normal((bs, bs)))
    got = O.synthesis_dynamic(wav, sc, K, P, S, J, B, N, bs, alpha_)
    ref = direct_synthesis(wav, sc, K, P, S, J, B, N, bs, alpha_)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 2e-14, f"max|f_oracle - f_direct|/max|f| = {err:.2e}"


def test_direct_sum_is_the_rotated_wavelet_inner_product():
    """For a real signal (f_{l,-m} = (-1)^m conj f_lm) the c2r form equals the
    full sum over m in [-l, l] of f_lm Psi*_ln D^{l*}_{mn} (real-valued)."""
    B, N, alpha_ = 8, 3, 2.0
    J, K, P, bs, S = _setup(B, N, alpha_, None)
    flm = _flm(B, seed=5)
    flm[:, 0] = flm[:, 0].real
    j = 1
    bl, blo = O.band_limits(j, B, alpha_)
    w = direct_analysis_scale(j, flm, K, S, B, N, alpha_)
    al, be, ga = _grids(bl, N)
    full = np.zeros((2 * bl - 1, 2 * bl, N), dtype=np.clongdouble)
    for l in range(blo + 1, bl):
        for n in _nset(N, l, True):
            psi = K[j, l] * S[l, n] if n >= 0 else (-1) ** n * np.conj(K[j, l] * S[l, -n])
            for m in range(-l, l + 1):
                f = flm[l, m] if m >= 0 else (-1) ** m * np.conj(flm[l, -m])
                d = wigner_d(l, m, n, be)
                # D^{l*}_{mn}(alpha, beta, gamma) = e^{i m alpha} d^l_{mn}(beta) e^{i n gamma}
                Dc = (np.exp(1j * m * al.astype(float))[:, None, None] * d.astype(float)[None, :, None]
                      * np.exp(1j * n * ga.astype(float))[None, None, :])
                full += f * np.conj(psi) * Dc
    assert np.abs(full.imag).max() < 1e-14 * np.abs(full.real).max()
    assert np.abs(full.real - w).max() < 1e-14 * np.abs(w).max()
