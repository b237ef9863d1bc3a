"""Smallest band limits and empty scales on the GPU against the oracle.

At B=2 (alpha=2), B=3 (alpha=1.5), B=6 (alpha=1.2) and B=7 (alpha=1.25) some
scale's l range (bl_lo, bl) is empty (s2dw_core_mod.f90:372-381 give
bl_lo >= bl-1): its coefficients are zero in the reference and here.  The
input has every l < B filled (including l = 0, 1), so that the scaling part
and the lowest scales carry signal.
"""
import numpy as np
import pytest

from oracle import oracle as O
from s2dw_b200 import core
from s2dw_b200.workload import transform_setup

CASES = [(2, 1, 2.0), (2, 2, 2.0), (3, 3, 1.5), (6, 4, 1.2), (7, 5, 1.25)]


def _flm(B, seed):
    r = np.random.default_rng(seed)
    f = np.zeros((B, B), complex, order="F")
    for l in range(B):
        f[l, 0] = r.standard_normal()
        for m in range(1, l + 1):
            f[l, m] = r.standard_normal() + 1j * r.standard_normal()
    return f


@pytest.mark.gpu
@pytest.mark.parametrize("B,N,alpha", CASES, ids=[f"B{b}-N{n}-a{a}" for b, n, a in CASES])
def test_tiny_sizes_and_empty_scales(B, N, alpha):
    t = transform_setup(B, N, alpha)
    J, bs = t["J"], t["bl_scoeff"]
    empty = [j for j in range(J + 1) if core.band_limits(j, B, alpha)[1] >= core.band_limits(j, B, alpha)[0] - 1]
    assert empty, "the case must contain an empty scale"
    f = _flm(B, 10 * B + N)
    a = (t["K_gamma"], t["Slm"], J, B, N, bs, alpha)
    w, sc = core.s2dw_core_analysis_flm2wav_dynamic(f, *a)
    wr, scr = O.analysis_dynamic(f, *a)
    top = max(np.abs(x).max() for x in wr)
    for j, (x, r) in enumerate(zip(w, wr)):
        scale = np.abs(r).max()
        if j in empty:
            assert scale == 0.0 and np.abs(x).max() == 0.0, f"scale {j} should be empty"
        else:
            assert np.abs(x - r).max() <= 1e-12 * max(scale, top * 1e-3), f"scale {j}"
    np.testing.assert_array_equal(sc, scr)
    ws, scs = core.s2dw_core_analysis_flm2wav(f, *a)
    for j, x in enumerate(w):
        np.testing.assert_array_equal(ws[j, :x.shape[0], :x.shape[1], :], x)
    s = (t["K_gamma"], t["Phi2"], t["Slm"], J, B, N, bs, alpha)
    fg = core.s2dw_core_synthesis_wav2flm_dynamic([x.copy(order="F") for x in wr], scr, *s)
    fo = O.synthesis_dynamic([x.copy(order="F") for x in wr], scr, *s)
    assert np.abs(fg - fo).max() <= 1e-12 * np.abs(fo).max()
    np.testing.assert_array_equal(core.s2dw_core_synthesis_wav2flm(ws, scs, *s), core.s2dw_core_synthesis_wav2flm_dynamic(
        [x.copy(order="F") for x in w], sc, *s))
    assert np.abs(fg - f).max() <= 1e-10
