"""GPU checks at the benchmark sizes, where the CPU oracle is too slow to run
whole: parity with the oracle on the scales it finishes in seconds, and
size-independent properties on every scale (analysis -> synthesis
reconstruction, linearity).  Also parity with the committed oracle fixtures.

Tolerances: wavelet coefficients within 1e-12 of the oracle relative to the
scale's max|w|; reconstruction within 1e-10 (plain FP64 form).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from s2dw_b200 import core
from s2dw_b200.workload import gaussian_flm, transform_setup

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["oracle_B16_N3_a2", "oracle_B32_N4_a2", "oracle_B27_N2_a3"])
def test_matches_golden_fixtures(name):
    g = np.load(os.path.join(GOLD, name + ".npz"))
    B, N, alpha, J, bs = int(g["B"]), int(g["N"]), float(g["alpha"]), int(g["J"]), int(g["bl_scoeff"])
    K, P, S = g["K_gamma"], g["Phi2"], g["Slm"]
    wav, sc = core.s2dw_core_analysis_flm2wav_dynamic(g["flm"], K, S, J, B, N, bs, alpha)
    for j, w in enumerate(wav):
        ref = g[f"wav{j}"]
        if np.abs(ref).max() > 0:
            assert _rel(w, ref) <= 1e-12
    f = core.s2dw_core_synthesis_wav2flm_dynamic([g[f"wav{j}"] for j in range(J + 1)], g["scoeff"], K, P, S, J, B,
                                                 N, bs, alpha)
    assert _rel(f, g["flm_syn"]) <= 1e-12


@pytest.mark.gpu
def test_B256_N5_full_parity():
    B, N, alpha = 256, 5, 2.0
    t = transform_setup(B, N, alpha)
    flm = gaussian_flm(B, seed=0)
    a = (t["K_gamma"], t["Slm"], t["J"], B, N, t["bl_scoeff"], alpha)
    s = (t["K_gamma"], t["Phi2"], t["Slm"], t["J"], B, N, t["bl_scoeff"], alpha)
    wav, sc = core.s2dw_core_analysis_flm2wav_dynamic(flm, *a)
    ref, sc_ref = O.analysis_dynamic(flm, *a)
    for j, (w, r) in enumerate(zip(wav, ref)):
        assert _rel(w, r) <= 1e-12, f"scale {j}: {_rel(w, r):.2e}"
    f = core.s2dw_core_synthesis_wav2flm_dynamic(list(ref), sc_ref, *s)
    f_ref = O.synthesis_dynamic(ref, sc_ref, *s)
    assert _rel(f, f_ref) <= 1e-12
    assert np.abs(f - flm).max() <= 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("B,N,alpha,power", [(1024, 4, 2.0, 1.0), (1024, 8, 3.0, 1.0), (2048, 8, 2.0, 1.2),
                                             (700, 3, 2.5, 1.0)])
def test_large_roundtrip_and_small_scale_parity(B, N, alpha, power):
    t = transform_setup(B, N, alpha)
    J = t["J"]
    flm = gaussian_flm(B, seed=1, power=power)
    a = (t["K_gamma"], t["Slm"], J, B, N, t["bl_scoeff"], alpha)
    s = (t["K_gamma"], t["Phi2"], t["Slm"], J, B, N, t["bl_scoeff"], alpha)
    wav, sc = core.s2dw_core_analysis_flm2wav_dynamic(flm, *a)
    # oracle parity on the scales with bl <= 128 (seconds of CPU work)
    checked = 0
    for j in range(J + 1):
        bl, _ = core.band_limits(j, B, alpha)
        if bl <= 128:
            ref = O.analysis_scale(j, flm, t["K_gamma"], t["Slm"], J, B, N, alpha)
            if np.abs(ref).max() > 0:
                assert _rel(wav[j], ref) <= 1e-12, f"scale {j}"
                checked += 1
    assert checked >= 2
    for w in wav:
        assert np.isfinite(w).all()
    f = core.s2dw_core_synthesis_wav2flm_dynamic(wav, sc, *s)
    err = np.abs(f - flm).max()
    assert err <= 1e-10, f"reconstruction error {err:.3e}"


@pytest.mark.gpu
def test_large_linearity():
    B, N, alpha = 1024, 4, 2.0
    t = transform_setup(B, N, alpha)
    a = (t["K_gamma"], t["Slm"], t["J"], B, N, t["bl_scoeff"], alpha)
    f1, f2 = gaussian_flm(B, seed=5), gaussian_flm(B, seed=6)
    w1, _ = core.s2dw_core_analysis_flm2wav_dynamic(f1, *a)
    w2, _ = core.s2dw_core_analysis_flm2wav_dynamic(f2, *a)
    w3, _ = core.s2dw_core_analysis_flm2wav_dynamic(np.asfortranarray(f1 - 2.0 * f2), *a)
    for x, y, z in zip(w1, w2, w3):
        scale = max(np.abs(x).max(), np.abs(y).max(), 1e-300)
        assert np.abs(z - (x - 2.0 * y)).max() <= 1e-12 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("B,N,alpha", [(1024, 4, 2.0), (2048, 2, 2.0), (700, 3, 2.5), (1500, 2, 2.0)])
def test_alpha_prefetch_kernel_identical(B, N, alpha, monkeypatch):
    """The persistent kernels of the synthesis alpha and analysis beta stages
    (next row's input prefetched into shared memory) do the same arithmetic
    as the one-row-per-CTA kernel: wavelets and synthesis agree bit for bit
    (M = 4096 and 8192)."""
    from s2dw_b200.device import Plan

    import torch

    t = transform_setup(B, N, alpha)
    flm = gaussian_flm(B, seed=2)
    d_flm = torch.from_numpy(np.ascontiguousarray(flm.T)).cuda()
    out = {}
    for pf in ("1", "0"):
        monkeypatch.setenv("S2DW_ALPHA_PREFETCH", pf)
        p = Plan(B, N, alpha, t["J"])
        p.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
        w = torch.empty(p.wav_size, dtype=torch.float64, device="cuda")
        sc = torch.empty(max(1, t["bl_scoeff"] ** 2), dtype=torch.complex128, device="cuda")
        f = torch.empty_like(d_flm)
        p.analysis(d_flm, w, sc)
        p.synthesis(w, sc, f)
        torch.cuda.synchronize()
        out[pf] = (w.cpu().numpy(), f.cpu().numpy())
        p.close()
    monkeypatch.setenv("S2DW_ALPHA_PREFETCH", "1")
    Plan(16, 2, 2.0, core.s2dw_core_comp_Jmax(16, 2.0)).close()  # restore the default for later tests
    np.testing.assert_array_equal(out["1"][0], out["0"][0])
    np.testing.assert_array_equal(out["1"][1], out["0"][1])
    assert np.abs(out["1"][1].T - flm).max() <= 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("B,N", [(1024, 4), (2048, 2)])
def test_prime_factor_alpha_matches_bluestein(B, N, monkeypatch):
    """At bl = 256, 512, 1024 and 2048 the alpha stages run as prime-factor
    DFTs (S2DW_PFA=1, the default): 511 = 7*73 and 2047 = 23*89 with Rader's
    algorithm for the prime factor, 1023 = 3*11*31, 4095 = 5*7*9*13;
    S2DW_PFA=0 runs them as Bluestein convolutions of 1024 to 8192 points
    (B=1024 has scales with bl = 256, 512 and 1024, B=2048 also 2048).  Both are the same transform, so
    the coefficients of every scale and the synthesised flm agree to
    rounding (1e-13 relative)."""
    import torch

    from s2dw_b200.device import Plan

    alpha = 2.0
    t = transform_setup(B, N, alpha)
    flm = gaussian_flm(B, seed=5, power=1.2)
    d_flm = torch.from_numpy(np.ascontiguousarray(flm.T)).cuda()
    out = {}
    for pf in ("1", "0"):
        monkeypatch.setenv("S2DW_PFA", pf)
        p = Plan(B, N, alpha, t["J"])
        p.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
        w = torch.empty(p.wav_size, dtype=torch.float64, device="cuda")
        sc = torch.empty(max(1, t["bl_scoeff"] ** 2), dtype=torch.complex128, device="cuda")
        f = torch.empty_like(d_flm)
        p.analysis(d_flm, w, sc)
        p.synthesis(w, sc, f)
        torch.cuda.synchronize()
        out[pf] = (w.cpu().numpy(), f.cpu().numpy(), p.wav_offsets)
        p.close()
    monkeypatch.setenv("S2DW_PFA", "1")
    Plan(16, 2, 2.0, core.s2dw_core_comp_Jmax(16, 2.0)).close()  # restore the default for later tests
    offs = out["1"][2]
    for j in range(t["J"] + 1):
        a, b = out["1"][0][offs[j]:offs[j + 1]], out["0"][0][offs[j]:offs[j + 1]]
        if np.abs(b).max() > 0:
            assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max(), j
    fa, fb = out["1"][1], out["0"][1]
    assert np.abs(fa - fb).max() <= 1e-13 * np.abs(fb).max()
    assert np.abs(fa.T - flm).max() <= 1e-10 * np.abs(flm).max()
