"""Pins the CPU restatement of the reference (oracle/) before it is trusted.

The reference (Fortran + FFTW) cannot be built here and ships no golden
vectors, so the oracle is checked against mathematics: high-precision
Wigner-d values, the symmetries the reference's plane fill relies on
(src/mod/s2dw_dl_mod.f90:258-304), orthogonality, the admissibility
condition (src/mod/s2dw_core_mod.f90:285-304) and the reference's own
self-test criterion, exact reconstruction (src/prog/s2dw_test.f90:137-160).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_dl_planes_match_high_precision_values():
    g = np.load(os.path.join(GOLD, "dl_known.npz"))
    small = g["l"] <= 1023
    worst = 0.0
    planes = {}
    for l, a, b, d in zip(g["l"][small], g["a"][small], g["b"][small], g["d"][small]):
        l = int(l)
        if l not in planes:
            planes[l] = O.dl_plane(l)
        worst = max(worst, abs(planes[l][a + l, b + l] - d))
    # The reference's Turok-Bucher planes (log-domain first row, recurrence
    # along the row) reach ~1e-13 absolute error near the plane edges at
    # l ~ 700-1000 (e.g. d^700_{3,700}); the restatement reproduces that.
    assert worst < 2e-13, worst
    # away from l ~ 1000 the planes are accurate to a few 1e-15
    lo = g["l"] <= 64
    err_lo = max(abs(planes[int(l)][a + l, b + l] - d)
                 for l, a, b, d in zip(g["l"][lo], g["a"][lo], g["b"][lo], g["d"][lo]))
    assert err_lo < 1e-14, err_lo


def test_accurate_dl_planes_match_all_high_precision_values():
    """The diagnostic long-double planes (oracle.dl_plane_accurate) agree with
    every 50-digit value up to l = 2047 to the double rounding, where the
    reference's Turok-Bucher planes are off by up to 1.4e-13."""
    g = np.load(os.path.join(GOLD, "dl_known.npz"))
    worst, worst_tb = 0.0, 0.0
    for l in sorted(set(int(x) for x in g["l"])):
        sel = g["l"] == l
        D = O.dl_plane_accurate(l)
        a, b, d = g["a"][sel], g["b"][sel], g["d"][sel]
        worst = max(worst, np.abs(D[a + l, b + l] - d).max())
        if l == 2047:
            T = O.dl_plane(l)
            worst_tb = np.abs(T[a + l, b + l] - d).max()
    assert worst < 1e-16, worst
    assert worst_tb > 1e-13  # the reference algorithm's error the fixture comparison separates


def test_dl_closed_forms_l1_l2():
    s2 = np.sqrt(0.5)
    d1 = O.dl_plane(1)  # d^1(pi/2), rows m' = -1..1, cols m = -1..1
    ref1 = np.array([[0.5, s2, 0.5], [-s2, 0.0, s2], [0.5, -s2, 0.5]])
    np.testing.assert_allclose(d1, ref1, atol=1e-15)
    d2 = O.dl_plane(2)
    # d^2_{00}(pi/2) = -1/2, d^2_{22} = 1/4, d^2_{20} = sqrt(6)/4
    assert abs(d2[2, 2] + 0.5) < 1e-15
    assert abs(d2[4, 4] - 0.25) < 1e-15
    assert abs(d2[4, 2] - np.sqrt(6) / 4) < 1e-15


@pytest.mark.parametrize("l", [5, 64, 300])
def test_dl_symmetries_and_orthogonality(l):
    D = O.dl_plane(l)
    idx = np.arange(-l, l + 1)
    a, b = np.meshgrid(idx, idx, indexing="ij")
    # d_{m'm} = (-1)^{m-m'} d_{mm'}
    np.testing.assert_allclose(D, ((-1.0) ** (b - a)) * D.T, atol=1e-13)
    # at pi/2: d_{m',-m} = (-1)^{l+m'} d_{m'm}
    np.testing.assert_allclose(D[:, ::-1], ((-1.0) ** (l + a)) * D, atol=1e-13)
    np.testing.assert_allclose(D.T @ D, np.eye(2 * l + 1), atol=1e-12)


@pytest.mark.parametrize("B,alpha", [(16, 2.0), (64, 2.0), (81, 3.0), (100, 2.5), (1024, 2.0)])
def test_admissibility(B, alpha):
    J = O.comp_jmax(B, alpha)
    K, P, bs = O.init_kernels(J, B, alpha)
    a, ok = O.admiss(K, P, B, J)
    assert ok
    assert np.abs(a - 1).max() < 1e-12


def test_band_limits_and_jmax():
    assert O.comp_jmax(1024, 2.0) == 10
    assert O.comp_jmax(64, 2.0) == 6
    assert O.comp_jmax(2048, 2.0) == 11
    # scales 0 and 1 both have bl = B; bl_lo = B/alpha^(j+1)
    assert O.band_limits(0, 1024, 2.0) == (1024, 512)
    assert O.band_limits(1, 1024, 2.0) == (1024, 256)
    assert O.band_limits(2, 1024, 2.0) == (512, 128)
    assert O.band_limits(10, 1024, 2.0) == (2, 0)
    assert O.band_limits(3, 1024, 3.0) == (114, 12)


@pytest.mark.parametrize("name", ["oracle_B16_N3_a2", "oracle_B32_N4_a2", "oracle_B27_N2_a3"])
def test_oracle_regression_fixtures(name):
    g = np.load(os.path.join(GOLD, name + ".npz"))
    B, N, alpha, J, bs = int(g["B"]), int(g["N"]), float(g["alpha"]), int(g["J"]), int(g["bl_scoeff"])
    K, P, S = np.asfortranarray(g["K_gamma"]), g["Phi2"], np.asfortranarray(g["Slm"])
    flm = np.asfortranarray(g["flm"])
    wav, sc = O.analysis_dynamic(flm, K, S, J, B, N, bs, alpha)
    for j, w in enumerate(wav):
        np.testing.assert_allclose(w, g[f"wav{j}"], rtol=0, atol=1e-13 * max(1.0, np.abs(g[f"wav{j}"]).max()))
    f2 = O.synthesis_dynamic(wav, sc, K, P, S, J, B, N, bs, alpha)
    np.testing.assert_allclose(f2, g["flm_syn"], rtol=0, atol=1e-14)
    assert np.abs(f2 - flm).max() < 1e-12


@pytest.mark.parametrize("B,N,alpha", [(16, 1, 2.0), (16, 2, 2.0), (24, 3, 2.0), (32, 4, 2.0),
                                       (27, 5, 3.0), (20, 3, 2.5)])
def test_oracle_reconstructs(B, N, alpha):
    J = O.comp_jmax(B, alpha)
    K, P, bs = O.init_kernels(J, B, alpha)
    S = O.init_directionality(B, N)
    flm = O.test_gen_flm(B - 1, 1)
    wav, sc = O.analysis_dynamic(flm, K, S, J, B, N, bs, alpha)
    f2 = O.synthesis_dynamic(wav, sc, K, P, S, J, B, N, bs, alpha)
    assert np.abs(f2 - flm).max() < 1e-12


def test_static_and_dynamic_layouts_agree():
    B, N, alpha = 16, 3, 2.0
    J = O.comp_jmax(B, alpha)
    K, P, bs = O.init_kernels(J, B, alpha)
    S = O.init_directionality(B, N)
    flm = O.test_gen_flm(B - 1, 1)
    wd, sc = O.analysis_dynamic(flm, K, S, J, B, N, bs, alpha)
    ws, _ = O.analysis_static(flm, K, S, J, B, N, bs, alpha)
    for j, w in enumerate(wd):
        n, nb, _ = w.shape
        np.testing.assert_array_equal(ws[j, :n, :nb, :], w)
    f_d = O.synthesis_dynamic(wd, sc, K, P, S, J, B, N, bs, alpha)
    f_s = O.synthesis_static(ws, sc, K, P, S, J, B, N, bs, alpha)
    np.testing.assert_allclose(f_s, f_d, atol=1e-15)


def test_test_generator_is_deterministic_and_uniform():
    a = O.test_gen_flm(31, 1)
    b = O.test_gen_flm(31, 1)
    np.testing.assert_array_equal(a, b)
    tri = np.tril(np.ones((32, 32), bool))
    assert np.all(a[~tri] == 0)
    assert np.all(a[:, 0].imag == 0)
    v = np.concatenate([a[tri].real, a[tri][a[tri].imag != 0].imag])
    assert np.all(np.abs(v) < 1) and abs(v.mean()) < 0.1


def test_linearity():
    B, N, alpha = 16, 2, 2.0
    J = O.comp_jmax(B, alpha)
    K, P, bs = O.init_kernels(J, B, alpha)
    S = O.init_directionality(B, N)
    f1, f2 = O.test_gen_flm(B - 1, 1), O.test_gen_flm(B - 1, 3) * 0.5
    w1, _ = O.analysis_dynamic(f1, K, S, J, B, N, bs, alpha)
    w2, _ = O.analysis_dynamic(f2, K, S, J, B, N, bs, alpha)
    w3, _ = O.analysis_dynamic(np.asfortranarray(2 * f1 - f2), K, S, J, B, N, bs, alpha)
    for a, b, c in zip(w1, w2, w3):
        np.testing.assert_allclose(c, 2 * a - b, atol=1e-13)


def _np_moments(ws, masks=None):
    """Straight numpy statement of s2dw_stat_moments' formulas."""
    out, status = [], 0
    for j, w in enumerate(ws):
        x = np.asarray(w, dtype=np.float64).ravel(order="F")
        if masks is not None:
            m = np.asarray(masks[j]).ravel(order="F")
            nj = int(round(m.sum()))
            x = (x * m)[np.abs(m - 1.0) < 1e-12]
        else:
            nj = x.size
        mu = x.sum() / nj
        s = x - mu
        v = ((s ** 2).sum() - s.sum() ** 2 / nj) / (nj - 1)
        if v < 1e-12:
            status = 6
            out.append([mu, v, 0, 0, 0, 0])
        else:
            sd = np.sqrt(v)
            out.append([mu, v, (s ** 3).sum() / (nj * sd ** 3), (s ** 4).sum() / (nj * v * v) - 3,
                        (s ** 5).sum() / (nj * sd ** 5), (s ** 6).sum() / (nj * v ** 3) - 15])
    return np.array(out), status


def test_oracle_stat_moments_match_numpy():
    from s2dw_b200 import core

    B, N, alpha = 16, 3, 2.0
    J = core.s2dw_core_comp_Jmax(B, alpha)
    rng = np.random.default_rng(4)
    ws = [np.asfortranarray(rng.standard_normal(core.wav_scale_shape(j, B, N, alpha)) ** 3 + 0.1)
          for j in range(J + 1)]
    st, m, _ = O.stat_moments(ws, J, B, N, alpha)
    ref, st_ref = _np_moments(ws)
    assert st == st_ref == 0
    np.testing.assert_allclose(m, ref, rtol=1e-10, atol=1e-12)
    masks = [np.asfortranarray((rng.random(w.shape) < 0.7).astype(np.float64)) for w in ws]
    st, m, masked = O.stat_moments(ws, J, B, N, alpha, mask=masks)
    ref, _ = _np_moments(ws, masks)
    np.testing.assert_allclose(m, ref, rtol=1e-10, atol=1e-12)
    for w, mk, wm in zip(ws, masks, masked):
        np.testing.assert_array_equal(wm, w * mk)  # masked in place, as the reference


def test_oracle_stat_moments_zero_variance_and_too_few_samples():
    from s2dw_b200 import core

    B, N, alpha = 8, 2, 2.0
    J = core.s2dw_core_comp_Jmax(B, alpha)
    ws = [np.full(core.wav_scale_shape(j, B, N, alpha), 0.25, order="F") for j in range(J + 1)]
    st, m, _ = O.stat_moments(ws, J, B, N, alpha)
    assert st == 6 and np.all(m[:, 2:] == 0) and np.allclose(m[:, 0], 0.25)
    masks = [np.zeros(w.shape, order="F") for w in ws]
    masks[0].flat[0] = 1.0
    st, _, _ = O.stat_moments(ws, J, B, N, alpha, mask=masks)
    assert st == 8
