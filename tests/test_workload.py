"""The seeded synthetic input (s2dw_b200/workload.py gaussian_flm): a real
signal's harmonic coefficients with only m >= 0 stored, flm(l, m) with l
fastest and m <= l; f_00 = f_1m = 0; f_l0 ~ N(0, C_l) real; Re and Im of
f_lm (m > 0) ~ N(0, C_l / 2); C_l = 1/(l(l+1)) or its 1.2 power; numpy's
PCG64 (default_rng(seed)) drawn l-major, then m, Re before Im."""
import numpy as np

from s2dw_b200.workload import gaussian_flm


def test_layout_and_zeros():
    f = gaussian_flm(64, seed=0)
    assert f.shape == (64, 64) and f.dtype == np.complex128 and f.flags.f_contiguous
    assert np.all(f[:2] == 0)
    assert np.all(f.imag[:, 0] == 0)
    assert np.all(f[np.triu_indices(64, 1)] == 0)          # m > l
    assert np.all(f[np.tril_indices(64, 0)][np.tril_indices(64, 0)[0] >= 2] != 0)


def test_seeded_and_draw_order():
    np.testing.assert_array_equal(gaussian_flm(32, seed=5), gaussian_flm(32, seed=5))
    assert not np.array_equal(gaussian_flm(32, seed=5), gaussian_flm(32, seed=6))
    z = np.random.default_rng(3).standard_normal(5 + 7)     # l = 2 then l = 3
    f = gaussian_flm(4, seed=3)
    c2, c3 = 1 / 6.0, 1 / 12.0
    assert f[2, 0] == z[0] * np.sqrt(c2)
    assert f[2, 1] == np.sqrt(c2 / 2) * (z[1] + 1j * z[2])
    assert f[2, 2] == np.sqrt(c2 / 2) * (z[3] + 1j * z[4])
    assert f[3, 0] == z[5] * np.sqrt(c3)
    assert f[3, 3] == np.sqrt(c3 / 2) * (z[10] + 1j * z[11])


def test_power_spectrum():
    B = 1024
    for power in (1.0, 1.2):
        f = gaussian_flm(B, seed=1, power=power)
        l = np.arange(2, B)
        cl = (1.0 / (l * (l + 1.0))) ** power
        # E sum_{m=0..l} |f_lm|^2 = C_l + l C_l
        ratio = (np.abs(f[2:]) ** 2).sum(axis=1) / ((l + 1) * cl)
        assert abs(ratio.mean() - 1.0) < 0.01
