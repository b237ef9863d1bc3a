"""More than 16 scales (J > 15): alpha close to 1 gives J = 16, 20 and 30 at
B = 64, 32 and 16 (s2dw_core_comp_Jmax, s2dw_core_mod.f90:1365-1376).  The
analysis, the synthesis (whose scale sum takes every scale's band limits as
kernel arguments) and the moments per scale (s2dw_stat_mod.f90:81-275) match
the oracle; the transform reconstructs."""
import numpy as np
import pytest

from oracle import oracle as O
from s2dw_b200 import core
from s2dw_b200.workload import gaussian_flm, transform_setup

CASES = [(64, 4, 1.3), (32, 3, 1.2), (16, 2, 1.1)]


@pytest.mark.gpu
@pytest.mark.parametrize("B,N,alpha", CASES, ids=[f"B{b}-N{n}-a{a}" for b, n, a in CASES])
def test_many_scales_match_oracle(B, N, alpha):
    t = transform_setup(B, N, alpha)
    J, bs = t["J"], t["bl_scoeff"]
    assert J > 15
    f = gaussian_flm(B, seed=B)
    a = (t["K_gamma"], t["Slm"], J, B, N, bs, alpha)
    w, sc = core.s2dw_core_analysis_flm2wav_dynamic(f, *a)
    wr, scr = O.analysis_dynamic(f, *a)
    assert len(w) == J + 1
    top = max(np.abs(x).max() for x in wr)
    for j, (x, r) in enumerate(zip(w, wr)):
        assert np.abs(x - r).max() <= 1e-12 * max(np.abs(r).max(), top * 1e-3), f"scale {j}"
    np.testing.assert_array_equal(sc, scr)
    s = (t["K_gamma"], t["Phi2"], t["Slm"], J, B, N, bs, alpha)
    fg = core.s2dw_core_synthesis_wav2flm_dynamic([x.copy(order="F") for x in wr], scr, *s)
    fo = O.synthesis_dynamic([x.copy(order="F") for x in wr], scr, *s)
    assert np.abs(fg - fo).max() <= 1e-12 * np.abs(fo).max()
    assert np.abs(fg - f).max() <= 1e-10
    st_ref, ref, _ = O.stat_moments(wr, J, B, N, alpha)
    out, st = core.s2dw_stat_moments([x.copy(order="F") for x in wr], J, B, N, alpha)
    assert st == st_ref
    m = np.array(out).T
    sd = np.sqrt(np.abs(ref[:, 1]))
    assert np.all(np.abs(m[:, 0] - ref[:, 0]) <= 1e-12 * (sd + 1e-15 * np.abs(ref[:, 0])) + 1e-300)
    assert np.all(np.abs(m[:, 1] - ref[:, 1]) <= 1e-12 * np.abs(ref[:, 1]) + 1e-28)
    np.testing.assert_allclose(m[:, 2:], ref[:, 2:], rtol=0, atol=1e-9)
