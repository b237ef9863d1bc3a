"""Coefficients computed on the GPU go through the wavelet files and back:
analysis -> FITS (and Matlab) file -> read -> synthesis reconstructs the map,
as the reference's s2dw_analysis / s2dw_synthesis programs do through their
files (src/prog/s2dw_analysis.f90:126-138, src/prog/s2dw_synthesis.f90)."""
import numpy as np
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["fits", "matlab"])
def test_analysis_file_synthesis_round_trip(tmp_path, kind):
    from s2dw_b200 import core, fileio
    from s2dw_b200.workload import gaussian_flm, transform_setup

    B, N, alpha = 64, 3, 2.0
    J = core.s2dw_core_comp_Jmax(B, alpha)
    t = transform_setup(B, N, alpha, J)
    flm = gaussian_flm(B, seed=4)
    F = np.asfortranarray(flm)
    wavdyn, sc = core.s2dw_core_analysis_flm2wav_dynamic(F, t["K_gamma"], t["Slm"], J, B, N, t["bl_scoeff"], alpha)
    path = str(tmp_path / ("w.fits" if kind == "fits" else "w.m"))
    write = getattr(fileio, f"s2dw_fileio_{kind}_wav_write")
    read = getattr(fileio, f"s2dw_fileio_{kind}_wav_read")
    write(wavdyn, sc, J, B, N, t["bl_scoeff"], alpha, path)
    w2, sc2, J2, B2, N2, bs2, a2 = read(path)
    assert (J2, B2, N2, bs2, a2) == (J, B, N, t["bl_scoeff"], alpha)
    for a, b in zip(w2, wavdyn):
        np.testing.assert_array_equal(a, b)
    out = core.s2dw_core_synthesis_wav2flm_dynamic(w2, sc2, t["K_gamma"], t["Phi2"], t["Slm"], J2, B2, N2, bs2, a2)
    assert np.abs(out - F).max() < 1e-12
