"""s2dwc_plan_analysis_noalloc (workspace in the library's static device
scratch) gives the results of s2dwc_plan_analysis (workspace in the plan), on
two calls in a row, and rejects plans larger than its scratch.

The file name sorts last so that the test also runs after every other GPU test
in one process; it passes alone in a fresh process as well, where its first
call performs the scratch lookup."""
import numpy as np
import pytest

from s2dw_b200.workload import gaussian_flm, transform_setup

# Both paths run the same kernels on the same inputs, so the results are
# expected to be identical; the test allows 1e-14 relative to max|w|.
TOL = 1e-14


def _device_inputs(plan, t, B, seed):
    import torch

    flm = gaussian_flm(B, seed=seed)
    d_flm = torch.from_numpy(np.ascontiguousarray(flm.T)).cuda()
    d_wav = torch.empty(plan.wav_size, dtype=torch.float64, device="cuda")
    d_sc = torch.empty(max(1, t["bl_scoeff"] ** 2), dtype=torch.complex128, device="cuda")
    return d_flm, d_wav, d_sc


@pytest.mark.gpu
@pytest.mark.parametrize("B,N,alpha", [(64, 3, 2.0), (256, 5, 2.0), (96, 8, 3.0)])
def test_noalloc_matches_plan_analysis_twice(B, N, alpha):
    import torch

    from s2dw_b200.device import Plan

    t = transform_setup(B, N, alpha)
    plan = Plan(B, N, alpha, t["J"])
    plan.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
    for call, seed in enumerate((11, 12)):  # two calls in a row, different maps
        d_flm, d_ref, d_sc_ref = _device_inputs(plan, t, B, seed)
        d_wav = torch.full_like(d_ref, np.nan)
        d_sc = torch.full_like(d_sc_ref, np.nan)
        plan.analysis(d_flm, d_ref, d_sc_ref)
        plan.analysis_noalloc(d_flm, d_wav, d_sc)
        torch.cuda.synchronize()
        ref, got = d_ref.cpu().numpy(), d_wav.cpu().numpy()
        scale = np.abs(ref).max()
        err = np.abs(got - ref).max() / scale
        assert np.isfinite(got).all(), f"call {call}: non-finite output"
        assert err <= TOL, f"call {call}: max|dw|/max|w| = {err:.3e}"
        np.testing.assert_array_equal(d_sc.cpu().numpy(), d_sc_ref.cpu().numpy())
    plan.close()


@pytest.mark.gpu
def test_noalloc_rejects_plans_beyond_the_scratch():
    from s2dw_b200._lib import S2DWError
    from s2dw_b200.device import Plan

    B, N, alpha = 512, 4, 2.0  # needs 16 (512*512 + 3*4*512^2) B = 54.5 MB > 32 MiB
    t = transform_setup(B, N, alpha)
    plan = Plan(B, N, alpha, t["J"])
    plan.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
    d_flm, d_wav, d_sc = _device_inputs(plan, t, B, 0)
    with pytest.raises(S2DWError) as ei:
        plan.analysis_noalloc(d_flm, d_wav, d_sc)
    assert ei.value.code == 8 and "static scratch" in str(ei.value)
    plan.close()


def _general_slm(B, N, seed):
    """A complex Slm not of the init_directionality form, on the n the
    transform uses: the analysis then runs its second contraction (the
    imaginary part of S/eta) through the same scratch."""
    rng = np.random.default_rng(seed)
    S = np.zeros((B, N), dtype=np.complex128, order="F")
    for n in range(N):
        if (N + n) % 2 == 1:
            S[n:, n] = rng.standard_normal(B - n) + 1j * rng.standard_normal(B - n)
    return S


@pytest.mark.gpu
@pytest.mark.parametrize("B,N,alpha", [(64, 4, 2.0), (256, 10, 2.0)])
def test_noalloc_general_slm_and_largest_n(B, N, alpha):
    """A random complex Slm at B=64 and the largest N the scratch holds at
    B=256 (N=10: 31 MiB of the 32 MiB), two calls in a row each."""
    import torch

    from s2dw_b200.device import Plan

    t = transform_setup(B, N, alpha)
    S = _general_slm(B, N, seed=B + N) if B == 64 else t["Slm"]
    plan = Plan(B, N, alpha, t["J"])
    plan.set_tables(t["K_gamma"], t["Phi2"], S, t["bl_scoeff"])
    for call, seed in enumerate((21, 22)):
        d_flm, d_ref, d_sc_ref = _device_inputs(plan, t, B, seed)
        d_wav = torch.full_like(d_ref, np.nan)
        d_sc = torch.full_like(d_sc_ref, np.nan)
        plan.analysis(d_flm, d_ref, d_sc_ref)
        plan.analysis_noalloc(d_flm, d_wav, d_sc)
        torch.cuda.synchronize()
        ref, got = d_ref.cpu().numpy(), d_wav.cpu().numpy()
        assert np.isfinite(got).all(), f"call {call}: non-finite output"
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err <= TOL, f"call {call}: max|dw|/max|w| = {err:.3e}"
        np.testing.assert_array_equal(d_sc.cpu().numpy(), d_sc_ref.cpu().numpy())
    plan.close()


@pytest.mark.gpu
def test_noalloc_rejects_split_form_and_n_beyond_the_scratch():
    """The entry point runs the FP64 form only: a split-form plan gets
    S2DW_ERROR_ARG_INVALID (10).  B=256 with N=11 needs 34.6 MB of scratch and
    gets S2DW_ERROR_SIZE_INVALID (8)."""
    from s2dw_b200._lib import S2DWError
    from s2dw_b200.device import Plan

    B, N, alpha = 64, 4, 2.0
    t = transform_setup(B, N, alpha)
    sp = Plan(B, N, alpha, t["J"], form=Plan.SPLIT)
    sp.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
    d_flm, d_wav, d_sc = _device_inputs(sp, t, B, 0)
    with pytest.raises(S2DWError) as ei:
        sp.analysis_noalloc(d_flm, d_wav, d_sc)
    assert ei.value.code == 10 and "FP64 form" in str(ei.value)
    sp.close()

    B, N = 256, 11
    t = transform_setup(B, N, alpha)
    plan = Plan(B, N, alpha, t["J"])
    plan.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
    d_flm, d_wav, d_sc = _device_inputs(plan, t, B, 0)
    with pytest.raises(S2DWError) as ei:
        plan.analysis_noalloc(d_flm, d_wav, d_sc)
    assert ei.value.code == 8
    plan.close()
