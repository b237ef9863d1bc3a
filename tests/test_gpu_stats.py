"""Moments of the wavelet coefficients per scale (s2dw_stat_moments) on the
GPU against the oracle: the host drop-in s2dwc_stat_moments (masked and
unmasked, its warning and error codes, in-place masking) and the device batch
entry point s2dwc_plan_stat_moments on coefficients that never leave the GPU.

Tolerances (the sums run in a different order from the reference's):
|d mean| <= 1e-12 (sqrt(var) + 1e-15 |mean|), |d var| <= 1e-12 var + 1e-28,
standardised moments within 1e-9."""
import numpy as np
import pytest

from oracle import oracle as O
from s2dw_b200 import core
from s2dw_b200.workload import gaussian_flm, transform_setup


def _close(m, ref):
    sd = np.sqrt(np.abs(ref[:, 1]))
    scale = sd + 1e-15 * np.abs(ref[:, 0])  # rounding of the mean itself
    assert np.all(np.abs(m[:, 0] - ref[:, 0]) <= 1e-12 * scale + 1e-300), (m[:, 0], ref[:, 0])
    assert np.all(np.abs(m[:, 1] - ref[:, 1]) <= 1e-12 * np.abs(ref[:, 1]) + 1e-28), (m[:, 1], ref[:, 1])
    np.testing.assert_allclose(m[:, 2:], ref[:, 2:], rtol=0, atol=1e-9)


def _wavelets(B, N, alpha, seed):
    t = transform_setup(B, N, alpha)
    w, _ = core.s2dw_core_analysis_flm2wav_dynamic(gaussian_flm(B, seed=seed), t["K_gamma"], t["Slm"], t["J"], B,
                                                   N, t["bl_scoeff"], alpha)
    return t["J"], w


@pytest.mark.gpu
def test_host_stat_moments_match_oracle():
    B, N, alpha = 64, 3, 2.0
    J, w = _wavelets(B, N, alpha, 5)
    st_ref, ref, _ = O.stat_moments(w, J, B, N, alpha)
    out, st = core.s2dw_stat_moments([x.copy(order="F") for x in w], J, B, N, alpha)
    assert st == st_ref
    _close(np.array(out).T, ref)
    rng = np.random.default_rng(2)
    masks = [np.asfortranarray((rng.random(x.shape) < 0.6).astype(np.float64)) for x in w]
    st_ref, ref, masked = O.stat_moments(w, J, B, N, alpha, mask=masks)
    ws = [np.array(x, order="F", copy=True) for x in w]
    out, st = core.s2dw_stat_moments(ws, J, B, N, alpha, wavdyn_mask=masks)
    assert st == st_ref
    _close(np.array(out).T, ref)
    for a, b in zip(ws, masked):
        np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
def test_host_stat_moments_warning_and_error():
    from s2dw_b200._lib import S2DWError

    B, N, alpha = 16, 2, 2.0
    J = core.s2dw_core_comp_Jmax(B, alpha)
    ws = [np.full(core.wav_scale_shape(j, B, N, alpha), -1.5, order="F") for j in range(J + 1)]
    out, st = core.s2dw_stat_moments(ws, J, B, N, alpha)
    assert st == 6
    assert np.allclose(out[0], -1.5) and all(np.all(o == 0) for o in out[2:])
    masks = [np.ones(x.shape, order="F") for x in ws]
    masks[1][...] = 0.0
    with pytest.raises(S2DWError) as ei:
        core.s2dw_stat_moments(ws, J, B, N, alpha, wavdyn_mask=masks)
    assert ei.value.code == 8


@pytest.mark.gpu
def test_device_batched_moments_match_oracle():
    import torch

    from s2dw_b200.device import Plan

    B, N, alpha, n = 128, 4, 2.0, 5
    t = transform_setup(B, N, alpha)
    J = t["J"]
    plan = Plan(B, N, alpha, J)
    plan.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
    d_flm = torch.from_numpy(np.stack([np.ascontiguousarray(gaussian_flm(B, seed=40 + k).T) for k in range(n)])).cuda()
    d_wav = torch.empty((n, plan.wav_size), dtype=torch.float64, device="cuda")
    d_sc = torch.empty((n, max(1, t["bl_scoeff"] ** 2)), dtype=torch.complex128, device="cuda")
    plan.analysis_batch(d_flm, d_wav, d_sc)
    rng = np.random.default_rng(8)
    mask = (rng.random(plan.wav_size) < 0.8).astype(np.float64)
    d_mask = torch.from_numpy(mask).cuda()
    mom = torch.empty((n, J + 1, 6), dtype=torch.float64, device="cuda")
    mom_m = torch.empty_like(mom)
    plan.stat_moments(d_wav, mom)
    plan.stat_moments(d_wav, mom_m, mask=d_mask)
    torch.cuda.synchronize()
    wh, m1, m2 = d_wav.cpu().numpy(), mom.cpu().numpy(), mom_m.cpu().numpy()
    offs = plan.wav_offsets
    for k in range(n):
        w = [wh[k, offs[j]:offs[j + 1]].reshape(core.wav_scale_shape(j, B, N, alpha), order="F")
             for j in range(J + 1)]
        mk = [mask[offs[j]:offs[j + 1]].reshape(core.wav_scale_shape(j, B, N, alpha), order="F")
              for j in range(J + 1)]
        _, ref, _ = O.stat_moments(w, J, B, N, alpha)
        _close(m1[k], ref)
        _, ref, _ = O.stat_moments(w, J, B, N, alpha, mask=mk)
        _close(m2[k], ref)
    plan.close()
