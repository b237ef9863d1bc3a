"""Split-precision form (tensor-core int8 digit contractions) against the FP64
form on the same maps, for batches of maps.

Tolerances (the split form's stated bound; its design error is ~1e-11):
analysis, per map and per scale, max|w_split - w_fp64| <= 1e-10 * max|w_fp64|;
synthesis of the same coefficients, max|flm_split - flm_fp64| <= 1e-10 *
max|flm_fp64|; split analysis then split synthesis reconstructs flm within
1e-10.  Cases cover every size of the positive-n set (NP = 1..4), alpha = 3, a
batch larger than one 32-map group, and a batch of one."""
import numpy as np
import pytest

from s2dw_b200.workload import gaussian_flm, transform_setup

TOL_W = 1e-10
TOL_RECON = 1e-10


def _run(B, N, alpha, nmaps, seed0=100):
    import torch

    from s2dw_b200.device import Plan

    t = transform_setup(B, N, alpha)
    J = t["J"]
    plain = Plan(B, N, alpha, J)
    split = Plan(B, N, alpha, J, form=Plan.SPLIT)
    for p in (plain, split):
        p.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
    flms = [gaussian_flm(B, seed=seed0 + k) for k in range(nmaps)]
    d_flm = torch.from_numpy(np.stack([np.ascontiguousarray(f.T) for f in flms])).cuda()
    bs2 = max(1, t["bl_scoeff"] ** 2)
    w_ref = torch.empty((nmaps, plain.wav_size), dtype=torch.float64, device="cuda")
    s_ref = torch.empty((nmaps, bs2), dtype=torch.complex128, device="cuda")
    w_sp = torch.full_like(w_ref, np.nan)
    s_sp = torch.full_like(s_ref, np.nan)
    plain.analysis_batch(d_flm, w_ref, s_ref)
    split.analysis_batch(d_flm, w_sp, s_sp)
    split.check()
    out = torch.empty_like(d_flm)
    out_plain = torch.empty_like(d_flm)
    split.synthesis_batch(w_sp, s_sp, out)
    split.check()
    plain.synthesis_batch(w_sp, s_sp, out_plain)
    torch.cuda.synchronize()
    wr, ws = w_ref.cpu().numpy(), w_sp.cpu().numpy()
    offs = plain.wav_offsets
    worst = 0.0
    for k in range(nmaps):
        for j in range(J + 1):
            a, b = wr[k, offs[j]:offs[j + 1]], ws[k, offs[j]:offs[j + 1]]
            scale = np.abs(a).max()
            if scale == 0:
                assert np.abs(b).max() == 0
                continue
            worst = max(worst, np.abs(a - b).max() / scale)
    np.testing.assert_array_equal(s_sp.cpu().numpy(), s_ref.cpu().numpy())
    recon = max(np.abs(out[k].cpu().numpy().T - flms[k]).max() for k in range(nmaps))
    fs, fp = out.cpu().numpy(), out_plain.cpu().numpy()
    syn = max(np.abs(fs[k] - fp[k]).max() / np.abs(fp[k]).max() for k in range(nmaps))
    plain.close()
    split.close()
    return worst, recon, syn


@pytest.mark.gpu
@pytest.mark.parametrize("B,N,alpha,nmaps", [
    (64, 3, 2.0, 5),    # NP = 2 (n = 0, 2)
    (64, 2, 2.0, 3),    # NP = 1
    (48, 5, 3.0, 4),    # NP = 3
    (64, 8, 2.0, 2),    # NP = 4
    (32, 4, 2.0, 40),   # two map groups
    (96, 4, 2.0, 1),    # one map
])
def test_split_matches_fp64(B, N, alpha, nmaps):
    worst, recon, syn = _run(B, N, alpha, nmaps)
    assert worst <= TOL_W, f"max|dw|/max|w| = {worst:.3e}"
    assert syn <= TOL_W, f"max|dflm|/max|flm| = {syn:.3e}"
    assert recon <= TOL_RECON, f"recon {recon:.3e}"


@pytest.mark.gpu
def test_split_b256_n5():
    """The split-form comparison configuration: B=256, N=5, alpha=2."""
    worst, recon, syn = _run(256, 5, 2.0, 4)
    assert worst <= TOL_W, f"max|dw|/max|w| = {worst:.3e}"
    assert syn <= TOL_W, f"max|dflm|/max|flm| = {syn:.3e}"
    assert recon <= TOL_RECON, f"recon {recon:.3e}"


@pytest.mark.gpu
def test_bounded_wait_gives_up_then_the_plan_recovers():
    """Failure detection without a GPU fault: with a wait limit of 0 every
    split-kernel wait that is not already satisfied gives up at once; the
    kernels drain their own copies and tensor-core operations, free their
    tensor memory and return, and s2dwc_plan_check reports S2DW_ERROR 15
    (once).  The same plan at the default 2 s limit then gives the FP64
    results again, and a second check is clean."""
    import torch

    from s2dw_b200._lib import S2DWError
    from s2dw_b200.device import Plan

    B, N, alpha, nmaps = 64, 4, 2.0, 3
    t = transform_setup(B, N, alpha)
    J = t["J"]
    plain = Plan(B, N, alpha, J)
    split = Plan(B, N, alpha, J, form=Plan.SPLIT)
    for p in (plain, split):
        p.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
    flms = [gaussian_flm(B, seed=300 + k) for k in range(nmaps)]
    d_flm = torch.from_numpy(np.stack([np.ascontiguousarray(f.T) for f in flms])).cuda()
    bs2 = max(1, t["bl_scoeff"] ** 2)
    w_ref = torch.empty((nmaps, plain.wav_size), dtype=torch.float64, device="cuda")
    s_ref = torch.empty((nmaps, bs2), dtype=torch.complex128, device="cuda")
    w_sp = torch.empty_like(w_ref)
    s_sp = torch.empty_like(s_ref)
    plain.analysis_batch(d_flm, w_ref, s_ref)

    split.set_wait_limit(0)
    split.analysis_batch(d_flm, w_sp, s_sp)
    out = torch.empty_like(d_flm)
    split.synthesis_batch(w_ref, s_ref, out)
    with pytest.raises(S2DWError) as e:
        split.check()
    assert e.value.code == 15 and "gave up" in str(e.value)

    split.set_wait_limit(2_000_000_000)
    split.analysis_batch(d_flm, w_sp, s_sp)
    split.check()
    torch.cuda.synchronize()
    wr, ws = w_ref.cpu().numpy(), w_sp.cpu().numpy()
    offs = plain.wav_offsets
    for k in range(nmaps):
        for j in range(J + 1):
            a, b = wr[k, offs[j]:offs[j + 1]], ws[k, offs[j]:offs[j + 1]]
            if np.abs(a).max() > 0:
                assert np.abs(a - b).max() <= TOL_W * np.abs(a).max()
    with pytest.raises(S2DWError):
        split.set_wait_limit(-1)
    plain.close()
    split.close()


@pytest.mark.gpu
def test_split_min_batch_runs_small_batches_in_fp64():
    """s2dwc_plan_set_split_min_batch: a split-form plan runs batches under
    the threshold on the FP64 path (bit-identical to an FP64 plan) and larger
    ones on the tensor cores (within the split bound)."""
    import torch

    from s2dw_b200.device import Plan

    B, N, alpha = 64, 4, 2.0
    t = transform_setup(B, N, alpha)
    J = t["J"]
    plain = Plan(B, N, alpha, J)
    split = Plan(B, N, alpha, J, form=Plan.SPLIT)
    for p in (plain, split):
        p.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
    split.set_split_min_batch(4)
    bs2 = max(1, t["bl_scoeff"] ** 2)
    for nmaps, same in ((2, True), (5, False)):
        flms = [gaussian_flm(B, seed=500 + k) for k in range(nmaps)]
        d_flm = torch.from_numpy(np.stack([np.ascontiguousarray(f.T) for f in flms])).cuda()
        w_ref = torch.empty((nmaps, plain.wav_size), dtype=torch.float64, device="cuda")
        s_ref = torch.empty((nmaps, bs2), dtype=torch.complex128, device="cuda")
        w_sp, s_sp = torch.empty_like(w_ref), torch.empty_like(s_ref)
        plain.analysis_batch(d_flm, w_ref, s_ref)
        split.analysis_batch(d_flm, w_sp, s_sp)
        f_ref, f_sp = torch.empty_like(d_flm), torch.empty_like(d_flm)
        plain.synthesis_batch(w_ref, s_ref, f_ref)
        split.synthesis_batch(w_ref, s_ref, f_sp)
        split.check()
        torch.cuda.synchronize()
        a, b = w_ref.cpu().numpy(), w_sp.cpu().numpy()
        fa, fb = f_ref.cpu().numpy(), f_sp.cpu().numpy()
        if same:
            np.testing.assert_array_equal(a, b)
            np.testing.assert_array_equal(fa, fb)
        else:
            assert not np.array_equal(a, b)
            assert np.abs(a - b).max() <= TOL_W * np.abs(a).max()
            assert np.abs(fa - fb).max() <= TOL_W * np.abs(fa).max()
    plain.close()
    split.close()
