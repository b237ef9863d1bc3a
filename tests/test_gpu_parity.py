"""Parity of the CUDA transforms with the CPU restatement of the reference.

Tolerance (plain FP64 form): every wavelet coefficient within 1e-12 of the
oracle relative to max|w| of its scale; synthesised flm within 1e-12
relative to max|flm|; analysis->synthesis reconstruction within 1e-10
(the reference itself reconstructs to ~1e-12).
"""
import numpy as np
import pytest

from oracle import oracle as O
from s2dw_b200 import core
from s2dw_b200.workload import gaussian_flm, transform_setup

TOL = 1e-12
RECON_TOL = 1e-10

CASES = [
    # (B, N, alpha, J or None for Jmax)
    (8, 1, 2.0, None),
    (16, 2, 2.0, None),
    (32, 3, 2.0, None),
    (64, 3, 2.0, None),     # the reference's own CPU-runnable configuration
    (48, 4, 2.0, None),     # B not a power of two
    (64, 5, 2.0, 3),        # J below Jmax
    (81, 6, 3.0, None),     # alpha = 3
    (40, 7, 2.5, None),     # non-integer alpha
    (64, 8, 2.0, None),
    (128, 4, 2.0, None),
]


def _ids(c):
    return "B{}-N{}-a{}-J{}".format(*c)


@pytest.fixture(scope="module", params=CASES, ids=_ids)
def case(request):
    B, N, alpha, J = request.param
    t = transform_setup(B, N, alpha, J)
    flm = gaussian_flm(B, seed=B + N)
    return t, flm


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.gpu
def test_analysis_dynamic_matches_oracle(case):
    t, flm = case
    args = (t["K_gamma"], t["Slm"], t["J"], t["B"], t["N"], t["bl_scoeff"], t["alpha"])
    wav, sc = core.s2dw_core_analysis_flm2wav_dynamic(flm, *args)
    wav_ref, sc_ref = O.analysis_dynamic(flm, *args)
    assert len(wav) == t["J"] + 1
    for j, (w, r) in enumerate(zip(wav, wav_ref)):
        assert w.shape == r.shape
        if np.abs(r).max() == 0:
            assert np.abs(w).max() < 1e-300, f"scale {j} should be zero"
        else:
            assert _rel(w, r) <= TOL, f"scale {j}: rel err {_rel(w, r):.3e}"
    np.testing.assert_array_equal(sc, sc_ref)


@pytest.mark.gpu
def test_synthesis_dynamic_matches_oracle(case):
    t, flm = case
    a = (t["K_gamma"], t["Slm"], t["J"], t["B"], t["N"], t["bl_scoeff"], t["alpha"])
    wav_ref, sc_ref = O.analysis_dynamic(flm, *a)
    s = (t["K_gamma"], t["Phi2"], t["Slm"], t["J"], t["B"], t["N"], t["bl_scoeff"], t["alpha"])
    f_ref = O.synthesis_dynamic(wav_ref, sc_ref, *s)
    f = core.s2dw_core_synthesis_wav2flm_dynamic(list(wav_ref), sc_ref, *s)
    assert _rel(f, f_ref) <= TOL, f"rel err {_rel(f, f_ref):.3e}"


@pytest.mark.gpu
def test_roundtrip_reconstructs(case):
    t, flm = case
    a = (t["K_gamma"], t["Slm"], t["J"], t["B"], t["N"], t["bl_scoeff"], t["alpha"])
    s = (t["K_gamma"], t["Phi2"], t["Slm"], t["J"], t["B"], t["N"], t["bl_scoeff"], t["alpha"])
    wav, sc = core.s2dw_core_analysis_flm2wav_dynamic(flm, *a)
    f = core.s2dw_core_synthesis_wav2flm_dynamic(wav, sc, *s)
    err = np.abs(f - flm).max()
    assert err <= RECON_TOL * max(1.0, np.abs(flm).max()), f"reconstruction error {err:.3e}"


@pytest.mark.gpu
def test_static_layout_matches_dynamic():
    B, N, alpha = 32, 3, 2.0
    t = transform_setup(B, N, alpha)
    flm = gaussian_flm(B, seed=7)
    a = (t["K_gamma"], t["Slm"], t["J"], B, N, t["bl_scoeff"], alpha)
    sentinel = np.full((t["J"] + 1, 2 * B - 1, 2 * B, N), 7.25, order="F")
    wav_s, sc = core.s2dw_core_analysis_flm2wav(flm, *a, wav=sentinel)
    wav_d, _ = core.s2dw_core_analysis_flm2wav_dynamic(flm, *a)
    for j, w in enumerate(wav_d):
        n, nb, _ = w.shape
        np.testing.assert_array_equal(wav_s[j, :n, :nb, :], w)
        # outside the scale's region the caller's data is left untouched
        assert np.all(wav_s[j, n:, :, :] == 7.25) and np.all(wav_s[j, :, nb:, :] == 7.25)
    wav_ref, _ = O.analysis_static(flm, *a)
    for j, w in enumerate(wav_d):
        n, nb, _ = w.shape
        r = wav_ref[j, :n, :nb, :]
        assert _rel(w, r) <= TOL
    s = (t["K_gamma"], t["Phi2"], t["Slm"], t["J"], B, N, t["bl_scoeff"], alpha)
    f_s = core.s2dw_core_synthesis_wav2flm(wav_s, sc, *s)
    f_ref = O.synthesis_static(np.where(wav_s == 7.25, 0.0, wav_s), sc, *s)
    assert _rel(f_s, f_ref) <= TOL


@pytest.mark.gpu
def test_reference_self_test_generator():
    """The reference's s2dw_test: uniform(-1,1) flm from ran2_dp (seed 1), N=3,
    alpha=2, J=Jmax, analysis then synthesis; passes below 1e-6
    (src/prog/s2dw_test.f90:67-160)."""
    B, N, alpha = 64, 3, 2.0
    t = transform_setup(B, N, alpha)
    flm = O.test_gen_flm(B - 1, 1)
    a = (t["K_gamma"], t["Slm"], t["J"], B, N, t["bl_scoeff"], alpha)
    s = (t["K_gamma"], t["Phi2"], t["Slm"], t["J"], B, N, t["bl_scoeff"], alpha)
    wav, sc = core.s2dw_core_analysis_flm2wav_dynamic(flm, *a)
    f = core.s2dw_core_synthesis_wav2flm_dynamic(wav, sc, *s)
    err = np.abs(flm - f).max()
    assert err < 1e-6
    assert err < 1e-12


@pytest.mark.gpu
def test_device_plan_matches_host_api():
    import torch

    from s2dw_b200.device import Plan

    B, N, alpha = 64, 4, 2.0
    t = transform_setup(B, N, alpha)
    flm = gaussian_flm(B, seed=3)
    a = (t["K_gamma"], t["Slm"], t["J"], B, N, t["bl_scoeff"], alpha)
    wav_h, sc_h = core.s2dw_core_analysis_flm2wav_dynamic(flm, *a)
    plan = Plan(B, N, alpha, t["J"])
    plan.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
    d_flm = torch.from_numpy(np.ascontiguousarray(flm.T)).cuda()
    d_wav = torch.empty(plan.wav_size, dtype=torch.float64, device="cuda")
    d_sc = torch.empty(t["bl_scoeff"] ** 2, dtype=torch.complex128, device="cuda")
    plan.analysis(d_flm, d_wav, d_sc)
    torch.cuda.synchronize()
    for j in range(t["J"] + 1):
        w = plan.scale_view(d_wav, j).cpu().numpy()  # [g, b, a]
        np.testing.assert_array_equal(w.transpose(2, 1, 0), wav_h[j])
    d_out = torch.empty_like(d_flm)
    plan.synthesis(d_wav, d_sc, d_out)
    torch.cuda.synchronize()
    f = d_out.cpu().numpy().T
    assert np.abs(f - flm).max() < 1e-12
    plan.close()


@pytest.mark.gpu
def test_host_api_pinned_buffers_match_pageable():
    """Page-locked per-scale buffers take the path whose copies overlap the
    scales' kernels; the results are the same as with pageable buffers."""
    import ctypes

    import torch

    from s2dw_b200._lib import check, lib

    B, N, alpha = 128, 4, 2.0
    t = transform_setup(B, N, alpha)
    J, bs = t["J"], t["bl_scoeff"]
    flm = gaussian_flm(B, seed=9)
    a = (t["K_gamma"], t["Slm"], J, B, N, bs, alpha)
    wav_ref, sc_ref = core.s2dw_core_analysis_flm2wav_dynamic(flm, *a)
    dp = ctypes.POINTER(ctypes.c_double)
    shapes = [core.wav_scale_shape(j, B, N, alpha) for j in range(J + 1)]
    wav_p = [torch.empty(s[::-1], dtype=torch.float64, pin_memory=True).numpy().T for s in shapes]
    wptr = (dp * (J + 1))(*[w.ctypes.data_as(dp) for w in wav_p])
    sc = np.zeros((bs, bs), dtype=np.complex128, order="F")
    K = np.asfortranarray(t["K_gamma"])
    S = np.asfortranarray(t["Slm"])
    f = np.asfortranarray(flm)
    check(lib().s2dwc_analysis_flm2wav_dynamic(wptr, sc.ctypes.data_as(dp), f.ctypes.data_as(dp),
                                               K.ctypes.data_as(dp), S.ctypes.data_as(dp), J, B, N, bs, alpha))
    for j in range(J + 1):
        np.testing.assert_array_equal(wav_p[j], wav_ref[j])
    np.testing.assert_array_equal(sc, sc_ref)
    out = torch.empty((B, B), dtype=torch.complex128, pin_memory=True).numpy().T
    P = np.ascontiguousarray(t["Phi2"])
    check(lib().s2dwc_synthesis_wav2flm_dynamic(out.ctypes.data_as(dp), wptr, sc.ctypes.data_as(dp),
                                                K.ctypes.data_as(dp), P.ctypes.data_as(dp), S.ctypes.data_as(dp),
                                                J, B, N, bs, alpha))
    ref = core.s2dw_core_synthesis_wav2flm_dynamic(wav_ref, sc_ref, t["K_gamma"], t["Phi2"], t["Slm"], J, B, N,
                                                   bs, alpha)
    np.testing.assert_array_equal(out, ref)
    assert np.abs(out - flm).max() < 1e-12


def _general_slm(B, N, seed):
    """A complex Slm not of the init_directionality form: S(l,n) = eta (a + i b)
    with both real parts nonzero (random, seeded), on the n the transform uses."""
    rng = np.random.default_rng(seed)
    S = np.zeros((B, N), dtype=np.complex128, order="F")
    for n in range(N):
        if (N + n) % 2 == 1:
            S[n:, n] = rng.standard_normal(B - n) + 1j * rng.standard_normal(B - n)
    return np.asfortranarray(S)


@pytest.mark.gpu
@pytest.mark.parametrize("B,N,alpha", [(32, 3, 2.0), (40, 4, 2.5), (24, 1, 2.0), (32, 8, 3.0)])
def test_general_complex_slm_matches_oracle(B, N, alpha):
    """Any complex Slm (the reference's API accepts one): analysis and
    synthesis against the oracle, whose loops take S as given
    (s2dw_core_mod.f90:417-428, :1228-1253)."""
    t = transform_setup(B, N, alpha)
    S = _general_slm(B, N, seed=B + N)
    flm = gaussian_flm(B, seed=7)
    a = (t["K_gamma"], S, t["J"], B, N, t["bl_scoeff"], alpha)
    s = (t["K_gamma"], t["Phi2"], S, t["J"], B, N, t["bl_scoeff"], alpha)
    wav, sc = core.s2dw_core_analysis_flm2wav_dynamic(flm, *a)
    wav_ref, sc_ref = O.analysis_dynamic(flm, *a)
    for j, (w, r) in enumerate(zip(wav, wav_ref)):
        if np.abs(r).max() > 0:
            assert _rel(w, r) <= TOL, f"scale {j}: rel err {_rel(w, r):.3e}"
    f = core.s2dw_core_synthesis_wav2flm_dynamic(list(wav_ref), sc_ref, *s)
    f_ref = O.synthesis_dynamic(wav_ref, sc_ref, *s)
    assert _rel(f, f_ref) <= TOL, f"synthesis rel err {_rel(f, f_ref):.3e}"


@pytest.mark.gpu
def test_general_slm_device_plan_and_split_rejection():
    """The device plan with a general Slm agrees with the host entry point;
    the no-allocation analysis runs the second contraction too; the split
    form refuses such an Slm (S2DW_ERROR_ARG_INVALID)."""
    import torch

    from s2dw_b200._lib import S2DWError
    from s2dw_b200.device import Plan

    B, N, alpha = 32, 4, 2.0
    t = transform_setup(B, N, alpha)
    S = _general_slm(B, N, seed=3)
    flm = gaussian_flm(B, seed=8)
    wav_h, sc_h = core.s2dw_core_analysis_flm2wav_dynamic(flm, t["K_gamma"], S, t["J"], B, N, t["bl_scoeff"], alpha)
    p = Plan(B, N, alpha, t["J"])
    p.set_tables(t["K_gamma"], t["Phi2"], S, t["bl_scoeff"])
    d_flm = torch.from_numpy(np.ascontiguousarray(flm.T)).cuda()
    w = torch.empty(p.wav_size, dtype=torch.float64, device="cuda")
    w2 = torch.empty_like(w)
    sc = torch.empty(max(1, t["bl_scoeff"] ** 2), dtype=torch.complex128, device="cuda")
    p.analysis(d_flm, w, sc)
    p.analysis_noalloc(d_flm, w2, sc)
    torch.cuda.synchronize()
    wn, wn2 = w.cpu().numpy(), w2.cpu().numpy()
    offs = p.wav_offsets
    for j in range(t["J"] + 1):
        np.testing.assert_array_equal(wn[offs[j]:offs[j + 1]], wav_h[j].ravel(order="F"))
    np.testing.assert_array_equal(wn2, wn)
    p.close()
    sp = Plan(B, N, alpha, t["J"], form=Plan.SPLIT)
    sp.set_tables(t["K_gamma"], t["Phi2"], S, t["bl_scoeff"])
    with pytest.raises(S2DWError) as e:
        sp.analysis_batch(d_flm.reshape(1, B, B), w.reshape(1, -1), sc.reshape(1, -1))
    assert e.value.code == 10
    sp.close()


@pytest.mark.gpu
@pytest.mark.parametrize("B,N,alpha", [(32, 12, 2.0), (24, 16, 2.0), (40, 9, 2.5), (64, 10, 3.0)])
def test_large_n_matches_oracle(B, N, alpha):
    """Azimuthal band limits 8 < N <= 16 (FP64 form): analysis and synthesis
    against the oracle, reconstruction, and a general complex Slm."""
    t = transform_setup(B, N, alpha)
    flm = gaussian_flm(B, seed=N)
    for S in (t["Slm"], _general_slm(B, N, seed=N)):
        a = (t["K_gamma"], S, t["J"], B, N, t["bl_scoeff"], alpha)
        s = (t["K_gamma"], t["Phi2"], S, t["J"], B, N, t["bl_scoeff"], alpha)
        wav, sc = core.s2dw_core_analysis_flm2wav_dynamic(flm, *a)
        wav_ref, sc_ref = O.analysis_dynamic(flm, *a)
        for j, (w, r) in enumerate(zip(wav, wav_ref)):
            if np.abs(r).max() > 0:
                assert _rel(w, r) <= TOL, f"scale {j}: rel err {_rel(w, r):.3e}"
        f = core.s2dw_core_synthesis_wav2flm_dynamic(list(wav_ref), sc_ref, *s)
        f_ref = O.synthesis_dynamic(wav_ref, sc_ref, *s)
        assert _rel(f, f_ref) <= TOL, f"synthesis rel err {_rel(f, f_ref):.3e}"
    a = (t["K_gamma"], t["Slm"], t["J"], B, N, t["bl_scoeff"], alpha)
    s = (t["K_gamma"], t["Phi2"], t["Slm"], t["J"], B, N, t["bl_scoeff"], alpha)
    wav, sc = core.s2dw_core_analysis_flm2wav_dynamic(flm, *a)
    f = core.s2dw_core_synthesis_wav2flm_dynamic(wav, sc, *s)
    assert np.abs(f - flm).max() <= RECON_TOL


@pytest.mark.gpu
def test_n_limits():
    """N up to 16 in the FP64 form, up to 8 in the split form."""
    from s2dw_b200._lib import S2DWError
    from s2dw_b200.device import Plan

    with pytest.raises(S2DWError) as e:
        Plan(64, 17, 2.0, 2)
    assert e.value.code == 8
    with pytest.raises(S2DWError) as e:
        Plan(64, 12, 2.0, 2, form=Plan.SPLIT)
    assert e.value.code == 8
    Plan(64, 16, 2.0, 2).close()


@pytest.mark.gpu
def test_host_api_staged_copies_multichunk():
    """Pageable caller arrays go through the plan's page-locked staging
    buffers in 32 MB chunks, a scale at a time and overlapped with the other
    scales' kernels: at B=512, N=5 each full-band scale (42 MB) spans two
    chunks; the dynamic and the static layouts agree with each other and with
    a page-locked run."""
    import torch

    B, N, alpha = 512, 5, 2.0
    t = transform_setup(B, N, alpha)
    J, bs = t["J"], t["bl_scoeff"]
    flm = gaussian_flm(B, seed=21)
    a = (t["K_gamma"], t["Slm"], J, B, N, bs, alpha)
    s = (t["K_gamma"], t["Phi2"], t["Slm"], J, B, N, bs, alpha)
    wav_d, sc_d = core.s2dw_core_analysis_flm2wav_dynamic(flm, *a)
    wav_s, sc_s = core.s2dw_core_analysis_flm2wav(flm, *a)
    for j, w in enumerate(wav_d):
        np.testing.assert_array_equal(wav_s[j, :w.shape[0], :w.shape[1], :], w)
    pinned = []
    for w in wav_d:
        buf = torch.empty(w.size, dtype=torch.float64, pin_memory=True).numpy().reshape(w.shape, order="F")
        buf[...] = w
        pinned.append(buf)
    f_pageable = core.s2dw_core_synthesis_wav2flm_dynamic([w.copy(order="F") for w in wav_d], sc_d, *s)
    f_pinned = core.s2dw_core_synthesis_wav2flm_dynamic(pinned, sc_d, *s)
    f_static = core.s2dw_core_synthesis_wav2flm(wav_s, sc_s, *s)
    np.testing.assert_array_equal(f_pageable, f_pinned)
    np.testing.assert_array_equal(f_static, f_pinned)
    assert np.abs(f_pinned - flm).max() <= RECON_TOL


@pytest.mark.gpu
def test_host_api_table_changes_take_effect():
    """The host entry points keep the folded tables while the caller passes the
    same K_gamma, Slm and bl_scoeff; a change of any of them (in place, through
    the same array) or of Phi2 gives the result of the new tables, and going
    back gives the first result bit for bit."""
    B, N, alpha = 64, 3, 2.0
    t = transform_setup(B, N, alpha)
    J, bs = t["J"], t["bl_scoeff"]
    flm = gaussian_flm(B, seed=31)
    flm[0, 0] = 0.7  # a nonzero scaling coefficient, so that Phi2 enters the synthesis
    K = np.asfortranarray(t["K_gamma"].copy())
    S = np.asfortranarray(t["Slm"].copy())
    P = t["Phi2"].copy()

    def ana(bsv=bs):
        return core.s2dw_core_analysis_flm2wav_dynamic(flm, K, S, J, B, N, bsv, alpha)

    def syn(w, sc, bsv=bs):
        return core.s2dw_core_synthesis_wav2flm_dynamic([x.copy(order="F") for x in w], sc, K, P, S, J, B, N,
                                                        bsv, alpha)

    wA, scA = ana()
    fA = syn(wA, scA)
    K0 = K.copy()
    K[...] = K0 * 1.25
    wK, _ = ana()
    assert any(not np.array_equal(a, b) for a, b in zip(wA, wK))
    K[...] = K0
    S0 = S.copy()
    S[...] = S0 * (0.5 + 0.25j)
    wS, _ = ana()
    assert any(not np.array_equal(a, b) for a, b in zip(wA, wS))
    S[...] = S0
    w2, sc2 = ana()
    for a, b in zip(wA, w2):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(scA, sc2)
    # Phi2 alone
    P[...] = t["Phi2"] * 2.0
    fP = syn(wA, scA)
    assert not np.array_equal(fA, fP)
    P[...] = t["Phi2"]
    np.testing.assert_array_equal(syn(wA, scA), fA)
    # K changed in place between two syntheses
    K[...] = K0 * 1.25
    fK = syn(wA, scA)
    assert not np.array_equal(fA, fK)
    K[...] = K0
    np.testing.assert_array_equal(syn(wA, scA), fA)
    # bl_scoeff
    wb, scb = ana(bs + 1)
    assert scb.shape == (bs + 1, bs + 1)
    np.testing.assert_array_equal(scb[:bs, :bs], scA)
    w3, sc3 = ana()
    for a, b in zip(wA, w3):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(scA, sc3)


@pytest.mark.gpu
@pytest.mark.parametrize("B,N,alpha,general", [(64, 3, 2.0, False), (128, 4, 2.0, False), (96, 5, 2.0, False),
                                               (128, 8, 2.0, False), (64, 4, 2.0, True)])
def test_mwalk_two_l_kernel_is_bit_identical(B, N, alpha, general, monkeypatch):
    """The synthesis contraction with two l per thread and transposed tables
    (S2DW_MWALK_VARIANT=4, the default for N <= 8) does the same operations
    per (l, m) pair in the same order as the 32-l kernel (variant 0), so the
    synthesised flm is bit-identical (also for a general complex Slm, whose
    second pass reads the tables of b)."""
    import torch

    from s2dw_b200.device import Plan

    t = transform_setup(B, N, alpha)
    J, bs2 = t["J"], max(1, t["bl_scoeff"] ** 2)
    Slm = t["Slm"]
    if general:
        rng = np.random.default_rng(7)
        Slm = np.asfortranarray(Slm + 0.3j * rng.standard_normal(Slm.shape) * (np.abs(Slm) > 0))
    out = {}
    for v in ("0", "4"):
        monkeypatch.setenv("S2DW_MWALK_VARIANT", v)
        p = Plan(B, N, alpha, J)
        p.set_tables(t["K_gamma"], t["Phi2"], Slm, t["bl_scoeff"])
        w = torch.from_numpy(np.random.default_rng(B + N).standard_normal(p.wav_size)).cuda()
        sc = torch.zeros(bs2, dtype=torch.complex128, device="cuda")
        f = torch.empty((B, B), dtype=torch.complex128, device="cuda")
        p.synthesis(w, sc, f)
        torch.cuda.synchronize()
        out[v] = f.cpu().numpy()
        p.close()
    monkeypatch.delenv("S2DW_MWALK_VARIANT")
    Plan(16, 2, 2.0, core.s2dw_core_comp_Jmax(16, 2.0)).close()  # restore the default for later tests
    assert np.abs(out["4"]).max() > 0
    np.testing.assert_array_equal(out["4"], out["0"])
