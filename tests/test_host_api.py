"""The C-ABI library on the host: it loads, exports every symbol the header
declares, reproduces the reference's kernel tables and reports the
reference's error codes.  No GPU is needed for any of these."""
import ctypes
import os
import re

import numpy as np
import pytest

import s2dw_b200
from oracle import oracle as O
from s2dw_b200 import S2DWError, core
from s2dw_b200._lib import SIGNATURES, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "s2dw_cuda.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(s2dwc_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = lib()
    names = header_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/s2dw_cuda.h but not exported"
        assert n in SIGNATURES, f"{n} has no ctypes signature"
    assert L.s2dwc_version().decode().startswith("s2dw-b200")
    assert os.path.abspath(s2dw_b200.LIB_PATH).startswith(ROOT)


def test_ctypes_signatures_match_header_arity():
    txt = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "s2dw_cuda.h")).read(), flags=re.S)
    protos = {m.group(1): m.group(2) for m in
              re.finditer(r"\b(s2dwc_\w+)\s*\(([^;]*?)\)\s*;", txt, re.S)}
    assert len(protos) >= 25
    for name, params in protos.items():
        n = 0 if params.strip() in ("", "void") else len(params.split(","))
        assert len(SIGNATURES[name][1]) == n, f"{name}: ctypes has {len(SIGNATURES[name][1])} arguments, C has {n}"


@pytest.mark.parametrize("B,alpha", [(64, 2.0), (1024, 2.0), (256, 3.0), (100, 2.5), (2048, 2.0), (7, 2.0)])
def test_kernel_tables_bit_identical_to_oracle(B, alpha):
    J = core.s2dw_core_comp_Jmax(B, alpha)
    assert J == O.comp_jmax(B, alpha)
    K, P, bs = core.s2dw_core_init_kernels(J, B, alpha)
    K2, P2, bs2 = O.init_kernels(J, B, alpha)
    np.testing.assert_array_equal(K, K2)
    np.testing.assert_array_equal(P, P2)
    assert bs == bs2
    a, ok = core.s2dw_core_admiss(K, P, B, J)
    a2, ok2 = O.admiss(K2, P2, B, J)
    np.testing.assert_array_equal(a, a2)
    assert ok == ok2
    for j in range(J + 1):
        assert core.band_limits(j, B, alpha) == O.band_limits(j, B, alpha)


@pytest.mark.parametrize("J_below", [1, 2])
def test_kernel_tables_for_J_below_Jmax(J_below):
    B, alpha = 128, 2.0
    J = core.s2dw_core_comp_Jmax(B, alpha) - J_below
    K, P, bs = core.s2dw_core_init_kernels(J, B, alpha)
    K2, P2, bs2 = O.init_kernels(J, B, alpha)
    np.testing.assert_array_equal(K, K2)
    np.testing.assert_array_equal(P, P2)
    assert bs == bs2 > 1


@pytest.mark.parametrize("B,N", [(64, 1), (64, 3), (64, 8), (33, 5), (8, 8), (512, 4)])
def test_directionality_identical_to_oracle(B, N):
    np.testing.assert_array_equal(core.s2dw_core_init_directionality(B, N), O.init_directionality(B, N))


def test_assimilate_int():
    assert core.s2dw_core_assimilate_int(3.000001) == (True, 3)
    assert core.s2dw_core_assimilate_int(2.999999) == (True, 3)
    assert core.s2dw_core_assimilate_int(2.5) == (False, 0)
    for x in [0.3, 7.0, 1e3 + 1e-7, 12.49999]:
        assert core.s2dw_core_assimilate_int(x) == O.assimilate_int(x)


def test_invalid_sizes_raise_reference_codes():
    with pytest.raises(S2DWError) as e:
        core.s2dw_core_init_kernels(11, 1024, 2.0)  # J > Jmax
    assert e.value.code == 8
    with pytest.raises(S2DWError) as e:
        core.s2dw_core_init_kernels(0, 64, 2.0)  # J < 1
    assert e.value.code == 8
    with pytest.raises(S2DWError) as e:
        core.s2dw_core_init_directionality(4, 8)  # N > B
    assert e.value.code == 8


def test_null_pointers_rejected():
    L = lib()
    assert L.s2dwc_init_kernels(None, None, None, 6, 64, 2.0) == 10
    assert L.s2dwc_analysis_flm2wav_dynamic(None, None, None, None, None, 6, 64, 3, 1, 2.0) == 10
    assert L.s2dwc_synthesis_wav2flm(None, None, None, None, None, None, 6, 64, 3, 1, 2.0) == 10
    assert b"null" in L.s2dwc_last_error_message()


def test_error_strings_follow_reference_table():
    L = lib()
    assert L.s2dwc_error_string(0) == b"No error"
    assert L.s2dwc_error_string(8) == b"Invalid sizes"
    assert L.s2dwc_error_string(13).startswith(b"Admissibility test failed")
    assert L.s2dwc_error_string(15) == b"CUDA runtime error"


def test_wav_scale_sizes():
    B, N, alpha = 1024, 4, 2.0
    J = core.s2dw_core_comp_Jmax(B, alpha)
    total = 0
    for j in range(J + 1):
        shape = core.wav_scale_shape(j, B, N, alpha)
        n = int(np.prod(shape))
        assert lib().s2dwc_wav_scale_size(j, B, N, alpha) == n
        total += n
    assert total == 39122256  # 313 MB of FP64 wavelet coefficients


def test_invalid_sizes_for_transforms_reported_before_any_device_work():
    B, N, alpha = 64, 17, 2.0  # N > 16 is outside the supported range
    J = core.s2dw_core_comp_Jmax(B, alpha)
    K, P, bs = core.s2dw_core_init_kernels(J, B, alpha)
    S = np.zeros((B, N), dtype=np.complex128, order="F")
    with pytest.raises(S2DWError) as e:
        core.s2dw_core_analysis_flm2wav_dynamic(np.zeros((B, B), complex), K, S, J, B, N, bs, alpha)
    assert e.value.code == 8


def _kgamma_pairwise(J, B, alpha):
    """K_gamma of s2dw_core_init_kernels (s2dw_core_mod.f90:97-157) with each
    Simpson level's sum formed pairwise over directly computed sample points
    (numpy's summation order, the order a parallel reduction takes) instead of
    the reference's left-to-right sum over accumulated points."""
    def f(k, bw, lo):
        t = 2.0 * ((k - lo) / (bw - lo)) - 1.0
        return np.exp(-2.0 / (1.0 - t * t)) / k

    def simpson(bw, lo, a, b):
        st = os_ = ost = 0.0
        for j in range(1, 41):
            if j == 1:
                st = 0.5 * (b - a) * (f(a, bw, lo) + f(b, bw, lo))
            else:
                it = 1 << (j - 2)
                dl = (b - a) / it
                st = 0.5 * (st + (b - a) * np.sum(f(a + (np.arange(it) + 0.5) * dl, bw, lo)) / it)
            s = (4.0 * st - ost) / 3.0
            if j > 5 and (abs(s - os_) < 1e-12 * abs(os_) or (s == 0.0 and os_ == 0.0)):
                return s
            os_, ost = s, st
        raise AssertionError("no convergence")

    def snap(x, rnd):
        ok, y = core.s2dw_core_assimilate_int(x)
        return y if ok else int(rnd(x))

    phi2 = np.zeros((J + 2, B))
    for jj in range(J + 2):
        bw = snap(B / alpha ** (jj - 1), np.ceil)
        lo = snap(bw / alpha, np.floor)
        c = simpson(bw, lo, lo + 1e-12, bw - 1e-12)
        for el in range(B):
            phi2[jj, el] = 1.0 if el <= lo else 0.0 if el >= bw else simpson(bw, lo, float(el), bw - 1e-12) / c
    return np.sqrt(np.maximum(phi2[:-1] - phi2[1:], 0.0))


@pytest.mark.parametrize("B", [64, 256])
def test_kernel_tables_need_the_reference_summation_order(B):
    """Why the kernel tables are built on the host in the reference's order:
    K_gamma = sqrt(Phi2_{j-1} - Phi2_j), and in each scale's tails the two
    quadratures nearly cancel, so a reordered sum that changes K_gamma^2 only
    within the quadrature's own tolerance (TOL_QUAD = 1e-12,
    s2dw_types_mod.f90:54) moves K_gamma far beyond the 1e-12 parity bar."""
    J = core.s2dw_core_comp_Jmax(B, 2.0)
    K, _, _ = core.s2dw_core_init_kernels(J, B, 2.0)
    Kp = _kgamma_pairwise(J, B, 2.0)
    assert np.abs(Kp ** 2 - K ** 2).max() <= 1e-12
    assert np.abs(Kp - K).max() > 1e-10
