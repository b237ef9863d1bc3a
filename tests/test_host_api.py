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
