"""Plan footprints and the plan memory limit, on the host: a plan refused by
the limit fails with S2DW_ERROR_MEM_ALLOC_FAIL (the reference's status for a
failed allocate, s2dw_core_mod.f90:384-385) before any device call, so these
tests run without a GPU."""
import ctypes

import pytest

from s2dw_b200._lib import S2DWError, check, lib
from s2dw_b200.core import s2dw_core_comp_Jmax
from s2dw_b200.device import plan_footprint, set_plan_memory_limit


def test_footprint_grows_with_the_plan():
    small = plan_footprint(64, 3, 2.0, s2dw_core_comp_Jmax(64, 2.0))
    big = plan_footprint(1024, 4, 2.0, s2dw_core_comp_Jmax(1024, 2.0))
    assert 0 < small < big
    # B=1024 N=4: the per-scale workspaces alone (Tb/V N*bl*2bl and Tg
    # N*bl*bl complex values per scale) are at least 16*(2+1)*N*B^2 bytes for
    # each of the two full-band scales
    assert big >= 2 * 16 * 3 * 4 * 1024 ** 2
    assert big < 2 << 30


def test_footprint_rejects_invalid_sizes():
    with pytest.raises(S2DWError) as e:
        plan_footprint(4096, 4, 2.0, 12)
    assert e.value.code == 8
    with pytest.raises(S2DWError) as e:
        plan_footprint(64, 3, 2.0, 6, form=7)
    assert e.value.code == 10


def test_memory_limit_refuses_plan_creation_before_any_device_call():
    B, N, alpha = 64, 3, 2.0
    J = s2dw_core_comp_Jmax(B, alpha)
    need = plan_footprint(B, N, alpha, J)
    h = ctypes.c_void_p()
    set_plan_memory_limit(need - 1)
    try:
        code = lib().s2dwc_plan_create(ctypes.byref(h), B, N, alpha, J, 0, 0)
        assert code == 4, code
        assert not h.value
        msg = lib().s2dwc_last_error_message().decode()
        assert "plan memory limit" in msg and str(need) in msg
        # the host entry points create their plans the same way
        with pytest.raises(S2DWError) as e:
            check(lib().s2dwc_plan_create(ctypes.byref(h), B, N, alpha, J, 1, 0))
        assert e.value.code == 4
    finally:
        set_plan_memory_limit(0)
    with pytest.raises(S2DWError) as e:
        set_plan_memory_limit(-1)
    assert e.value.code == 10
