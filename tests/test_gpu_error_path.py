"""GPU: the bounded waits of the tile kernel give up and report instead of
hanging.  fpho_patch_set_test_stall makes every staging wait expect 16 bytes
that no copy delivers; the evaluation must return FPHO_ERR_KERNEL with the
error word set, and, with the stall switched off, the same handle must
evaluate correctly again (the context stays usable).  Nothing faults or
hangs: each wait ends after its bounded spin."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_and_recovers():
    import ctypes
    from forcepho_b200 import _lib
    from forcepho_b200.proposal import GPUProposer
    P, prop, d = load_golden("single_seed1")
    P.send_to_device()
    h = P.device_patch.handle
    good = GPUProposer().evaluate_proposal(prop, patch=P)
    _lib.call("fpho_patch_set_test_stall", h, 1)
    with pytest.raises(_lib.FphoError) as exc:
        GPUProposer().evaluate_proposal(prop, patch=P)
    assert exc.value.code == 6  # FPHO_ERR_KERNEL
    w = ctypes.c_int()
    _lib.call("fpho_patch_error_word", h, ctypes.byref(w))
    assert w.value & 1
    _lib.call("fpho_patch_set_test_stall", h, 0)
    again = GPUProposer().evaluate_proposal(prop, patch=P)
    np.testing.assert_array_equal(again[0], good[0])
    np.testing.assert_array_equal(again[1], good[1])
    _lib.call("fpho_patch_error_word", h, ctypes.byref(w))
    assert w.value == 0
    P.free()


def test_stall_refused_where_unsafe():
    from forcepho_b200 import _lib, synth
    P = synth.make_workload("field20", seed=0)
    P.send_to_device()
    with pytest.raises(_lib.FphoError):      # 900 Gaussians per exposure > one stage
        _lib.call("fpho_patch_set_test_stall", P.device_patch.handle, 1)
    P.free()
