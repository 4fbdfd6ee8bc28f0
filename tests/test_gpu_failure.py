"""Failure detection without a GPU fault: a bounded device wait that runs out
(a counter nothing increments) reports through the status word within its
limit, and the device keeps working afterwards."""
import ctypes
import time

import pytest

from conftest import golden_graph

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_reports(cuda_device):
    from qtensor_b200 import _lib
    lib = _lib.lib()
    _lib.check(lib.qtb_init(0))
    status = ctypes.c_int32(-1)
    t0 = time.perf_counter()
    _lib.check(lib.qtb_selftest_wait_timeout(1 << 14, ctypes.byref(status)))
    assert time.perf_counter() - t0 < 30
    assert status.value == _lib.STATUS_WAIT_TIMEOUT
    # the context is intact: a normal contraction still matches the reference
    from qtensor_b200.engine import QAOAEnergyEngine
    G, w = golden_graph('cfg2')
    eng = QAOAEnergyEngine()
    E = eng.energy_expectation(G, w['gamma'], w['beta'])
    assert abs(E - w['energy']) <= 1e-5 * abs(w['energy'])
    assert eng.compile(G, 3, w['gamma'], w['beta']).plan.device_status() == 0


def test_selftest_rejects_bad_arguments(cuda_device):
    from qtensor_b200 import _lib
    status = ctypes.c_int32(0)
    assert _lib.lib().qtb_selftest_wait_timeout(0, ctypes.byref(status)) == _lib.QTB_ERR_ARG
    assert _lib.lib().qtb_selftest_wait_timeout(16, None) == _lib.QTB_ERR_ARG
