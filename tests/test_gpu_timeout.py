"""The bounded wait of the stage kernel's tensor copies: when a copy never
arrives (a test hook arms the barrier and skips the copy), the kernel gives
up after one second, the step reports FVM_ERR_TIMEOUT, and the context goes
on working once the hook is off and a state is uploaded again. Nothing here
faults or hangs the GPU: the wait is on a barrier that nothing completes."""
import ctypes
import time

import numpy as np
import pytest

from fvm3d import abi, cases
from fvm3d.solver import FvmError, Solver

pytestmark = pytest.mark.gpu


def test_tensor_copy_timeout_is_reported_and_recoverable():
    lib = abi.load_library()
    lib.fvm_test_drop_tensor_copies.argtypes = [ctypes.c_void_p, ctypes.c_int]
    c = cases.isentropic_vortex(N=32, layout="blocks8", precision=abi.PREC_FP32_FLUX, rk_stages=3)
    s = c.apply(Solver(c.config()))
    ref = c.apply(Solver(c.config()))
    ref.step(2)
    s.step(1)  # warm: the plan and graph exist
    assert lib.fvm_test_drop_tensor_copies(s.h, 1) == 0
    t0 = time.perf_counter()
    with pytest.raises(FvmError) as e:
        s.step(1)
    assert e.value.code == 6  # FVM_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 60
    assert lib.fvm_test_drop_tensor_copies(s.h, 0) == 0
    # the context still works: upload the initial state again and compare
    # with an untouched context (the step counter and time differ, the
    # states after the same number of steps from the same state do not)
    fresh = c.apply(Solver(c.config()))
    for b, q in enumerate(c.states):
        s.set_state(b, q)
    s.step(2)
    fresh.step(2)
    for b in range(len(c.blocks)):
        assert np.array_equal(s.get_state(b), fresh.get_state(b))
