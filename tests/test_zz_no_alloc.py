"""fvm_residual_norms_noalloc, the allocation-free residual entry point.

Host codes that hand all GPU memory to their own pool cannot let a library
call cudaMalloc; this entry point serves them from a fixed array inside the
library. It must give the same norms as fvm_residual_norms (which allocates
its scratch per call), call after call, and refuse blocks larger than its
array. This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from fvm3d import abi

pytestmark = pytest.mark.gpu


def _lib():
    lib = abi.load_library()
    for name in ("fvm_residual_norms", "fvm_residual_norms_noalloc"):
        f = getattr(lib, name)
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p, ctypes.c_void_p]
    return lib


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    import torch

    lib = _lib()
    rng = np.random.default_rng(42)
    acc_a = torch.zeros(6, dtype=torch.float64, device="cuda")
    acc_b = torch.zeros(6, dtype=torch.float64, device="cuda")
    # two calls in a row, the second on a smaller block so stale partials of
    # the first call sit beyond the planes it reads
    for shape in ((5, 40, 24, 33), (5, 17, 30, 21)):
        rhs = torch.from_numpy(rng.normal(size=shape)).cuda()
        nv = (ctypes.c_int64 * 3)(shape[3], shape[2], shape[1])
        torch.cuda.synchronize()
        assert lib.fvm_residual_norms(ctypes.c_void_p(rhs.data_ptr()), nv, ctypes.c_void_p(acc_a.data_ptr()),
                                      None) == 0
        assert lib.fvm_residual_norms_noalloc(ctypes.c_void_p(rhs.data_ptr()), nv,
                                              ctypes.c_void_p(acc_b.data_ptr()), None) == 0
        torch.cuda.synchronize()
        a, b = acc_a.cpu().numpy(), acc_b.cpu().numpy()
        np.testing.assert_allclose(b, a, rtol=1e-12, atol=0)
        assert np.all(a > 0)


def test_noalloc_rejects_blocks_beyond_its_array():
    import torch

    lib = _lib()
    rhs = torch.zeros(5 * 4097, dtype=torch.float64, device="cuda")
    out = torch.zeros(6, dtype=torch.float64, device="cuda")
    nv = (ctypes.c_int64 * 3)(1, 1, 4097)
    rc = lib.fvm_residual_norms_noalloc(ctypes.c_void_p(rhs.data_ptr()), nv, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1  # FVM_ERR_INVALID
    buf = ctypes.create_string_buffer(256)
    lib.fvm_last_error(None, buf, 256)
    assert b"4096" in buf.value
