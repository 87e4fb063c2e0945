"""fvm_residual_norms: the reference's per-block residual on a device rhs."""
import ctypes

import numpy as np
import pytest

from fvm3d import abi, cases
from fvm3d.solver import Solver

pytestmark = pytest.mark.gpu


def _norms(lib, rhs_host, res0=None):
    import torch

    nk, nj, ni = rhs_host.shape[1:]
    r = torch.from_numpy(np.ascontiguousarray(rhs_host)).cuda()
    out = torch.zeros(6, dtype=torch.float64, device="cuda") if res0 is None else \
        torch.from_numpy(np.array(res0, dtype=np.float64)).cuda()
    nv = (ctypes.c_int64 * 3)(ni, nj, nk)
    torch.cuda.synchronize()
    rc = lib.fvm_residual_norms(ctypes.c_void_p(r.data_ptr()), nv, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_matches_numpy_formula():
    lib = abi.load_library()
    rng = np.random.default_rng(0)
    rhs = rng.normal(size=(5, 7, 9, 11))
    got = _norms(lib, rhs)
    res2 = (rhs ** 2).reshape(5, -1).mean(axis=1)
    np.testing.assert_allclose(got[:5], np.sqrt(res2), rtol=1e-14)
    np.testing.assert_allclose(got[5], np.sqrt(res2.mean()), rtol=1e-14)


def test_accumulates_over_blocks_like_fvm_step():
    lib = abi.load_library()
    c = cases.isentropic_vortex(N=32, layout="blocks8")
    s = c.apply(Solver(c.config(store_rhs=1)))
    t, res_abs, _ = s.step(2)
    acc = np.zeros(6)
    for b in range(8):
        acc = _norms(lib, s.get_rhs(b), acc)
    np.testing.assert_allclose(acc, res_abs, rtol=1e-12)
