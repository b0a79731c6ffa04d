"""CG without device allocation (phb_cg_solve_noalloc), checked against the workspace CG
(phb_solve_run) through the C ABI.

This entry point is for hosts that cannot give the library device memory: programs that
split the GPU into fixed slices at start-up and forbid later allocation, or plugin hosts
whose allocator the C ABI cannot reach. Its workspace is a static device array inside the
library, shared by all calls, so the test solves twice in a row on the same array: the
second call must not see anything the first one left behind. The file name makes pytest
collect it last."""
import ctypes as ct

import numpy as np
import pytest
import torch

from phipict_b200 import _C, _lib
from phipict_b200.solvers import CG, solver_for
from cases import duct_3d, hartmann_2d, seeded_state

pytestmark = pytest.mark.gpu


def _pressure_system(make, dtype, cuda, seed):
    dom = make(dtype)
    seeded_state(dom, seed, scale=0.2)
    dom.PrepareSolve()
    ts = torch.tensor([0.01], dtype=torch.float64)
    _C.SetupAdvectionMatrix(dom, ts, 0)
    _C.SetupPressureMatrix(dom, ts)
    g = torch.Generator().manual_seed(seed + 1)
    b = torch.randn(dom.getTotalSize() * dom.getBatchSize(), generator=g, dtype=torch.float64).to(dtype).to(cuda)
    b -= b.mean()
    return dom, b


def _noalloc(dom, b, x, tol, maxit=5000):
    t = _lib.PhbTolerance()
    t.mode = 0
    t.atol = tol
    out = (_lib.PhbSolveResult * dom.getBatchSize())()
    rc = _lib.load().phb_cg_solve_noalloc(ct.byref(dom.desc()), _lib.dtype_code(b.dtype), 1, dom._P_st.data_ptr(),
                                          b.data_ptr(), x.data_ptr(), ct.byref(t), maxit, 0, out,
                                          _lib.stream_ptr(dom.getDevice()))
    assert rc == 0, _lib.load().phb_last_error()
    return list(out)


@pytest.mark.parametrize("dtype,make,tol,bar", [
    (torch.float64, lambda dt: duct_3d(8, 6, 5, 2, dtype=dt), 1e-11, 1e-12),
    (torch.float32, lambda dt: hartmann_2d(16, 12, dtype=dt), 1e-5, 1e-5),
])
def test_noalloc_cg_matches_workspace_cg(cuda, dtype, make, tol, bar):
    dom, b = _pressure_system(make, dtype, cuda, 31)
    s = solver_for(dom, CG, dtype, 1, tag="reference-path")
    x_ref = torch.zeros_like(b)
    s.solve(dom._P_st, b, x_ref, tol, 5000)
    ref = s.results()[0]
    assert ref.converged
    for call in range(2):
        x = torch.zeros_like(b)
        out = _noalloc(dom, b, x, tol)
        torch.cuda.synchronize()
        assert out[0].converged, f"call {call}"
        assert out[0].used_iterations == ref.usedIterations
        xr = x_ref.double().cpu().numpy()
        err = float(np.abs(x.double().cpu().numpy() - xr).max() / np.abs(xr).max())
        assert err < bar, f"call {call}: {err}"


def test_noalloc_rejects_sizes_beyond_the_static_array():
    """A descriptor whose workspace exceeds the array is refused before any device work."""
    lib = _lib.load()
    d = _lib.PhbDomain()
    d.dims = 3
    d.dtype = _lib.PHB_F64
    d.ninst = 1
    d.ncells = 64 << 20
    d.ntiles = d.ncells // _lib.TILE
    assert lib.phb_cg_noalloc_bytes(ct.byref(d), _lib.PHB_F64, 1) > _lib.NOALLOC_SCRATCH_BYTES
    t = _lib.PhbTolerance()
    t.mode = 0
    t.atol = 1e-8
    dummy = ct.c_void_p(1)
    rc = lib.phb_cg_solve_noalloc(ct.byref(d), _lib.PHB_F64, 1, dummy, dummy, dummy, ct.byref(t), 10, 0, None, None)
    assert rc == -3
    assert b"scratch" in lib.phb_last_error()
