"""Backend functions that phiPICT's differentiable driver and diagnostics call on ``_C``:
SolveLinear with transposeA, SparseOuterProduct and ComputeVelocityDivergence, against SciPy
and the CPU oracle."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

import phipict_b200 as pb
from phipict_b200 import _C
from cases import duct_3d, hartmann_2d, seeded_state
from oracle.oracle import OracleDomain

pytestmark = pytest.mark.gpu


def host(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_transposed_momentum_solve(cuda, dtype):
    """The momentum matrix is not symmetric: a solve with transposeA=True solves C^T x = b."""
    dom = duct_3d(6, 5, 4, 2, dtype=dtype)
    seeded_state(dom, 7, scale=0.5)
    dom.PrepareSolve()
    ts = torch.tensor([0.05], dtype=torch.float64)
    _C.SetupAdvectionMatrix(dom, ts, 0)
    n = dom.getTotalSize()
    g = torch.Generator().manual_seed(3)
    b = torch.randn(n, generator=g, dtype=torch.float64).to("cuda", dtype)
    x = torch.zeros_like(b)
    tol = 1e-11 if dtype == torch.float64 else 1e-5
    infos = _C.SolveLinear(dom.C, b, x, 2000, tol, useBiCG=True, transposeA=True)
    assert all(i.converged for i in infos)
    od = OracleDomain(dom)
    C = od.csr_matrix(host(dom.C.value.double()))
    ref = spla.spsolve(C.T.tocsc(), host(b.double()))
    err = np.abs(host(x.double()) - ref).max() / np.abs(ref).max()
    assert err < (1e-8 if dtype == torch.float64 else 1e-3)
    # and it is not the untransposed solve
    plain = spla.spsolve(C.tocsc(), host(b.double()))
    assert np.abs(plain - ref).max() / np.abs(ref).max() > 1e-6


def test_sparse_outer_product_plain_and_domain_matrix(cuda):
    g = torch.Generator().manual_seed(5)
    dense = (torch.rand(12, 12, generator=g) < 0.3).double() + torch.eye(12, dtype=torch.float64)
    sp = dense.to_sparse_csr()
    M = pb.CSRmatrix(torch.zeros(sp.values().numel(), dtype=torch.float64, device="cuda"),
                     sp.col_indices().int().cuda(), sp.crow_indices().int().cuda())
    a = torch.randn(12, generator=g, dtype=torch.float64).cuda()
    b = torch.randn(12, generator=g, dtype=torch.float64).cuda()
    _C.SparseOuterProduct(a, b, M)
    expect = (torch.outer(a.cpu(), b.cpu()) * (dense != 0))
    got = torch.sparse_csr_tensor(M.row.long().cpu(), M.index.long().cpu(), M.value.cpu(), (12, 12)).to_dense()
    assert torch.allclose(got, expect, rtol=0, atol=1e-15)
    # a domain matrix: the product lands in its stencil and reads back through the CSR view
    dom = hartmann_2d(6, 5)
    dom.PrepareSolve()
    _C.SetupAdvectionMatrix(dom, torch.tensor([0.01], dtype=torch.float64), 0)
    _C.SetupPressureCorrection(dom, torch.tensor([0.01], dtype=torch.float64))
    n = dom.getTotalSize()
    a = torch.randn(n, generator=g, dtype=torch.float64).cuda()
    b = torch.randn(n, generator=g, dtype=torch.float64).cuda()
    _C.SparseOuterProduct(a, b, dom.P)
    row, col = dom.P.row.long(), dom.P.index.long()
    rows = torch.repeat_interleave(torch.arange(n, device="cuda"), row[1:] - row[:-1])
    assert torch.equal(dom.P.value, a[rows] * b[col])


@pytest.mark.parametrize("case", ["hartmann2d", "duct3d"])
def test_velocity_divergence_matches_oracle(cuda, case):
    dom = hartmann_2d(10, 8) if case == "hartmann2d" else duct_3d(6, 5, 4, 2)
    seeded_state(dom, 2)
    dom.PrepareSolve()
    div = _C.ComputeVelocityDivergence(dom)
    od = OracleDomain(dom)
    u = host(dom._u_block).reshape(-1)
    ref = od.divergence(u)
    assert np.abs(host(div) - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())
    assert np.abs(ref).max() > 1e-3
