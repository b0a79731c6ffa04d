"""Multigrid preconditioner on the GPU.

- the coarse operators equal scale * P^T A P of the level above, with P built here on the
  host from the level records (SciPy), on a periodic 2D channel, a connected 3D duct and a
  2D pair joined with rotated axes;
- the coarsest generalised inverse solves consistent coarse systems;
- the V-cycle is a symmetric operator (CG needs one);
- preconditioned CG converges in far fewer iterations than CG, to the same solution, with
  identical results from the host loop, the CUDA graph and the persistent kernel;
- full MHD steps with preconditioned pressure and potential solves stay within 1e-8 of the
  plain FP64 step."""
import ctypes as ct

import numpy as np
import pytest
import scipy.sparse as sp
import torch

import phipict_b200 as pb
from phipict_b200 import _C, _lib
from phipict_b200.amg import AmgHierarchy
from phipict_b200.solvers import CG, refiner_for, solver_for
from cases import duct_3d, hartmann_2d, rotated_pair_2d, seeded_state

pytestmark = pytest.mark.gpu

CASES = {
    "hartmann2d": lambda dt: hartmann_2d(16, 12, dtype=dt),
    "duct3d": lambda dt: duct_3d(8, 6, 5, 2, dtype=dt),
    "rotated2d": lambda dt: rotated_pair_2d(8, dtype=dt),
}


def _pressure_system(dom, seed):
    seeded_state(dom, seed, scale=0.2)
    dom.PrepareSolve()
    ts = torch.tensor([0.01], dtype=torch.float64)
    _C.SetupAdvectionMatrix(dom, ts, 0)
    _C.SetupPressureMatrix(dom, ts)
    g = torch.Generator().manual_seed(seed + 1)
    n = dom.getTotalSize() * dom.getBatchSize()
    b = torch.randn(n, generator=g, dtype=torch.float64).to(dom.getDtype()).to(dom.getDevice())
    b -= b.mean()
    return b


def _dense(level_dom: _lib.PhbDomain, A: torch.Tensor) -> sp.csr_matrix:
    """CSR of a level's stencil through the library's CSR export."""
    lib = _lib.load()
    n = int(level_dom.ncells)
    dev = A.device
    stream = _lib.stream_ptr(dev)
    rowsize = torch.zeros(n, dtype=torch.int32, device=dev)
    assert lib.phb_csr_row_sizes(ct.byref(level_dom), rowsize.data_ptr(), stream) == 0
    row = torch.zeros(n + 1, dtype=torch.int32, device=dev)
    row[1:] = torch.cumsum(rowsize, 0, dtype=torch.int32)
    nnz = int(row[-1])
    col = torch.zeros(nnz, dtype=torch.int32, device=dev)
    perm = torch.zeros(nnz, dtype=torch.int32, device=dev)
    assert lib.phb_csr_pattern(ct.byref(level_dom), row.data_ptr(), col.data_ptr(), perm.data_ptr(), stream) == 0
    val = A.reshape(-1)[perm.long()].double()
    m = sp.csr_matrix((val.cpu().numpy(), col.cpu().numpy(), row.cpu().numpy()), shape=(n, n))
    m.sum_duplicates()
    return m


def _prolongation(fine, coarse, dims) -> sp.csr_matrix:
    """Piecewise-constant P: fine cell -> the coarse cell of its aggregate."""
    fb, cb = fine[0], coarse[0]
    nf = int(fine[2][:, 1].sum())
    nc = int(coarse[2][:, 1].sum())
    rows, cols = [], []
    for i in range(fb.shape[0]):
        fs, cs = fb[i, 0:3], cb[i, 0:3]
        z, y, x = np.meshgrid(np.arange(fs[2]), np.arange(fs[1]), np.arange(fs[0]), indexing="ij")
        p = [x.ravel(), y.ravel(), z.ravel()]
        q = [p[a] // 2 if cs[a] < fs[a] else p[a] for a in range(3)]
        rows.append(fb[i, 3] + p[0] + fs[0] * (p[1] + fs[1] * p[2]))
        cols.append(cb[i, 3] + q[0] + cs[0] * (q[1] + cs[1] * q[2]))
    r, c = np.concatenate(rows), np.concatenate(cols)
    return sp.csr_matrix((np.ones(r.size), (r, c)), shape=(nf, nc))


@pytest.mark.parametrize("case", list(CASES))
def test_coarse_operators_are_scaled_galerkin_products(cuda, case):
    dom = CASES[case](torch.float32)
    _pressure_system(dom, 3)
    h = AmgHierarchy(dom, coarse_cells=4, dense_cells=0)
    h.setup(dom._P_st)
    torch.cuda.synchronize()
    dims = dom.getSpatialDims()
    scale = h.options["coarse_scale"]
    assert h.nlevels >= 3
    for l in range(h.nlevels - 1):
        Af = _dense(h.struct().levels[l].dom, h.level_A[l])
        Ac = _dense(h.struct().levels[l + 1].dom, h.level_A[l + 1])
        P = _prolongation(h.records[l], h.records[l + 1], dims)
        G = (scale * (P.T @ Af @ P)).toarray()
        assert np.abs(Ac.toarray() - G).max() <= 1e-5 * np.abs(G).max(), f"level {l + 1}"
    # the coarsest inverse solves consistent systems: A_c (G A_c y) = A_c y
    L = h.nlevels - 1
    Ac = _dense(h.struct().levels[L].dom, h.level_A[L]).toarray()
    n = Ac.shape[0]
    inv = h.coarse_inv.view(-1, h.coarse_n, h.coarse_n)[0, :n, :n].cpu().numpy()
    y = np.random.default_rng(0).standard_normal(n)
    rhs = Ac @ y
    assert np.abs(Ac @ (inv @ rhs) - rhs).max() <= 1e-8 * np.abs(rhs).max()


@pytest.mark.parametrize("case", ["hartmann2d", "duct3d", "rotated2d"])
def test_folded_levels_give_the_same_cycle(cuda, case):
    """The cycle below the dense level T applied as one dense operator equals running it
    level by level down to the coarsest inverse (float32 roundoff apart)."""
    dom = {"hartmann2d": lambda: hartmann_2d(64, 48, dtype=torch.float32),
           "duct3d": lambda: duct_3d(16, 12, 10, 2, dtype=torch.float32),
           "rotated2d": lambda: rotated_pair_2d(32, dtype=torch.float32)}[case]()
    _pressure_system(dom, 23)
    h0 = AmgHierarchy(dom, dense_cells=0)
    h1 = AmgHierarchy(dom)
    assert h1.tail_level < h1.nlevels - 1 == h0.tail_level, (h1.sizes, h1.tail_level)
    h0.setup(dom._P_st)
    h1.setup(dom._P_st)
    r = torch.randn(dom.getTotalSize(), generator=torch.Generator().manual_seed(4)).cuda()
    z0, z1 = h0.vcycle(r).double(), h1.vcycle(r).double()
    assert float((z0 - z1).abs().max() / z0.abs().max()) < 1e-5


def _host_cycle(h, dims, r):
    """The V-cycle in float64 on the host from the hierarchy's own operators: x0 = S b,
    b' = P^T (b - A x0), e = cycle(b'), x1 = x0 + P e, z = x1 + S (b - A x1), and the dense
    operator C_T (per instance) at the last level of the cycle."""
    T = h.tail_level
    A = [_dense(h.struct().levels[l].dom, h.level_A[l]) for l in range(T + 1)]
    P = [_prolongation(h.records[l], h.records[l + 1], dims) for l in range(T)]
    S = [h.level_wdinv[l].double().cpu().numpy() for l in range(T)]
    cn = h.coarse_n
    insts = h.records[T][2]
    C = h.coarse_inv.view(-1, cn, cn).cpu().numpy()

    def cyc(l, b):
        if l == T:
            x = np.zeros_like(b)
            for i in range(insts.shape[0]):
                off, n = int(insts[i, 0]), int(insts[i, 1])
                x[off:off + n] = C[i, :n, :n] @ b[off:off + n]
            return x
        x0 = S[l] * b
        e = cyc(l + 1, P[l].T @ (b - A[l] @ x0))
        x1 = x0 + P[l] @ e
        return x1 + S[l] * (b - A[l] @ x1)

    return cyc(0, r)


VCYCLE_CASES = {
    "hartmann2d": lambda: hartmann_2d(64, 48, dtype=torch.float32),
    "duct3d": lambda: duct_3d(16, 12, 10, 2, dtype=torch.float32),
    "rotated2d": lambda: rotated_pair_2d(32, dtype=torch.float32),
    "duct3d_odd": lambda: duct_3d(13, 7, 9, 2, dtype=torch.float32),
    # above the size where the finest level switches to the one-coarse-cell-per-thread
    # restriction and the quad prolongation
    "hartmann2d_large": lambda: hartmann_2d(1024, 1040, dtype=torch.float32),
    "duct3d_large": lambda: duct_3d(64, 96, 88, 2, dtype=torch.float32),
}


@pytest.mark.parametrize("case", list(VCYCLE_CASES))
def test_vcycle_matches_host_emulation(cuda, case):
    """The device cycle equals the cycle evaluated with SciPy from the same level operators,
    float32 roundoff apart: per-cell and lane-group forms on small grids; vector, fixed-stride
    and per-cell paths of the finest level on large ones."""
    dom = VCYCLE_CASES[case]()
    _pressure_system(dom, 29)
    h = AmgHierarchy(dom)
    h.setup(dom._P_st)
    r = torch.randn(dom.getTotalSize(), generator=torch.Generator().manual_seed(6)).cuda()
    z = h.vcycle(r).double().cpu().numpy()
    torch.cuda.synchronize()
    ref = _host_cycle(h, dom.getSpatialDims(), r.double().cpu().numpy())
    assert np.abs(z - ref).max() <= 1e-4 * np.abs(ref).max()


@pytest.mark.parametrize("case", ["hartmann2d", "duct3d"])
def test_vcycle_is_symmetric(cuda, case):
    dom = CASES[case](torch.float32)
    _pressure_system(dom, 5)
    h = AmgHierarchy(dom, coarse_cells=8)
    h.setup(dom._P_st)
    g = torch.Generator().manual_seed(7)
    n = dom.getTotalSize()
    u = torch.randn(n, generator=g).cuda()
    v = torch.randn(n, generator=g).cuda()
    Mu = h.vcycle(u).double()
    Mv = h.vcycle(v).double()
    a, b = float(u.double() @ Mv), float(Mu @ v.double())
    assert abs(a - b) <= 1e-4 * max(abs(a), abs(b))
    # positive on this (negative or positive semidefinite) operator's range: same sign as (u, A^-1 u)
    assert float(u.double() @ Mu) != 0.0


@pytest.mark.parametrize("case", ["hartmann2d", "duct3d"])
def test_pcg_converges_faster_to_the_same_solution(cuda, case):
    dom = {"hartmann2d": lambda: hartmann_2d(64, 48, dtype=torch.float32),
           "duct3d": lambda: duct_3d(24, 16, 16, 2, dtype=torch.float32)}[case]()
    b = _pressure_system(dom, 11)
    tol = 1e-5 * float(b.abs().max())
    cg = solver_for(dom, CG, torch.float32, 1, tag="plain")
    x0 = torch.zeros_like(b)
    cg.solve(dom._P_st, b, x0, tol, 20000)
    i0 = cg.results()[0]
    assert i0.converged
    h = AmgHierarchy(dom)
    h.setup(dom._P_st)
    xs, its = [], []
    for mode in (0, 1, 2):
        s = solver_for(dom, CG, torch.float32, 1, tag=f"pcg{mode}")
        x = torch.zeros_like(b)
        s.solve(dom._P_st, b, x, tol, 2000, use_graph=mode, amg=h)
        info = s.results()[0]
        assert info.converged, (mode, info)
        xs.append(x)
        its.append(info.usedIterations)
    # the host loop and the graph launch the same kernels: identical results; the persistent
    # kernel inlines the same per-tile code into one kernel, where the compiler may contract
    # multiply-adds differently: float32 roundoff apart
    assert its[0] == its[1] and torch.equal(xs[0], xs[1])
    assert abs(its[2] - its[1]) <= 1
    assert float((xs[2] - xs[1]).abs().max() / xs[1].abs().max()) < 1e-4
    assert its[2] * 4 < i0.usedIterations, (its, i0.usedIterations)
    d0 = (x0 - x0.mean()).double()
    d1 = (xs[2] - xs[2].mean()).double()
    assert float((d0 - d1).abs().max() / d0.abs().max()) < 1e-3


def test_refined_pcg_matches_fp64_cg(cuda):
    dom = duct_3d(16, 12, 10, 2)
    dom._mixed = True
    b = _pressure_system(dom, 17)
    x64 = torch.zeros_like(b)
    s = solver_for(dom, CG, torch.float64, 1, tag="fp64")
    s.solve(dom._P_st, b, x64, 1e-12, 20000)
    assert s.results()[0].converged
    lo = _C._lo(dom, "P")
    h = AmgHierarchy(dom)
    h.setup(lo)
    r = refiner_for(dom, CG, 1, tag="refined-pcg")
    x = torch.zeros_like(b)
    out = r.solve(dom._P_st, lo, b, x, 1e-12, 1000, fetch=True, amg=h)
    assert out[0].converged, out[0]
    d0 = x64 - x64.mean()
    d1 = x - x.mean()
    assert float((d0 - d1).abs().max() / d0.abs().max()) < 1e-8


def test_mhd_steps_with_multigrid_match_fp64(cuda):
    """Mixed-precision MHD steps with preconditioned pressure and potential solves stay within
    1e-8 of the plain FP64 steps (the bar of the unpreconditioned mixed-precision path)."""
    results = []
    for amg in (False, True):
        dom = duct_3d(16, 12, 10, 2)
        seeded_state(dom, 9, scale=0.1)
        dom.PrepareSolve()
        tol = dict(advection_tol=pb.SolverTolerance(rtol=1e-11), pressure_tol=pb.SolverTolerance(rtol=1e-11))
        sim = pb.MHDSimulation(dom, 0.01, torch.tensor(2.0), torch.tensor([0.0, 1.0, 0.0]), non_orthogonal=False,
                               potential_tol=pb.SolverTolerance(rtol=1e-11), mixed_precision=amg,
                               pressure_use_amg=amg, potential_use_preconditioner=amg, **tol)
        for _ in range(3):
            assert sim.single_step(), sim.last_error
        if amg:
            inner = {t: sum(i.innerIterations for i in infos) for t, infos in sim.solve_report()}
            assert inner["pressure0"] > 0
        results.append((dom._u_block.double().cpu().numpy().copy(), dom.epotResult.double().cpu().numpy().copy()))
    for k in range(2):
        ref = results[0][k]
        assert np.abs(results[1][k] - ref).max() / np.abs(ref).max() < 1e-8


def test_multigrid_needs_float32_or_mixed_precision(cuda):
    dom = duct_3d(8, 6, 5, 2)
    dom.PrepareSolve()
    with pytest.raises(NotImplementedError):
        pb.Simulation(dom, 0.01, non_orthogonal=False, pressure_use_amg=True)
