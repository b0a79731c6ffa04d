"""Initial guesses of the pressure of every corrector and of the potential
(Simulation(extrapolate_guesses=...)): polynomial extrapolations of the last results (a fixed
degree, or the degree that predicted the last result best) and the Galerkin projection onto
the span of the last results. A guess changes only where the Krylov iteration starts, so the
fields agree with the default run's to the solver tolerance, and the solves take fewer
iterations."""
import pytest
import torch

import phipict_b200 as pb
from cases import duct_3d, hartmann_2d, seeded_state


def _run(extrapolate, steps: int = 8):
    dom = duct_3d(16, 12, 12, 2)
    seeded_state(dom, 31, scale=0.2)
    dom.PrepareSolve()
    tol = pb.SolverTolerance(rtol=1e-10)
    sim = pb.MHDSimulation(dom, 1e-2, torch.tensor(4.0, dtype=torch.float64), torch.tensor([0.0, 1.0, 0.0]),
                           non_orthogonal=False, mixed_precision=True, pressure_use_amg=True,
                           potential_use_preconditioner=True, advection_tol=tol, pressure_tol=tol, potential_tol=tol,
                           pressure_warm_start=True, extrapolate_guesses=extrapolate)
    its = 0
    for _ in range(steps):
        assert sim.single_step(), sim.last_error
        its += sum(max(i.innerIterations for i in infos) for tag, infos in sim.solve_report() if tag != "velocity")
    return dom, its


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [True, "adaptive", "projection:6"])
def test_extrapolated_guesses_keep_the_fields(cuda, mode):
    d0, its0 = _run(False)
    d1, its1 = _run(mode)
    for a, b in ((d0._u_block, d1._u_block), (d0.pressureResult, d1.pressureResult), (d0.epotResult, d1.epotResult)):
        assert float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(a)) < 1e-8
    assert its1 < its0, (its0, its1)


def _run_2d(extrapolate, steps: int = 8):
    dom = hartmann_2d(48, 32)
    seeded_state(dom, 5, scale=0.2)
    dom.PrepareSolve()
    tol = pb.SolverTolerance(rtol=1e-10)
    sim = pb.Simulation(dom, 1e-2, non_orthogonal=False, mixed_precision=True, pressure_use_amg=True,
                        advection_tol=tol, pressure_tol=tol, extrapolate_guesses=extrapolate)
    its = 0
    for _ in range(steps):
        assert sim.single_step(), sim.last_error
        its += sum(max(i.innerIterations for i in infos) for tag, infos in sim.solve_report() if tag != "velocity")
    return dom, its


@pytest.mark.gpu
def test_projected_guesses_in_2d(cuda):
    """The 2D stencil product on the projection path: same fields, fewer iterations."""
    d0, its0 = _run_2d(False)
    d1, its1 = _run_2d("projection:8")
    for a, b in ((d0._u_block, d1._u_block), (d0.pressureResult, d1.pressureResult)):
        assert float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(a)) < 1e-8
    assert its1 < its0, (its0, its1)
    import ctypes as ct

    from phipict_b200 import _lib

    N = d1.getTotalSize()
    X = torch.randn(2, (N + 3) // 4 * 4, dtype=torch.float64, device="cuda")
    Y = torch.empty_like(X)
    _lib.call("phb_stencil_apply", ct.byref(d1.desc()), d1._stencil("P").data_ptr(), X.data_ptr(), Y.data_ptr(), 2,
              X.stride(0), _lib.stream_ptr(X.device))
    M = d1.P
    A = torch.sparse_csr_tensor(M.row.to(torch.int64), M.index.to(torch.int64), M.value, size=(N, N))
    for v in range(2):
        ref = torch.mv(A, X[v, :N].contiguous())
        assert float(torch.linalg.vector_norm(Y[v, :N] - ref) / torch.linalg.vector_norm(ref)) < 1e-14


@pytest.mark.gpu
def test_stencil_apply_matches_the_csr_product(cuda):
    """phb_stencil_apply (the products of a projected guess's basis) against torch's CSR
    product of the same pressure and potential matrices, on several vectors at a stride."""
    import ctypes as ct

    from phipict_b200 import _lib

    dom, _ = _run(False, steps=1)
    N = dom.getTotalSize()
    g = torch.Generator(device="cuda").manual_seed(5)
    X = torch.randn(3, N + 40, dtype=torch.float64, device="cuda", generator=g)
    for which, M in (("P", dom.P), ("E", dom.Epot)):
        Y = torch.full_like(X, float("nan"))
        _lib.call("phb_stencil_apply", ct.byref(dom.desc()), dom._stencil(which).data_ptr(), X.data_ptr(),
                  Y.data_ptr(), 3, X.stride(0), _lib.stream_ptr(X.device))
        A = torch.sparse_csr_tensor(M.row.to(torch.int64), M.index.to(torch.int64), M.value, size=(N, N))
        for v in range(3):
            ref = torch.mv(A, X[v, :N].contiguous())
            assert float(torch.linalg.vector_norm(Y[v, :N] - ref) / torch.linalg.vector_norm(ref)) < 1e-14, which
        assert torch.isnan(Y[:, N:]).all()  # nothing past the cells of a row is written


@pytest.mark.gpu
@pytest.mark.parametrize("m,n", [(1, 1000), (12, 442368 // 7), (16, 130)])
def test_projection_gram_matches_torch(cuda, m, n):
    """phb_projection_gram (G = V Y^T, c = V b over padded rows) against torch's products."""
    from phipict_b200 import _lib

    g = torch.Generator(device="cuda").manual_seed(m)
    stride = (n + 3) // 4 * 4 + 4
    V = torch.randn(m, stride, dtype=torch.float64, device="cuda", generator=g)
    Y = torch.randn(m, stride, dtype=torch.float64, device="cuda", generator=g)
    b = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    G = torch.full((m, m), float("nan"), dtype=torch.float64, device="cuda")
    c = torch.full((m,), float("nan"), dtype=torch.float64, device="cuda")
    _lib.call("phb_projection_gram", V.data_ptr(), Y.data_ptr(), b.data_ptr(), m, n, stride, G.data_ptr(), c.data_ptr(),
              _lib.stream_ptr(V.device))
    Gr, cr = V[:, :n] @ Y[:, :n].T, V[:, :n] @ b
    assert float((G - Gr).abs().max()) < 1e-12 * n ** 0.5 * 10, float((G - Gr).abs().max())
    assert float((c - cr).abs().max()) < 1e-12 * n ** 0.5 * 10


@pytest.mark.gpu
def test_projection_solve_matches_a_dense_solve(cuda):
    """phb_projection_solve against torch.linalg.solve on symmetric definite systems of both
    signs, and the coefficient 0 of a row that is linearly dependent on the others."""
    from phipict_b200 import _lib

    g = torch.Generator().manual_seed(2)
    for m in (1, 5, 16):
        for sign in (1.0, -1.0):
            B = torch.randn(m, m, dtype=torch.float64, generator=g)
            G = sign * (B @ B.T + m * torch.eye(m, dtype=torch.float64))
            c = torch.randn(m, dtype=torch.float64, generator=g)
            Gd, cd = G.cuda(), c.cuda()
            a = torch.empty(m, dtype=torch.float64, device="cuda")
            _lib.call("phb_projection_solve", Gd.data_ptr(), cd.data_ptr(), m, 0.0, a.data_ptr(), _lib.stream_ptr(a.device))
            ref = torch.linalg.solve(G, c)
            assert float(torch.linalg.vector_norm(a.cpu() - ref) / torch.linalg.vector_norm(ref)) < 1e-10, (m, sign)
    # a basis whose last row repeats the first: the Gram matrix is singular, the guess stays finite
    V = torch.randn(4, 50, dtype=torch.float64, generator=g)
    V[3] = V[0]
    S = torch.randn(50, 50, dtype=torch.float64, generator=g)
    A = S @ S.T + 50 * torch.eye(50, dtype=torch.float64)
    xs = torch.randn(50, dtype=torch.float64, generator=g)
    b = A @ xs
    G, c = (V @ A @ V.T).contiguous().cuda(), (V @ b).cuda()
    a = torch.empty(4, dtype=torch.float64, device="cuda")
    _lib.call("phb_projection_solve", G.data_ptr(), c.data_ptr(), 4, 1e-13, a.data_ptr(), _lib.stream_ptr(a.device))
    x0 = a.cpu() @ V
    assert torch.isfinite(a).all()
    Q, _ = torch.linalg.qr(V[:3].T)
    best = Q @ torch.linalg.solve(Q.T @ A @ Q, Q.T @ b)
    e = lambda y: float((y - xs) @ A @ (y - xs))  # noqa: E731
    assert e(x0) <= e(best) * (1 + 1e-6), (e(x0), e(best))


def test_extrapolation_reproduces_polynomials():
    """Order m extrapolates a polynomial of degree m in the step index exactly."""
    from phipict_b200.simulation import extrapolate_into, push_history

    for m in (1, 2, 3):
        f = lambda t: 1.0 + 2.0 * t + (0.5 * t * t if m >= 2 else 0.0) + (0.1 * t ** 3 if m >= 3 else 0.0)  # noqa: E731
        hist = []
        x = torch.zeros(1, dtype=torch.float64)
        for t in range(4):
            if t:
                push_history(hist, x, m)
            x = torch.tensor([f(t)], dtype=torch.float64)
        g = x.clone()
        extrapolate_into(g, hist, m)
        assert abs(float(g) - f(4)) < 1e-12, (m, float(g), f(4))


def test_adaptive_order_follows_the_sequence():
    """The adaptive extrapolator's degrees agree with the binomial formula and it picks the
    lowest degree that predicts the last result exactly (ties go to the lower degree)."""
    from phipict_b200.simulation import GuessExtrapolator, extrapolate_into

    ex = GuessExtrapolator(4, adaptive=True)
    seq = [torch.tensor([float(t * t), 3.0 - t * t], dtype=torch.float64) for t in range(8)]
    x = torch.zeros(2, dtype=torch.float64)
    for t, v in enumerate(seq):
        ex.guess(x)
        ex.update(v)
    assert ex.guess(x) and ex.order == 2, ex.order
    assert torch.equal(x, torch.tensor([64.0, 3.0 - 64.0], dtype=torch.float64))
    # backward-difference degrees (the comparison) against the binomial formula (the guess)
    hist = [torch.tensor([float(k) ** 3 + 0.5 * k]) for k in (6, 5, 4, 3)]
    last = torch.tensor([7.0 ** 3 + 3.5])
    ex = GuessExtrapolator(4, adaptive=True)
    ex.last, ex.hist = last.clone(), [h.clone() for h in hist]
    ex._compare(torch.zeros(1, dtype=last.dtype))
    errs = ex._errs[0]
    for m in range(5):
        g = last.clone()
        extrapolate_into(g, hist, m)
        assert abs(float(errs[m]) - abs(float(g))) < 1e-9, (m, float(errs[m]), float(g))
    # an alternating sequence is predicted best by the last value alone
    ex = GuessExtrapolator(4, adaptive=True)
    for t in range(8):
        ex.guess(x)
        ex.update(torch.tensor([1.0 + 0.01 * (-1) ** t, 0.0], dtype=torch.float64))
    ex.guess(x)
    assert ex.order == 0, ex.order


def test_projected_guess_is_the_galerkin_projection():
    """The projection basis (backward differences of the last results) spans the last `size`
    results, and the guess is the A-norm-best combination of them: exact when the new
    solution lies in their span, never worse in the A-norm than the degree-(size-1)
    polynomial extrapolation of the same results."""
    from phipict_b200.simulation import ProjectedGuess, extrapolate_into

    g = torch.Generator().manual_seed(7)
    n = 60
    S = torch.randn(n, n, dtype=torch.float64, generator=g)
    A = S @ S.T + n * torch.eye(n, dtype=torch.float64)

    def apply(M, V, Y, m):
        Y.copy_(V @ M.T)

    ex = ProjectedGuess(4, apply=apply, solve=lambda G, c: torch.linalg.solve(G, c))
    base = torch.randn(3, n, dtype=torch.float64, generator=g)
    sols = [torch.cos(torch.tensor(0.3 * t)) * base[0] + 0.1 * t * base[1] + 0.01 * t * t * base[2]
            for t in range(8)]
    x = torch.zeros(n, dtype=torch.float64)
    assert not ex.guess(x, A, A @ sols[0])
    for t, v in enumerate(sols):
        if t >= 3:  # three results span the three-dimensional solution space
            assert ex.guess(x, A, A @ v)
            assert float(torch.linalg.vector_norm(x - v) / torch.linalg.vector_norm(v)) < 1e-9, t
        ex.update(v)
    # the rows span the last four results
    V = ex.D[: ex.n]
    R = torch.stack(sols[-4:])
    coef = torch.linalg.lstsq(V.T, R.T).solution
    assert float(torch.linalg.vector_norm(V.T @ coef - R.T)) < 1e-10
    # against the cubic extrapolation on a sequence outside any small span
    ex = ProjectedGuess(4, apply=apply, solve=lambda G, c: torch.linalg.solve(G, c))
    hist = []
    seq = [torch.sin(torch.arange(n, dtype=torch.float64) * (0.1 + 0.02 * t)) for t in range(7)]
    for v in seq[:6]:
        ex.update(v)
    b = A @ seq[6]
    ex.guess(x, A, b)
    p = seq[5].clone()
    hist = [seq[4], seq[3], seq[2]]
    extrapolate_into(p, hist, 3)
    e = lambda y: float((y - seq[6]) @ A @ (y - seq[6]))  # noqa: E731
    assert e(x) <= e(p) * (1 + 1e-9), (e(x), e(p))
