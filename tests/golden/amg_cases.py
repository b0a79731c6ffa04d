"""Cases of the CSR AMG-preconditioned CG (``_C.AMGPCGSolve``), shared by the fixture generator
(make_ref_fields.py --amg, which runs phiPICT's own solver), the CPU oracle tests and the GPU
parity tests.

Each case is a seeded variable-coefficient Poisson matrix on a structured 2-D grid (the shape
of a pressure system), a smoothed-aggregation hierarchy built here with scipy (2x2 aggregates,
one Jacobi smoothing step of the tentative prolongator, R = P^T, Galerkin coarse operators,
the coarsest level's dense pseudo-inverse; the layout of phiPICT's AMGHierarchy.native_levels,
solvers/amg.py:311-369), right-hand sides, start vectors and solver options. Batched cases
hold one operator per environment on a shared pattern, like BatchedAMGHierarchy
(solvers/amg.py:1244-1420).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

# name: grid, environments, per-environment values, Neumann (singular), levels above the
# coarsest, options
CASES = {
    "poisson_f64": dict(nx=48, ny=40, nenv=1, batched=False, neumann=False, nlev=2, dtype="f64", hdtype="f64",
                        opts=dict(maxIterations=200, tolerance=1e-10)),
    "poisson_mixed": dict(nx=48, ny=40, nenv=1, batched=False, neumann=False, nlev=2, dtype="f64", hdtype="f32",
                          opts=dict(maxIterations=200, tolerance=1e-9)),
    "batched_values": dict(nx=32, ny=36, nenv=3, batched=True, neumann=False, nlev=2, dtype="f64", hdtype="f64",
                           warm=True, opts=dict(maxIterations=200, tolerance=1e-6, tolerances=[1e-6, 1e-9, 1e-11])),
    "shared_two_rhs": dict(nx=40, ny=24, nenv=2, batched=False, neumann=False, nlev=1, dtype="f64", hdtype="f64",
                           opts=dict(maxIterations=200, tolerance=1e-10, normalized=False)),
    "neumann_project": dict(nx=32, ny=32, nenv=2, batched=False, neumann=True, nlev=2, dtype="f64", hdtype="f64",
                            opts=dict(maxIterations=300, tolerance=1e-10, projectConstant=True, preSweeps=2,
                                      postSweeps=2, omega=0.8)),
    "best_maxit": dict(nx=48, ny=40, nenv=1, batched=False, neumann=False, nlev=2, dtype="f64", hdtype="f64",
                       warm=True, opts=dict(maxIterations=4, tolerance=1e-30, returnBestResult=True)),
    "poisson_f32": dict(nx=48, ny=40, nenv=2, batched=True, neumann=False, nlev=2, dtype="f32", hdtype="f32",
                        opts=dict(maxIterations=200, tolerance=1e-5)),
}
# cases whose iteration counts must agree exactly with the float64 oracle and phiPICT
EXACT = ("poisson_f64", "batched_values", "shared_two_rhs", "neumann_project", "best_maxit")


def poisson(nx: int, ny: int, coef: np.ndarray, neumann: bool) -> sp.csr_matrix:
    """Finite-volume Poisson operator with face coefficients the harmonic mean of the cell
    coefficients; Dirichlet walls (a ghost value of zero) or homogeneous Neumann walls."""
    n = nx * ny
    idx = np.arange(n).reshape(ny, nx)
    rows, cols, vals = [], [], []
    diag = np.zeros(n)
    for dy, dx in ((0, 1), (1, 0)):
        a = idx[: ny - dy, : nx - dx].ravel()
        b = idx[dy:, dx:].ravel()
        c = coef.ravel()
        w = 2.0 * c[a] * c[b] / (c[a] + c[b])
        rows += [a, b]
        cols += [b, a]
        vals += [-w, -w]
        np.add.at(diag, a, w)
        np.add.at(diag, b, w)
    if not neumann:
        c = coef.ravel()
        for edge in (idx[0, :], idx[-1, :], idx[:, 0], idx[:, -1]):
            np.add.at(diag, edge, 2.0 * c[edge])
    rows.append(np.arange(n))
    cols.append(np.arange(n))
    vals.append(diag)
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    return A


def aggregates(nx: int, ny: int) -> tuple[sp.csr_matrix, int, int]:
    """Tentative prolongator of 2x2 aggregates (n x nc, ones) and the coarse grid size."""
    cx, cy = (nx + 1) // 2, (ny + 1) // 2
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    agg = (j // 2) * cx + (i // 2)
    n = nx * ny
    T = sp.csr_matrix((np.ones(n), (np.arange(n), agg.ravel())), shape=(n, cx * cy))
    return T, cx, cy


def _on_pattern(M: sp.csr_matrix, pattern: sp.csr_matrix) -> np.ndarray:
    """Values of M at the nonzero positions of pattern (in its CSR order)."""
    d = M.toarray()
    r = np.repeat(np.arange(pattern.shape[0]), np.diff(pattern.indptr))
    return d[r, pattern.indices]


def build(name: str) -> dict:
    """Arrays of one case. Returns numpy arrays for AMGPCGSolve's arguments plus the per-
    environment scipy matrices the oracle solves with."""
    c = CASES[name]
    nx, ny, B = c["nx"], c["ny"], c["nenv"]
    seed = sum(ord(ch) for ch in name)
    rng = np.random.default_rng(seed)
    nmat = B if c["batched"] else 1
    coefs = [np.exp(rng.normal(0.0, 0.5, size=(ny, nx))) for _ in range(nmat)]
    A_fine = [poisson(nx, ny, k, c["neumann"]) for k in coefs]
    pattern = A_fine[0]
    for A in A_fine[1:]:
        assert np.array_equal(A.indptr, pattern.indptr) and np.array_equal(A.indices, pattern.indices)
    # shared transfer operators, smoothed with the first environment's operator
    levels_env = [[] for _ in range(B)]
    levels_arr = []
    A_cur = A_fine
    gx, gy = nx, ny
    for _ in range(c["nlev"]):
        T, cx, cy = aggregates(gx, gy)
        A0 = A_cur[0]
        d = A0.diagonal()
        Dinv = sp.diags(1.0 / d)
        lam = np.abs(Dinv @ A0).sum(axis=1).max()  # Gershgorin bound on rho(D^-1 A)
        P = ((sp.identity(A0.shape[0]) - (4.0 / 3.0 / lam) * (Dinv @ A0)) @ T).tocsr()
        P.sort_indices()
        R = P.T.tocsr()
        R.sort_indices()
        coarse = [(R @ A @ P).tocsr() for A in A_cur]
        cpat = (R.__abs__() @ A_cur[0].__abs__() @ P.__abs__()).tocsr()
        cpat.sort_indices()
        for A in A_cur[1:]:
            assert np.array_equal(A.indptr, A_cur[0].indptr) and np.array_equal(A.indices, A_cur[0].indices)
        lvl_vals = [A.data.copy() for A in A_cur]
        dinvs = [1.0 / A.diagonal() for A in A_cur]
        levels_arr.append(dict(
            a_row=A_cur[0].indptr.astype(np.int32), a_col=A_cur[0].indices.astype(np.int32),
            a_val=np.concatenate(lvl_vals), dinv=np.concatenate(dinvs),
            r_row=R.indptr.astype(np.int32), r_col=R.indices.astype(np.int32), r_val=R.data.copy(),
            p_row=P.indptr.astype(np.int32), p_col=P.indices.astype(np.int32), p_val=P.data.copy()))
        for e in range(B):
            m = e if nmat > 1 else 0
            levels_env[e].append((A_cur[m], dinvs[m], R, P))
        A_cur = [sp.csr_matrix((_on_pattern(A, cpat), cpat.indices, cpat.indptr), shape=cpat.shape) for A in coarse]
        gx, gy = cx, cy
    pinvs = [np.linalg.pinv(A.toarray()) for A in A_cur]
    n = nx * ny
    b = rng.normal(size=(B, n))
    x0 = rng.normal(scale=0.1, size=(B, n)) if c.get("warm") else np.zeros((B, n))
    return dict(
        name=name, n=n, nenv=B, dtype=c["dtype"], hdtype=c["hdtype"], opts=dict(c["opts"]),
        row=pattern.indptr.astype(np.int32), col=pattern.indices.astype(np.int32),
        val=np.concatenate([A.data for A in A_fine]),
        levels=levels_arr, pinv=np.stack(pinvs) if nmat > 1 else pinvs[0], b=b, x0=x0,
        A_env=[A_fine[e if nmat > 1 else 0] for e in range(B)], levels_env=levels_env,
        pinv_env=[pinvs[e if nmat > 1 else 0] for e in range(B)],
    )


def oracle_kwargs(case: dict) -> dict:
    """The options of a case in the oracle's names."""
    o = case["opts"]
    return dict(maxit=o["maxIterations"], tol=o["tolerance"], tolerances=o.get("tolerances", ()),
                normalized=o.get("normalized", True), return_best=o.get("returnBestResult", False),
                project=o.get("projectConstant", False), pre=o.get("preSweeps", 1), post=o.get("postSweeps", 1),
                omega=o.get("omega", 2.0 / 3.0))


def torch_args(case: dict, device, torch):
    """AMGPCGSolve's positional arguments and keyword options as torch tensors on device."""
    dt = {"f64": torch.float64, "f32": torch.float32}
    T, H = dt[case["dtype"]], dt[case["hdtype"]]

    def t(a, d):
        return torch.as_tensor(np.ascontiguousarray(a)).to(device=device, dtype=d)

    levels = []
    for lv in case["levels"]:
        levels.append([t(lv["a_row"], torch.int32), t(lv["a_col"], torch.int32), t(lv["a_val"], H),
                       t(lv["dinv"], H), t(lv["r_row"], torch.int32), t(lv["r_col"], torch.int32),
                       t(lv["r_val"], H), t(lv["p_row"], torch.int32), t(lv["p_col"], torch.int32),
                       t(lv["p_val"], H)])
    o = case["opts"]
    kwargs = dict(normalized=o.get("normalized", True), returnBestResult=o.get("returnBestResult", False),
                  projectConstant=o.get("projectConstant", False), preSweeps=o.get("preSweeps", 1),
                  postSweeps=o.get("postSweeps", 1), omega=o.get("omega", 2.0 / 3.0),
                  tolerances=list(o.get("tolerances", [])))
    args = [t(case["row"], torch.int32), t(case["col"], torch.int32), t(case["val"], T), levels,
            t(case["pinv"], H), t(case["b"].ravel(), T), t(case["x0"].ravel(), T),
            int(o["maxIterations"]), float(o["tolerance"])]
    return args, kwargs
