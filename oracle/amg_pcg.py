"""CPU restatement of phiPICT's native AMG-preconditioned CG (TEST INFRASTRUCTURE ONLY).

The solver behind ``_C.AMGPCGSolve`` (csrc/phipict/bindings.cpp:764-776), restated in numpy
float64 one environment at a time:

- driver and V-cycle: csrc/phipict/solvers/krylov/krylov.cu:1390-1546
  (kPresmoothResidual 1248, kJacobiSweep 1271, kLevelResidual 1292, kSpmvRect 1308,
  kCoarseSolve 1350, kMean 1364, kSubtractMean 1380);
- the start residual and its stop test: kResidual, krylov.cu:292-360 (CG stops before its
  first iteration only on a non-finite or exactly zero residual);
- (r, z) and beta: kCgDots, krylov.cu:572-590;
- the direction, q = A p and alpha: kCgDirection, krylov.cu:428-500;
- the update and the stop tests: kCgUpdate, krylov.cu:502-561 (RISING_CUTOFF 100,
  krylov.cu:125; the best iterate is stored lazily before the next update);
- the reported results and the best-iterate restore: collectResults, krylov.cu:958-980, and
  kRestoreBest, krylov.cu:370-374.

Only tests/ import this module; the CUDA solver never calls it.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

RUNNING, CONVERGED, NONFINITE, MAXIT, RISING = 0, 1, 2, 3, 4
RISING_CUTOFF = 100


@dataclass
class Info:
    finalResidual: float
    usedIterations: int
    converged: bool
    isFiniteResidual: bool
    status: int


def vcycle(levels, pinv, r, omega, pre, post, project):
    """z = M r for one environment (krylov.cu:1449-1512). levels: [(A, dinv, R, P)], A/R/P
    scipy CSR matrices; pinv: dense inverse of the coarsest operator."""
    shift = r.mean() if project else 0.0
    L = len(levels)
    xs, bs = [], []
    bl = r - shift
    for A, dinv, R, _ in levels:
        x = omega * dinv * bl
        for _ in range(1, max(1, pre)):
            x = x + omega * dinv * (bl - A @ x)
        res = bl - A @ x
        xs.append(x)
        bs.append(bl)
        bl = R @ res
    xc = pinv @ bl
    for l in range(L - 1, -1, -1):
        A, dinv, _, P = levels[l]
        coarse = xs[l + 1] if l + 1 < L else xc
        x = xs[l] + P @ coarse
        for _ in range(max(1, post)):
            x = x + omega * dinv * (bs[l] - A @ x)
        xs[l] = x
    z = xs[0]
    if project:
        z = z - z.mean()
    return z


def pcg_one(A, levels, pinv, b, x0, *, maxit, tol, normalized=True, return_best=False, project=False,
            pre=1, post=1, omega=2.0 / 3.0):
    """Solve one environment; returns (x, Info)."""
    n = A.shape[0]
    ns = 1.0 / math.sqrt(n) if normalized else 1.0
    b = np.asarray(b, dtype=np.float64).copy()
    x = np.asarray(x0, dtype=np.float64).copy()
    if project:
        b -= b.mean()
    r = b - A @ x
    crit = float(np.linalg.norm(r)) * ns
    state, it, used = RUNNING, 0, 0
    if not math.isfinite(crit):
        state = NONFINITE
    elif crit == 0.0:
        state = CONVERGED
    restart, rho, beta = True, 0.0, 0.0
    best, best_it, rising, last = math.inf, -1, 0, 0.0
    save_best, xbest = False, None
    p = np.zeros(n)
    while state == RUNNING:
        z = vcycle(levels, pinv, r, omega, pre, post, project)
        rz = float(r @ z)
        if not restart:
            beta = rz / rho if rho != 0.0 else math.inf
        rho = rz
        if not (math.isfinite(rho) and math.isfinite(beta)):
            state, used = NONFINITE, it
            break
        p = z if restart else z + beta * p
        q = A @ p
        pq = float(p @ q)
        alpha = rho / pq if pq != 0.0 else math.inf
        restart = False
        if not math.isfinite(alpha):
            state, used = NONFINITE, it
            break
        if save_best:
            xbest = x.copy()
        x = x + alpha * p
        r = r - alpha * q
        crit = float(np.linalg.norm(r)) * ns
        it += 1
        used = it - 1
        save_best = False
        if not math.isfinite(crit):
            state = NONFINITE
            break
        if return_best:
            if crit < best:
                best, best_it, save_best = crit, it - 1, True
            rising = rising + 1 if (it > 1 and crit >= last) else 0
            last = crit
        if crit < tol:
            state = CONVERGED
        elif it >= maxit:
            state = MAXIT
        elif return_best and rising >= RISING_CUTOFF:
            state = RISING
    info = Info(crit, used, state == CONVERGED, math.isfinite(crit), state)
    if return_best and state in (MAXIT, RISING) and best_it >= 0 and best < crit:
        x = xbest
        info.finalResidual, info.usedIterations = best, best_it
    return x, info


def amg_pcg(A_env, levels_env, pinv_env, b, x0, *, maxit, tol, tolerances=(), **kw):
    """All environments: A_env[e], levels_env[e] = [(A, dinv, R, P)], pinv_env[e]; b, x0 [B, n]."""
    B = len(A_env)
    tols = list(tolerances) if len(tolerances) else [tol] * B
    xs, infos = [], []
    for e in range(B):
        x, info = pcg_one(A_env[e], levels_env[e], pinv_env[e], b[e], x0[e], maxit=maxit, tol=tols[e], **kw)
        xs.append(x)
        infos.append(info)
    return np.stack(xs), infos
