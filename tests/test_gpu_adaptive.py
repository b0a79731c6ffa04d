"""Adaptive CFL substeps (core/piso_simulation.py:149-216, 4171-4340): the substep sizes follow
the computational-space maximum velocity re-derived before every substep, checked against the
CPU oracle stepped with the sizes the rule gives on the oracle's own state; and per-environment
substeps of a batch equal each environment run alone."""
import numpy as np
import pytest
import torch

import phipict_b200 as pb
from phipict_b200.simulation import _cfl_substep
from cases import duct_3d, hartmann_2d, seeded_state
from oracle.oracle import OracleDomain, OracleSim

pytestmark = pytest.mark.gpu


def host(t):
    return t.detach().cpu().numpy()


def _oracle_max_velocity(od, sim):
    """max |Minv u| over cells and fixed faces, from the oracle's state and metrics."""
    d, n = od.dims, od.n
    u = sim.u.reshape(d, n)
    Minv = od.Tc[:, d * d:2 * d * d].reshape(n, d, d)
    m = np.abs(np.einsum("nij,jn->in", Minv, u)).max()
    for k, (i, f, bd) in enumerate([(i, f, bd) for i, b in enumerate(od.blocks) for f, bd in enumerate(b.getBoundaries())
                                    if type(bd).__name__ == "FixedBoundary"]):
        v = host(bd.getVelocityVarying())[0].reshape(d, -1)
        fr = od.desc[8 + len(od.blocks) * 40 + k * 12:]
        to, fc = int(fr[9]), int(fr[8])
        Mf = od.Tf[to:to + fc, d * d:2 * d * d].reshape(fc, d, d)
        m = max(m, np.abs(np.einsum("nij,jn->in", Mf, v)).max())
    return m


@pytest.mark.parametrize("case", ["hartmann2d", "duct3d"])
def test_adaptive_substeps_match_the_oracle(cuda, case):
    dom = {"hartmann2d": lambda: hartmann_2d(16, 12), "duct3d": lambda: duct_3d(8, 6, 5, 2)}[case]()
    seeded_state(dom, 7, scale=0.3, base=(2.0,))
    dom.PrepareSolve()
    od = OracleDomain(dom)
    tol = pb.SolverTolerance(rtol=1e-12, atol=1e-14)
    T, CFL = 0.08, 0.5
    ref = OracleSim(od, host(dom._u_block).reshape(-1), T, float(dom.viscosity[0]), advection_tol=tol, pressure_tol=tol)
    sim = pb.Simulation(dom, T, substeps="ADAPTIVE", adaptive_CFL=CFL, non_orthogonal=False, advection_tol=tol,
                        pressure_tol=tol)
    assert sim.single_step(), sim.last_error
    torch.cuda.synchronize()
    remaining, n = T, 0
    while remaining > 0 and not np.isclose(remaining, 0):
        ts, _ = _cfl_substep(remaining, np.float64(_oracle_max_velocity(od, ref)), CFL)
        remaining -= ts
        ref.dt = float(ts)
        ref.step()
        n += 1
    assert n > 1 and sim.adaptive_substeps == n
    u = host(dom._u_block).reshape(-1)
    assert np.abs(u - ref.u).max() <= 1e-9 * np.abs(ref.u).max()


def test_per_environment_substeps_equal_each_environment_alone(cuda):
    envs = [(1, 1.0), (2, 4.0)]  # (seed, velocity scale) per environment

    def make(chosen):
        dom = duct_3d(8, 6, 5, 2, batch=len(chosen))
        for i, b in enumerate(dom.getBlocks()):
            v = torch.empty(b.velocity.shape, dtype=torch.float64)
            for e, (seed, scale) in enumerate(chosen):
                g = torch.Generator().manual_seed(1000 * i + seed)
                ve = 0.3 * torch.randn(v.shape[1:], generator=g, dtype=torch.float64)
                ve[0] += 1.5
                v[e] = scale * ve
            b.velocity.copy_(v.to("cuda"))
        dom.PrepareSolve()
        return dom

    tol = pb.SolverTolerance(rtol=1e-12, atol=1e-14)
    kw = dict(substeps="ADAPTIVE", adaptive_CFL=0.5, non_orthogonal=False, advection_tol=tol, pressure_tol=tol)
    both = make(envs)
    sim = pb.Simulation(both, 0.06, **kw)
    counts = []
    for _ in range(2):
        assert sim.single_step(), sim.last_error
        counts.append(list(sim.adaptive_substeps_per_env))
    assert counts[0][0] != counts[0][1]  # the faster environment needs more substeps
    assert sim.total_time == pytest.approx(0.12)
    for e in range(2):
        alone = make([envs[e]])
        sa = pb.Simulation(alone, 0.06, **kw)
        for k in range(2):
            assert sa.single_step(), sa.last_error
            assert sa.adaptive_substeps == counts[k][e]
        torch.cuda.synchronize()
        assert np.array_equal(host(alone._u_block)[0], host(both._u_block)[e])
        assert np.array_equal(host(alone._p_block)[0], host(both._p_block)[e])
