"""The continuous-batching request loop: requests of different grids, Stuart numbers and
magnetic fields join and leave running batches; each request's result must be the result it
gets alone (bitwise on the plain FP64 path: batch membership and the state copies at every
re-pack do not touch an instance's arithmetic)."""
import pytest
import torch

import phipict_b200 as pb
from phipict_b200.serve import Request, Server, poisson_arrivals
from cases import duct_3d, hartmann_2d, seeded_state

pytestmark = pytest.mark.gpu

KW = dict(non_orthogonal=False, advection_tol=pb.SolverTolerance(rtol=1e-12),
          pressure_tol=pb.SolverTolerance(rtol=1e-12), potential_tol=pb.SolverTolerance(rtol=1e-12))


def _builders():
    specs = [(2, (16, 12)), (3, (8, 6, 5, 2)), (2, (24, 10)), (2, (12, 8)), (3, (6, 5, 4, 1)), (2, (20, 16))]
    out = []
    for k, (dims, size) in enumerate(specs):
        def build(k=k, dims=dims, size=size):
            dom = hartmann_2d(*size, nu=0.01 * (1 + k % 3)) if dims == 2 else duct_3d(*size, seed=k)
            seeded_state(dom, 70 + k, scale=0.1)
            dom.PrepareSolve()
            return dom
        out.append(build)
    return out


class _Clock:
    """Deterministic server clock: advances a fixed amount per reading."""
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 0.004
        return self.t


def _requests():
    arrivals = poisson_arrivals(6, 40.0, seed=3)
    reqs = []
    for k, build in enumerate(_builders()):
        reqs.append(Request(rid=k, build=build, stuart=[0.5, 2.0, 1.0, 4.0, 0.25, 1.5][k],
                            e_b=(0.0, 1.0, 0.0) if k % 2 == 0 else (0.0, 0.6, 0.8), steps=3 + (k % 3), dt=0.01,
                            arrival=arrivals[k]))
    return reqs


def test_served_results_equal_results_alone(cuda):
    server = Server(sim_kwargs=KW, clock=_Clock())
    rep = server.run(_requests())
    assert rep["requests"] == 6 and rep["failed"] == 0
    assert rep["p50_s"] is not None and rep["p99_s"] >= rep["p50_s"]
    # membership changed while requests ran: more batch steps than the longest request
    assert rep["batch_steps"] > max(r.steps for r in server.finished)
    for req in sorted(server.finished, key=lambda r: r.rid):
        alone = _requests()[req.rid]
        dom = alone.build()
        sim = pb.MHDSimulation(dom, alone.dt, torch.tensor([alone.stuart], dtype=torch.float64),
                               torch.tensor(alone.e_b, dtype=torch.float64), **KW)
        for _ in range(alone.steps):
            assert sim.single_step()
        assert torch.equal(req.domain._u_block, dom._u_block), req.rid
        assert torch.equal(req.domain.pressureResult, dom.pressureResult), req.rid
        assert torch.equal(req.domain.epotResult, dom.epotResult), req.rid


def test_admission_respects_the_memory_budget(cuda):
    from phipict_b200.serve import estimate_bytes
    reqs = _requests()
    sizes = [estimate_bytes(r.build()) for r in reqs]
    budget = max(sizes) * 1.2
    server = Server(hbm_budget=budget, sim_kwargs=KW, clock=_Clock())
    for r in reqs:
        r.arrival = 0.0
    rep = server.run(reqs)
    assert rep["requests"] == 6 and rep["failed"] == 0
    assert max(sizes) <= rep["peak_held_bytes"] <= budget
    # a request larger than the whole budget is refused, not queued forever
    big = _requests()[1]
    server = Server(hbm_budget=min(sizes), sim_kwargs=KW, clock=_Clock())
    rep = server.run([big])
    assert rep["failed"] == 1 and "budget" in server.finished[0].failed
