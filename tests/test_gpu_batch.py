"""Heterogeneous instance batches (DomainBatch): domains of different grids, viscosities and
Stuart numbers advanced in one launch per kernel and solve.

Every per-instance quantity (reductions, stop decisions, tolerances) is computed over the
instance's own tiles in a fixed order, and a finished system's iterate is frozen while the
others continue, so an instance advanced in a batch gives bitwise the fields it gives alone
on the plain FP64 path. With multigrid the batch's hierarchy depends on its largest
instance, so there the fields agree to the solver tolerance."""
import numpy as np
import pytest
import torch

import phipict_b200 as pb
from cases import duct_3d, hartmann_2d, seeded_state

pytestmark = pytest.mark.gpu

TIGHT = dict(advection_tol=pb.SolverTolerance(rtol=1e-12), pressure_tol=pb.SolverTolerance(rtol=1e-12),
             potential_tol=pb.SolverTolerance(rtol=1e-12))


def _members_2d():
    out = []
    for k, (nx, ny, nu) in enumerate(((16, 12, 0.01), (24, 8, 0.02), (12, 20, 0.005))):
        dom = hartmann_2d(nx, ny, nu=nu)
        seeded_state(dom, 40 + k, scale=0.2)
        dom.PrepareSolve()
        out.append(dom)
    return out


def _members_3d():
    out = []
    for k, (nx, ny, nz, nb) in enumerate(((8, 6, 5, 2), (6, 5, 4, 1), (10, 6, 6, 2))):
        dom = duct_3d(nx, ny, nz, nb, seed=k)
        seeded_state(dom, 50 + k, scale=0.1)
        dom.PrepareSolve()
        out.append(dom)
    return out


def _run(dom, stuart, e_b, steps, **kw):
    sim = pb.MHDSimulation(dom, 0.01, stuart, e_b, non_orthogonal=False, **kw)
    for _ in range(steps):
        assert sim.single_step(), sim.last_error
    return sim


@pytest.mark.parametrize("dims", [2, 3])
def test_batch_equals_instances_alone_fp64(cuda, dims):
    make = _members_2d if dims == 2 else _members_3d
    stuart = torch.tensor([1.0, 4.0, 0.25], dtype=torch.float64)
    e_b = torch.tensor([[0.0, 1.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0] if dims == 3 else [0.0, 1.0, 0.0]],
                       dtype=torch.float64)
    alone = []
    for k, dom in enumerate(make()):
        _run(dom, stuart[k:k + 1], e_b[k], 3, **TIGHT)
        alone.append((dom._u_block.clone(), dom.pressureResult.clone(), dom.epotResult.clone()))
    members = make()
    batch = pb.DomainBatch(members)
    _run(batch, stuart, e_b, 3, **TIGHT)
    batch.scatter()
    for k, dom in enumerate(members):
        u, p, phi = alone[k]
        assert torch.equal(dom._u_block, u), k
        assert torch.equal(dom.pressureResult, p), k
        assert torch.equal(dom.epotResult, phi), k


def test_batch_with_multigrid_matches_alone(cuda):
    stuart = torch.tensor([2.0, 1.0, 0.5], dtype=torch.float64)
    e_b = torch.tensor([0.0, 1.0, 0.0], dtype=torch.float64)
    kw = dict(mixed_precision=True, pressure_use_amg=True, potential_use_preconditioner=True,
              advection_tol=pb.SolverTolerance(rtol=1e-11), pressure_tol=pb.SolverTolerance(rtol=1e-11),
              potential_tol=pb.SolverTolerance(rtol=1e-11))
    alone = []
    for k, dom in enumerate(_members_3d()):
        _run(dom, stuart[k:k + 1], e_b, 2, **kw)
        alone.append(dom._u_block.double().cpu().numpy().copy())
    members = _members_3d()
    batch = pb.DomainBatch(members)
    _run(batch, stuart, e_b.expand(3, 3).contiguous(), 2, **kw)
    batch.scatter()
    for k, dom in enumerate(members):
        ref = alone[k]
        err = np.abs(dom._u_block.double().cpu().numpy() - ref).max() / np.abs(ref).max()
        assert err < 1e-8, (k, err)


def test_state_round_trip_is_exact(cuda):
    members = _members_2d()
    batch = pb.DomainBatch(members)
    for k, m in enumerate(members):
        batch._u_block[batch.instance_slice(k, 2)] += float(k + 1)
    batch.scatter()
    again = pb.DomainBatch(members)
    assert torch.equal(again._u_block, batch._u_block)
