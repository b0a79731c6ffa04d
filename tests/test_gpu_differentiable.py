"""Simulation(differentiable=True): each PISO step one torch.autograd node whose backward is
the hand-written adjoint of the step (phipict_b200/differentiable.py).

- gradients against the reference's own differentiable backend (phiPICT core/piso_diff.py,
  run on a B200 by tests/golden/make_ref_fields.py --grads) on a 2D MHD channel (initial
  velocity, static velocity source, Stuart number; a loss on u and p) and on a 2-block MHD
  duct (shared inflow/outflow profile, initial velocity, Stuart number; a loss on u and phi);
- gradients against central finite differences of the forward (the north star's 1e-5 bar);
- the differentiable forward gives the same fields as the ordinary step;
- the same gradients from the checkpointed rollout (AdjointMHD) as from the simulation.
"""
import math
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

import phipict_b200 as pb

GOLD = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLD))
import ref_cases as rc  # noqa: E402
from test_ref_fixtures import load_fixture  # noqa: E402

pytestmark = pytest.mark.gpu

REF_BAR = 1e-6  # gradients of two FP64 implementations whose solves stop at rtol 1e-14
FD_BAR = 1e-5


def load_grad(case: str) -> dict:
    return load_fixture(f"{case}_grad")


def rel(a, b) -> float:
    a, b = np.asarray(a, dtype=np.float64).ravel(), np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("case", ["g1", "g2"])
def test_gradients_match_reference(cuda, case):
    data = load_grad(case)
    got = rc.grad_run(pb, case, data, cuda, viscosity="grad_viscosity" in data)
    assert abs(got["loss"] - float(data["loss"])) <= 1e-10 * abs(float(data["loss"]))
    for k in [k for k in data if k.startswith("grad_")]:
        e = rel(got[k], data[k])
        assert math.isfinite(e) and e < REF_BAR, f"{case} {k}: {e:.3e}"
        assert np.abs(data[k]).max() > 0


def _g1_loss(inputs, v0, src, stuart, nu=None, device="cuda", upwind=False):
    """The g1 loss as a plain function of its inputs (no autograd)."""
    p = rc.G1
    dtype = torch.float64
    nu = 1.0 / p["re"] if nu is None else nu
    dom = pb.Domain(2, torch.tensor([nu], dtype=dtype), name="g", device=device, dtype=dtype)
    if upwind:
        dom.setAdvectionScheme(pb.AdvectionScheme.LINEAR_UPWIND)
    b = dom.CreateBlock(vertexCoordinates=rc._t(inputs["vertices_0"], dtype, device), name="channel")
    b.CloseBoundary("-y")
    b.CloseBoundary("+y")
    b.MakePeriodic("x")
    dom.PrepareSolve()
    b.setVelocity(v0)
    b.setVelocitySource(src)
    dom.UpdateDomainData()
    kw = dict(dt=p["dt"], substeps=1, non_orthogonal=False, e_b=torch.tensor([0.0, 1.0, 0.0], dtype=dtype),
              stuart_number=torch.tensor(float(stuart), dtype=torch.float64))
    kw.update(rc.tolerances(pb, True))
    sim = pb.MHDSimulation(domain=dom, **kw)
    for _ in range(p["steps"]):
        assert sim.single_step()
    w = rc._t(inputs["loss_w"], dtype, device)
    return float((w * b.velocity ** 2).sum() + 0.1 * (b.pressure ** 2).sum())


def test_gradients_match_finite_differences(cuda):
    inputs = rc.g1_inputs()
    got = rc.grad_run(pb, "g1", inputs, cuda, viscosity=True)
    g = torch.Generator().manual_seed(11)
    v0 = torch.as_tensor(inputs["velocity_0"]).cuda()
    src = torch.as_tensor(inputs["source"]).cuda()
    N0 = rc.G1["ha"] ** 2 / rc.G1["re"]
    h = 1e-4
    for name in ("velocity_0", "source", "stuart"):
        if name == "stuart":
            dirn = torch.ones(1, dtype=torch.float64)
        else:
            base = v0 if name == "velocity_0" else src
            dirn = torch.randn(base.shape, generator=g, dtype=torch.float64)
            dirn /= dirn.abs().max()
        args = lambda s: (v0 + s * h * dirn.cuda() if name == "velocity_0" else v0,
                          src + s * h * dirn.cuda() if name == "source" else src,
                          N0 + s * h * float(dirn[0]) if name == "stuart" else N0)
        fd = (_g1_loss(inputs, *args(1)) - _g1_loss(inputs, *args(-1))) / (2 * h)
        ad = float((torch.as_tensor(got[f"grad_{name}"]) * dirn.reshape(got[f"grad_{name}"].shape)).sum())
        assert abs(ad - fd) <= FD_BAR * max(abs(fd), 1e-30), f"{name}: adjoint {ad:.10e} vs FD {fd:.10e}"
    # the viscosity, with a step of 1e-3 of its value
    nu0, hn = 1.0 / rc.G1["re"], 1e-3 / rc.G1["re"]
    fd = (_g1_loss(inputs, v0, src, N0, nu0 + hn) - _g1_loss(inputs, v0, src, N0, nu0 - hn)) / (2 * hn)
    ad = float(got["grad_viscosity"].sum())
    assert abs(ad - fd) <= FD_BAR * max(abs(fd), 1e-30), f"viscosity: adjoint {ad:.10e} vs FD {fd:.10e}"


def test_differentiable_forward_is_the_plain_step(cuda):
    """The recorded forward changes nothing: same fields as the non-differentiable run."""
    inputs = rc.g1_inputs()
    fields = []
    for diff in (False, True):
        p = rc.G1
        dtype = torch.float64
        dom = pb.Domain(2, torch.tensor([1.0 / p["re"]], dtype=dtype), name="g", device="cuda", dtype=dtype)
        b = dom.CreateBlock(vertexCoordinates=rc._t(inputs["vertices_0"], dtype, "cuda"), name="channel")
        b.CloseBoundary("-y")
        b.CloseBoundary("+y")
        b.MakePeriodic("x")
        dom.PrepareSolve()
        v0 = torch.as_tensor(inputs["velocity_0"]).cuda()
        b.setVelocity(v0.clone().requires_grad_(diff))
        b.setVelocitySource(torch.as_tensor(inputs["source"]).cuda())
        dom.UpdateDomainData()
        kw = dict(dt=p["dt"], substeps=1, non_orthogonal=False, e_b=torch.tensor([0.0, 1.0, 0.0], dtype=dtype),
                  stuart_number=torch.tensor(p["ha"] ** 2 / p["re"]), differentiable=diff)
        kw.update(rc.tolerances(pb, True))
        sim = pb.MHDSimulation(domain=dom, **kw)
        for _ in range(p["steps"]):
            assert sim.single_step()
        fields.append((b.velocity.detach().clone(), b.pressure.detach().clone()))
        assert b.velocity.requires_grad == diff
        dom.Detach()
        assert not b.velocity.requires_grad
    for a, c in zip(*fields):
        assert torch.equal(a, c)


def test_rollout_and_simulation_agree(cuda):
    """AdjointMHD's checkpointed rollout and Simulation(differentiable=True) differentiate the
    same steps: gradients of sum(w u^2) with respect to the duct's inflow profile and the
    Stuart number agree."""
    from phipict_b200.adjoint import AdjointMHD, rollout

    inputs = rc.g2_inputs()
    p = rc.G2
    dtype = torch.float64
    w = rc._t(inputs["loss_w"], dtype, "cuda")

    def build():
        dom = pb.Domain(3, torch.tensor([1.0 / p["re"]], dtype=dtype), name="gduct", device="cuda", dtype=dtype)
        blocks = [dom.CreateBlock(vertexCoordinates=rc._t(inputs[f"vertices_{i}"], dtype, "cuda"), name=f"b{i}")
                  for i in range(p["nblocks"])]
        blocks[0].ConnectBlock("+x", blocks[1], "-x", "-y", "-z")
        prof = rc._t(inputs["inflow"], dtype, "cuda")
        blocks[0].CloseBoundary("-x", prof.clone())
        blocks[1].CloseBoundary("+x", prof.clone())
        blocks[1].getBoundary("+x").setPotentialBC(pb.PotentialBC.OPEN)
        for b in blocks:
            for f in ("-y", "+y", "-z", "+z"):
                b.CloseBoundary(f)
        dom.PrepareSolve()
        for i, b in enumerate(blocks):
            b.setVelocity(rc._t(inputs[f"velocity_{i}"], dtype, "cuda"))
        dom.UpdateDomainData()
        return dom, blocks, prof

    N0 = p["ha"] ** 2 / p["re"]
    # the simulation
    dom, blocks, prof = build()
    prof = prof.clone().requires_grad_(True)
    stuart = torch.tensor([N0], dtype=dtype, requires_grad=True)
    blocks[0].getBoundary("-x").setVelocity(prof)
    blocks[1].getBoundary("+x").setVelocity(prof)
    kw = dict(dt=p["dt"], substeps=1, non_orthogonal=False, e_b=torch.tensor([0.0, 1.0, 0.0], dtype=dtype),
              stuart_number=stuart, differentiable=True, hooks=rc.reset_source_hook(pb, 3, dtype))
    kw.update(rc.tolerances(pb, True))
    sim = pb.MHDSimulation(domain=dom, **kw)
    for _ in range(p["steps"]):
        assert sim.single_step()
    loss = sum((w * b.velocity ** 2).sum() for b in blocks)
    g_prof, g_N = torch.autograd.grad(loss, [prof, stuart])
    dom.Detach()
    # the rollout
    dom, blocks, prof0 = build()
    model = AdjointMHD(dom, p["dt"], torch.tensor([N0]), torch.tensor([0.0, 1.0, 0.0]), p["steps"],
                       faces=[(0, "-x"), (1, "+x")], checkpoint_every=2, tol=1e-12)
    prof_r = prof0.clone().requires_grad_(True)
    st_r = torch.tensor([N0], dtype=dtype, requires_grad=True)
    u = rollout(model, prof_r, st_r)
    B, n = 1, dom.getTotalSize()
    uu = u.view(B, 3, n)
    loss_r = sum((w.reshape(1, 3, -1) * uu[:, :, b.globalOffset:b.globalOffset + b.ncells()] ** 2).sum() for b in blocks)
    g_prof_r, g_N_r = torch.autograd.grad(loss_r, [prof_r, st_r])
    assert rel(g_prof.cpu(), g_prof_r.cpu()) < REF_BAR
    assert rel(g_N.cpu(), g_N_r.cpu()) < REF_BAR


def _g3_loss(inputs, s0, v0, lo, hi, nu, device="cuda", upwind=False):
    """The g3 loss as a plain function of its inputs (no autograd)."""
    p = rc.G3
    dtype = torch.float64
    dom = pb.Domain(2, torch.tensor([nu], dtype=dtype), name="g3", device=device, dtype=dtype)
    if upwind:
        dom.setAdvectionScheme(pb.AdvectionScheme.LINEAR_UPWIND)
    b = dom.CreateBlock(vertexCoordinates=rc._t(inputs["vertices_0"], dtype, device), name="channel")
    b.CloseBoundary("-y")
    b.CloseBoundary("+y")
    b.MakePeriodic("x")
    b.getBoundary("-y").setPassiveScalar(torch.tensor([[lo]], dtype=dtype, device=device))
    b.getBoundary("+y").setPassiveScalar(torch.tensor([[hi]], dtype=dtype, device=device))
    b.getBoundary("+y").setPassiveScalarType(pb.BoundaryConditionType.NEUMANN)
    dom.PrepareSolve()
    b.setVelocity(v0)
    b.setPassiveScalar(s0)
    dom.UpdateDomainData()
    kw = dict(dt=p["dt"], substeps=1, corrector_steps=2, non_orthogonal=False, advection_use_BiCG=True,
              pressure_use_BiCG=False, pressure_use_amg=False)
    kw.update({k: v for k, v in rc.tolerances(pb, True).items() if k != "potential_tol"})
    sim = pb.Simulation(domain=dom, **kw)
    for _ in range(p["steps"]):
        assert sim.single_step()
    return float((rc._t(inputs["loss_w"], dtype, device) * b.passiveScalar ** 2).sum()
                 + 0.1 * (rc._t(inputs["loss_wu"], dtype, device) * b.velocity ** 2).sum())


# phiPICT's gradient of a Neumann-type passive-scalar face still follows an older forward
# formulation (piso/advection.cu:768-773 marks it as to be updated): it omits the face area of
# the diffusive term and sends the advective part to the boundary value. Its gradients with
# respect to that face's value and to the viscosity (which that term also carries) therefore
# disagree with its own forward; here both are held to central differences instead.
REFERENCE_NEUMANN_SCALAR_DEFECT = ("grad_wall_hi", "grad_viscosity")


def test_scalar_gradients_match_reference(cuda):
    """The passive-scalar stage of the differentiable step against phiPICT's own gradients."""
    data = load_grad("g3")
    got = rc.g3_grad_run(pb, data, cuda)
    assert abs(got["loss"] - float(data["loss"])) <= 1e-10 * abs(float(data["loss"]))
    keys = [k for k in data if k.startswith("grad_") and k not in REFERENCE_NEUMANN_SCALAR_DEFECT]
    assert {"grad_scalar_0", "grad_velocity_0", "grad_wall_lo"} <= set(keys)
    errs = {k: rel(got[k], data[k]) for k in keys}
    assert all(math.isfinite(e) and e < REF_BAR for e in errs.values()), errs
    # the defect itself: on this grid phiPICT's Neumann value gradient is the face-cell sum
    # without the face area dx = 1/12
    dx = rc.G3["length"] / rc.G3["nx"]
    assert abs(float(got["grad_wall_hi"].sum()) - dx * float(data["grad_wall_hi"].sum())) \
        <= 1e-8 * abs(float(got["grad_wall_hi"].sum()))


def test_scalar_gradients_match_finite_differences(cuda):
    inputs = rc.g3_inputs()
    got = rc.g3_grad_run(pb, inputs, cuda)
    g = torch.Generator().manual_seed(13)
    s0 = torch.as_tensor(inputs["scalar_0"]).cuda()
    v0 = torch.as_tensor(inputs["velocity_0"]).cuda()
    base = dict(s0=s0, v0=v0, lo=1.0, hi=0.5, nu=1.0 / rc.G3["re"])
    cases = []
    for name, key in (("scalar_0", "s0"), ("velocity_0", "v0")):
        dirn = torch.randn(base[key].shape, generator=g, dtype=torch.float64)
        dirn /= dirn.abs().max()
        cases.append((name, key, dirn.cuda(), 1e-4))
    cases += [("wall_lo", "lo", 1.0, 1e-4), ("wall_hi", "hi", 1.0, 1e-4), ("viscosity", "nu", 1.0, 1e-3 / rc.G3["re"])]
    bad = []
    for name, key, dirn, h in cases:
        def at(sgn):
            kw = dict(base)
            kw[key] = base[key] + sgn * h * dirn
            return _g3_loss(inputs, kw["s0"], kw["v0"], kw["lo"], kw["hi"], kw["nu"])
        fd = (at(1) - at(-1)) / (2 * h)
        grad = torch.as_tensor(got[f"grad_{name}"])
        ad = float((grad * dirn.cpu().reshape(grad.shape)).sum()) if isinstance(dirn, torch.Tensor) else float(grad.sum())
        if not abs(ad - fd) <= FD_BAR * max(abs(fd), 1e-30):
            bad.append(f"{name}: adjoint {ad:.10e} vs FD {fd:.10e}")
    assert not bad, bad


def test_upwind_forward_matches_reference(cuda):
    """LINEAR_UPWIND (upwinded faces of the momentum and scalar matrices, deferred corrections
    of the right-hand sides and of HbyA): the differentiable forward gives phiPICT's loss on g1
    and g3. phiPICT's own LINEAR_UPWIND gradients are not a usable pin: projected on random
    directions they differ from central differences of phiPICT's forward by 1-4 % (ours agree
    to 1e-9), so the gradients are held to central differences below."""
    for case, data, run in (("g1u", load_grad("g1u"), lambda d: rc.grad_run(pb, "g1", d, cuda, viscosity=True, upwind=True)),
                            ("g3u", load_grad("g3u"), lambda d: rc.g3_grad_run(pb, d, cuda, upwind=True))):
        got = run(data)
        assert abs(got["loss"] - float(data["loss"])) <= 1e-10 * abs(float(data["loss"])), case


def test_upwind_gradients_match_finite_differences(cuda):
    inputs = rc.g1_inputs()
    got = rc.grad_run(pb, "g1", inputs, cuda, viscosity=True, upwind=True)
    g = torch.Generator().manual_seed(17)
    v0 = torch.as_tensor(inputs["velocity_0"]).cuda()
    src = torch.as_tensor(inputs["source"]).cuda()
    N0, nu0 = rc.G1["ha"] ** 2 / rc.G1["re"], 1.0 / rc.G1["re"]
    dirn = torch.randn(v0.shape, generator=g, dtype=torch.float64)
    dirn = (dirn / dirn.abs().max()).cuda()
    bad = []
    h = 1e-4
    fd = (_g1_loss(inputs, v0 + h * dirn, src, N0, upwind=True)
          - _g1_loss(inputs, v0 - h * dirn, src, N0, upwind=True)) / (2 * h)
    ad = float((torch.as_tensor(got["grad_velocity_0"]).cuda() * dirn).sum())
    if not abs(ad - fd) <= FD_BAR * abs(fd):
        bad.append(f"velocity_0: adjoint {ad:.10e} vs FD {fd:.10e}")
    hn = 1e-3 * nu0
    fd = (_g1_loss(inputs, v0, src, N0, nu0 + hn, upwind=True)
          - _g1_loss(inputs, v0, src, N0, nu0 - hn, upwind=True)) / (2 * hn)
    ad = float(got["grad_viscosity"].sum())
    if not abs(ad - fd) <= FD_BAR * abs(fd):
        bad.append(f"viscosity: adjoint {ad:.10e} vs FD {fd:.10e}")
    inputs3 = rc.g3_inputs()
    got3 = rc.g3_grad_run(pb, inputs3, cuda, upwind=True)
    s0 = torch.as_tensor(inputs3["scalar_0"]).cuda()
    v3 = torch.as_tensor(inputs3["velocity_0"]).cuda()
    for name, key in (("scalar_0", "s0"), ("velocity_0", "v0")):
        base = s0 if key == "s0" else v3
        d3 = torch.randn(base.shape, generator=g, dtype=torch.float64)
        d3 = (d3 / d3.abs().max()).cuda()
        def at(sgn):
            ss = s0 + sgn * h * d3 if key == "s0" else s0
            vv = v3 + sgn * h * d3 if key == "v0" else v3
            return _g3_loss(inputs3, ss, vv, 1.0, 0.5, 1.0 / rc.G3["re"], upwind=True)
        fd = (at(1) - at(-1)) / (2 * h)
        ad = float((torch.as_tensor(got3[f"grad_{name}"]).cuda() * d3).sum())
        if not abs(ad - fd) <= FD_BAR * abs(fd):
            bad.append(f"g3u {name}: adjoint {ad:.10e} vs FD {fd:.10e}")
    assert not bad, bad
