"""Cases whose fields are pinned to the reference itself (phiPICT run on a GPU).

Each case is built through the Python API that phiPICT and phipict_b200 share
(``Domain``, ``CreateBlock``, ``CloseBoundary``, ``MakePeriodic``, ``ConnectBlock``,
``FixedBoundary.setPotentialBC``, ``MHDSimulation``), so the same function builds the case
on either implementation: ``pp`` is the package (``phipict`` or ``phipict_b200``).

Every input that is random or derived (vertices, initial velocities, inflow profile) is
stored in the fixture and read back from it, so a test rebuilds exactly the inputs the
reference ran on.

Cases:
- ``c1``: the plain 2D Hartmann channel, one block of 64x32 cells on [0, 4] x [-1, 1]
  (uniform), periodic in x, no-slip insulating walls, e_b = (0, 1, 0), Re 100, Ha 10
  (N = Ha^2/Re = 1), u = (1, 0) + seeded N(0, 1e-3^2) per cell, dt 1e-3, two correctors,
  BiCGStab momentum, CG pressure and potential, 200 steps, no forcing.
- ``c2r``: a reduced 3D MHD duct, 3 blocks of 16x12x12 connected along x, tanh wall
  stretching (beta 2) in y and z on [-1, 1]^2, inflow u = (1 + seeded N(0, 1e-2^2), 0, 0) at
  -x, the same profile as outflow at +x with an open potential face, insulating walls,
  e_b = (0, 1, 0), Re 1000, Ha 100 (N = 10), dt 1e-2, 20 steps.
"""
from __future__ import annotations

import numpy as np
import torch

C1 = dict(nx=64, ny=32, length=4.0, re=100.0, ha=10.0, dt=1e-3, steps=200, noise=1e-3, seed=0)
C2R = dict(nx=16, ny=12, nz=12, nblocks=3, re=1000.0, ha=100.0, beta=2.0, dt=1e-2, steps=20, noise=1e-2, seed=0)
# steps after which the fields are recorded
C1_RECORD = (1, 10, 200)
C2R_RECORD = (1, 5, 20)


def tanh_weights(n: int, beta: float) -> np.ndarray:
    """n+1 vertex positions in [-1, 1] clustered at both ends: tanh(beta xi)/tanh(beta)."""
    xi = np.linspace(-1.0, 1.0, n + 1)
    w = np.tanh(beta * xi) / np.tanh(beta)
    w[0], w[-1] = -1.0, 1.0
    return w


def vertices(xs, ys, zs=None) -> np.ndarray:
    if zs is None:
        Y, X = np.meshgrid(ys, xs, indexing="ij")
        return np.stack([X, Y])[None]
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    return np.stack([X, Y, Z])[None]


def c1_inputs() -> dict:
    p = C1
    xs = np.linspace(0.0, p["length"], p["nx"] + 1)
    ys = np.linspace(-1.0, 1.0, p["ny"] + 1)
    g = torch.Generator(device="cpu").manual_seed(p["seed"])
    u0 = p["noise"] * torch.randn(1, 2, p["ny"], p["nx"], generator=g, dtype=torch.float64)
    u0[:, 0] += 1.0
    return {"vertices_0": vertices(xs, ys), "velocity_0": u0.numpy()}


def c2r_inputs() -> dict:
    p = C2R
    ys = tanh_weights(p["ny"], p["beta"])
    zs = tanh_weights(p["nz"], p["beta"])
    g = torch.Generator(device="cpu").manual_seed(p["seed"])
    inflow = torch.zeros(1, 3, p["nz"], p["ny"], 1, dtype=torch.float64)
    inflow[0, 0] = 1.0 + p["noise"] * torch.randn(p["nz"], p["ny"], 1, generator=g, dtype=torch.float64)
    out = {"inflow": inflow.numpy()}
    for i in range(p["nblocks"]):
        xs = np.linspace(float(i), float(i + 1), p["nx"] + 1)
        out[f"vertices_{i}"] = vertices(xs, ys, zs)
        u0 = np.zeros((1, 3, p["nz"], p["ny"], p["nx"]))
        u0[0, 0] = 1.0
        out[f"velocity_{i}"] = u0
    return out


def _t(a, dtype, device):
    return torch.as_tensor(np.asarray(a)).to(device=device, dtype=dtype).contiguous()


def _finish(dom, blocks, inputs, dtype, device, prepare: bool):
    """Prepare the domain (on a CUDA device) and set the initial velocities. On the CPU, for
    the oracle, the domain is only described and the velocities are written into the blocks."""
    if prepare:
        dom.PrepareSolve()
    for i, b in enumerate(blocks):
        b.velocity.copy_(_t(inputs[f"velocity_{i}"], dtype, device))
    if prepare:
        dom.UpdateDomainData()
    return dom


def build_c1(pp, inputs: dict, dtype, device, prepare: bool = True):
    p = C1
    dom = pp.Domain(2, torch.tensor([1.0 / p["re"]], dtype=dtype), name="hartmann", device=device, dtype=dtype)
    b = dom.CreateBlock(vertexCoordinates=_t(inputs["vertices_0"], dtype, device), name="channel")
    b.CloseBoundary("-y")
    b.CloseBoundary("+y")
    b.MakePeriodic("x")
    return _finish(dom, [b], inputs, dtype, device, prepare)


def build_c2r(pp, inputs: dict, dtype, device, prepare: bool = True):
    p = C2R
    dom = pp.Domain(3, torch.tensor([1.0 / p["re"]], dtype=dtype), name="duct", device=device, dtype=dtype)
    blocks = [dom.CreateBlock(vertexCoordinates=_t(inputs[f"vertices_{i}"], dtype, device), name=f"b{i}")
              for i in range(p["nblocks"])]
    for i in range(p["nblocks"] - 1):
        blocks[i].ConnectBlock("+x", blocks[i + 1], "-x", "-y", "-z")
    inflow = _t(inputs["inflow"], dtype, device)
    blocks[0].CloseBoundary("-x", inflow)
    blocks[-1].CloseBoundary("+x", inflow.clone())
    blocks[-1].getBoundary("+x").setPotentialBC(pp.PotentialBC.OPEN)
    for b in blocks:
        for f in ("-y", "+y", "-z", "+z"):
            b.CloseBoundary(f)
    return _finish(dom, blocks, inputs, dtype, device, prepare)


TIGHT_RTOL, TIGHT_ATOL = 1e-14, 1e-16


def tolerances(pp, tight: bool) -> dict:
    """Tight: every solve to rtol 1e-14 / atol 1e-16, so that the fields are fixed to far
    below the FP64 parity bar (a pressure solved to rtol r is off by about cond(P) r, which at
    rtol 1e-12 already reaches 1e-10 on the duct). Otherwise the configuration's 1e-8, read as
    a relative tolerance (floored at 8 eps ||b||/sqrt(n) by SolverTolerance)."""
    t = pp.SolverTolerance(rtol=TIGHT_RTOL, atol=TIGHT_ATOL) if tight else pp.SolverTolerance(rtol=1e-8)
    return dict(advection_tol=t, pressure_tol=t, potential_tol=t)


def reset_source_hook(pp, dims: int, dtype):
    """A PRE_VELOCITY_SETUP hook that sets a zero static velocity source before the Lorentz
    force is added, so that the force of each step replaces the last instead of accumulating
    on it (as phiPICT's examples/hartmann.py resets its forcing every step). phiPICT adds its
    force onto an existing source only; without one, a multi-block domain hands the block a
    non-contiguous slice of the flat force (simulation/mhd.py:91-121,583-593), which its
    setVelocitySource refuses, so the duct case needs the reset to run on the reference."""

    def reset(domain, **kwargs):
        for b in domain.getBlocks():
            b.setVelocitySource(torch.zeros(1, dims, dtype=dtype, device=domain.getDevice()))
        domain.UpdateDomainData()

    return pp.Hooks().append(pp.Hook.PRE_VELOCITY_SETUP, reset)


def make_sim(pp, dom, case: str, tight: bool, **extra):
    """c1 keeps phiPICT's default of a Lorentz force accumulated onto the existing source;
    c2r resets the source every step (reset_source_hook)."""
    p = C1 if case == "c1" else C2R
    dtype = dom.getDtype()
    if case == "c2r":
        extra.setdefault("hooks", reset_source_hook(pp, dom.getSpatialDims(), dtype))
    kw = dict(dt=p["dt"], substeps=1, corrector_steps=2, non_orthogonal=False, advection_use_BiCG=True,
              pressure_use_BiCG=False, pressure_use_amg=False, potential_use_preconditioner=False,
              stuart_number=torch.tensor(p["ha"] ** 2 / p["re"], dtype=torch.float64),
              e_b=torch.tensor([0.0, 1.0, 0.0], dtype=dtype))
    kw.update(tolerances(pp, tight))
    kw.update(extra)
    return pp.MHDSimulation(domain=dom, **kw)


def fields(dom) -> dict:
    """u and p per block, phi as the flat potential vector."""
    out = {}
    for i, b in enumerate(dom.getBlocks()):
        out[f"u_{i}"] = b.velocity.detach().double().cpu().numpy().copy()
        out[f"p_{i}"] = b.pressure.detach().double().cpu().numpy().copy()
    out["phi"] = dom.epotResult.detach().double().cpu().numpy().copy()
    return out


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# --- gradient cases (the differentiable step) -------------------------------------------
G1 = dict(nx=24, ny=16, length=2.0, re=100.0, ha=10.0, dt=1e-2, steps=5, seed=3)
G2 = dict(nx=8, ny=6, nz=6, nblocks=2, re=100.0, ha=5.0, beta=2.0, dt=1e-2, steps=3, noise=1e-1, seed=4)


G3 = dict(nx=24, ny=16, length=2.0, re=50.0, dt=1e-2, steps=4, seed=5)


def g3_inputs() -> dict:
    """Seeded state of the passive-scalar gradient channel: u = (1, 0) + 0.2 N(0, 1), a scalar
    field U(0, 1), a Dirichlet scalar 1 on the -y wall and a Neumann scalar flux 0.5 on the +y
    wall."""
    p = G3
    xs = np.linspace(0.0, p["length"], p["nx"] + 1)
    ys = np.linspace(-1.0, 1.0, p["ny"] + 1)
    g = torch.Generator(device="cpu").manual_seed(p["seed"])
    u0 = 0.2 * torch.randn(1, 2, p["ny"], p["nx"], generator=g, dtype=torch.float64)
    u0[:, 0] += 1.0
    s0 = torch.rand(1, 1, p["ny"], p["nx"], generator=g, dtype=torch.float64)
    w = torch.rand(1, 1, p["ny"], p["nx"], generator=g, dtype=torch.float64)
    wu = torch.rand(1, 2, p["ny"], p["nx"], generator=g, dtype=torch.float64)
    return {"vertices_0": vertices(xs, ys), "velocity_0": u0.numpy(), "scalar_0": s0.numpy(),
            "wall_lo": np.array([[1.0]]), "wall_hi": np.array([[0.5]]), "loss_w": w.numpy(), "loss_wu": wu.numpy()}


def g3_grad_run(pp, inputs: dict, device, sim_kwargs: dict | None = None, upwind: bool = False) -> dict:
    """g3: the plain PISO step (no MHD) with one passive-scalar channel. loss = sum(w s^2) +
    0.1 sum(wu u^2) after G3 steps; gradients with respect to the initial scalar and
    velocity, the two wall scalar values and the viscosity (the scalar's diffusivity is the
    viscosity: the domain sets none)."""
    dtype = torch.float64
    p = G3
    nu = torch.tensor([1.0 / p["re"]], dtype=dtype, requires_grad=True)
    dom = pp.Domain(2, nu, name="gscalar", device=device, dtype=dtype)
    if upwind:
        dom.setAdvectionScheme(pp.AdvectionScheme.LINEAR_UPWIND)
    b = dom.CreateBlock(vertexCoordinates=_t(inputs["vertices_0"], dtype, device), name="channel")
    b.CloseBoundary("-y")
    b.CloseBoundary("+y")
    b.MakePeriodic("x")
    lo = _t(inputs["wall_lo"], dtype, device).requires_grad_(True)
    hi = _t(inputs["wall_hi"], dtype, device).requires_grad_(True)
    b.getBoundary("-y").setPassiveScalar(lo)
    b.getBoundary("+y").setPassiveScalar(hi)
    b.getBoundary("+y").setPassiveScalarType(pp.BoundaryConditionType.NEUMANN)
    dom.PrepareSolve()
    v0 = _t(inputs["velocity_0"], dtype, device).requires_grad_(True)
    s0 = _t(inputs["scalar_0"], dtype, device).requires_grad_(True)
    b.setVelocity(v0.clone())
    b.setPassiveScalar(s0.clone())
    dom.UpdateDomainData()
    kw = dict(dt=p["dt"], substeps=1, corrector_steps=2, non_orthogonal=False, advection_use_BiCG=True,
              pressure_use_BiCG=False, pressure_use_amg=False, differentiable=True)
    kw.update({k: v for k, v in tolerances(pp, True).items() if k != "potential_tol"})
    kw.update(sim_kwargs or {})
    sim = pp.Simulation(domain=dom, **kw)
    for _ in range(p["steps"]):
        sim.single_step()
    blk = dom.getBlocks()[0]
    loss = (_t(inputs["loss_w"], dtype, device) * blk.passiveScalar ** 2).sum() \
        + 0.1 * (_t(inputs["loss_wu"], dtype, device) * blk.velocity ** 2).sum()
    names, wrt = ["scalar_0", "velocity_0", "wall_lo", "wall_hi", "viscosity"], [s0, v0, lo, hi, nu]
    grads = torch.autograd.grad(loss, wrt, allow_unused=True)
    out = {"loss": float(loss.detach())}
    for k, g in zip(names, grads):
        if g is not None:
            out[f"grad_{k}"] = g.detach().double().cpu().numpy()
    dom.Detach()
    return out


def g1_inputs() -> dict:
    """Seeded state of the gradient channel: u = (1, 0) + 0.3 N(0, 1), a static source."""
    p = G1
    xs = np.linspace(0.0, p["length"], p["nx"] + 1)
    ys = np.linspace(-1.0, 1.0, p["ny"] + 1)
    g = torch.Generator(device="cpu").manual_seed(p["seed"])
    u0 = 0.3 * torch.randn(1, 2, p["ny"], p["nx"], generator=g, dtype=torch.float64)
    u0[:, 0] += 1.0
    w = torch.rand(1, 2, p["ny"], p["nx"], generator=g, dtype=torch.float64)
    return {"vertices_0": vertices(xs, ys), "velocity_0": u0.numpy(), "source": np.array([[0.5, -0.2]]),
            "loss_w": w.numpy()}


def g2_inputs() -> dict:
    """Seeded state of the gradient duct: an inflow profile 1 + 0.1 N(0, 1) shared by the inflow
    and outflow faces, u = 1 + 0.1 N(0, 1) in x."""
    p = G2
    ys = tanh_weights(p["ny"], p["beta"])
    zs = tanh_weights(p["nz"], p["beta"])
    g = torch.Generator(device="cpu").manual_seed(p["seed"])
    prof = torch.zeros(1, 3, p["nz"], p["ny"], 1, dtype=torch.float64)
    prof[0, 0] = 1.0 + p["noise"] * torch.randn(p["nz"], p["ny"], 1, generator=g, dtype=torch.float64)
    out = {"inflow": prof.numpy()}
    for i in range(p["nblocks"]):
        xs = np.linspace(float(i), float(i + 1), p["nx"] + 1)
        out[f"vertices_{i}"] = vertices(xs, ys, zs)
        u0 = torch.zeros(1, 3, p["nz"], p["ny"], p["nx"], dtype=torch.float64)
        u0[0, 0] = 1.0 + p["noise"] * torch.randn(p["nz"], p["ny"], p["nx"], generator=g, dtype=torch.float64)
        out[f"velocity_{i}"] = u0.numpy()
    out["loss_w"] = torch.rand(1, 3, p["nz"], p["ny"], p["nx"], generator=g, dtype=torch.float64).numpy()
    return out


def grad_run(pp, case: str, inputs: dict, device, sim_kwargs: dict | None = None, viscosity: bool = False,
             upwind: bool = False) -> dict:
    """The differentiable rollout of a gradient case on implementation pp; returns the loss
    and its gradients.

    g1: loss = sum(w u^2) + 0.1 sum(p^2) after G1 steps, gradients with respect to the initial
    velocity, the static velocity source and the Stuart number.
    g2: loss = sum(w u^2) over the outlet block + sum(phi^2) after G2 steps, gradients with
    respect to the shared inflow/outflow profile, the initial velocity of the first block and
    the Stuart number (the source is reset before every Lorentz force, so it has none).
    viscosity: also the gradient with respect to the domain's viscosity (a tensor with
    requires_grad handed to the Domain constructor). upwind: the LINEAR_UPWIND advection
    scheme instead of CENTRAL."""
    dtype = torch.float64
    p = G1 if case == "g1" else G2
    nu = torch.tensor([1.0 / p["re"]], dtype=dtype, requires_grad=viscosity)
    stuart = torch.tensor([p["ha"] ** 2 / p["re"]], dtype=dtype, requires_grad=True)
    v0 = _t(inputs["velocity_0"], dtype, device).requires_grad_(True)
    kw = dict(dt=p["dt"], substeps=1, corrector_steps=2, non_orthogonal=False, advection_use_BiCG=True,
              pressure_use_BiCG=False, pressure_use_amg=False, potential_use_preconditioner=False,
              e_b=torch.tensor([0.0, 1.0, 0.0], dtype=dtype), stuart_number=stuart, differentiable=True)
    kw.update(tolerances(pp, True))
    kw.update(sim_kwargs or {})
    if case == "g1":
        dom = pp.Domain(2, nu, name="gchannel", device=device, dtype=dtype)
        if upwind:
            dom.setAdvectionScheme(pp.AdvectionScheme.LINEAR_UPWIND)
        b = dom.CreateBlock(vertexCoordinates=_t(inputs["vertices_0"], dtype, device), name="channel")
        b.CloseBoundary("-y")
        b.CloseBoundary("+y")
        b.MakePeriodic("x")
        dom.PrepareSolve()
        src = _t(inputs["source"], dtype, device).requires_grad_(True)
        b.setVelocity(v0.clone())
        b.setVelocitySource(src.clone())
        dom.UpdateDomainData()
        sim = pp.MHDSimulation(domain=dom, **kw)
        for _ in range(p["steps"]):
            sim.single_step()
        w = _t(inputs["loss_w"], dtype, device)
        blk = dom.getBlocks()[0]
        loss = (w * blk.velocity ** 2).sum() + 0.1 * (blk.pressure ** 2).sum()
        names, wrt = ["velocity_0", "source", "stuart"], [v0, src, stuart]
    else:
        dom = pp.Domain(3, nu, name="gduct", device=device, dtype=dtype)
        if upwind:
            dom.setAdvectionScheme(pp.AdvectionScheme.LINEAR_UPWIND)
        blocks = [dom.CreateBlock(vertexCoordinates=_t(inputs[f"vertices_{i}"], dtype, device), name=f"b{i}")
                  for i in range(p["nblocks"])]
        for i in range(p["nblocks"] - 1):
            blocks[i].ConnectBlock("+x", blocks[i + 1], "-x", "-y", "-z")
        prof = _t(inputs["inflow"], dtype, device).requires_grad_(True)
        blocks[0].CloseBoundary("-x", prof.detach().clone())
        blocks[-1].CloseBoundary("+x", prof.detach().clone())
        blocks[-1].getBoundary("+x").setPotentialBC(pp.PotentialBC.OPEN)
        for b in blocks:
            for f in ("-y", "+y", "-z", "+z"):
                b.CloseBoundary(f)
        dom.PrepareSolve()
        blocks[0].setVelocity(v0.clone())
        for i in range(1, p["nblocks"]):
            blocks[i].setVelocity(_t(inputs[f"velocity_{i}"], dtype, device))
        blocks[0].getBoundary("-x").setVelocity(prof)
        blocks[-1].getBoundary("+x").setVelocity(prof)
        dom.UpdateDomainData()
        kw.setdefault("hooks", reset_source_hook(pp, 3, dtype))
        sim = pp.MHDSimulation(domain=dom, **kw)
        for _ in range(p["steps"]):
            sim.single_step()
        w = _t(inputs["loss_w"], dtype, device)
        loss = (w * blocks[-1].velocity ** 2).sum() + (dom.getBlocks()[-1].epot ** 2).sum()
        names, wrt = ["inflow", "velocity_0", "stuart"], [prof, v0, stuart]
    if viscosity:
        names, wrt = names + ["viscosity"], wrt + [nu]
    grads = torch.autograd.grad(loss, wrt, allow_unused=True)
    out = {"loss": float(loss.detach())}
    for k, g in zip(names, grads):
        if g is not None:
            out[f"grad_{k}"] = g.detach().double().cpu().numpy()
    dom.Detach()
    return out
