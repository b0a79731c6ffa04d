"""Seeded domains shared by the tests: 2D Hartmann channel, 3D connected MHD duct, a
2D block pair joined with rotated axes, and helpers to fill states.

Seeds follow the reference tests' convention: ``torch.Generator(device='cpu').manual_seed``
and ``.to(device)`` (tests/test_batching.py:40-45)."""
from __future__ import annotations

import numpy as np
import torch

import phipict_b200 as pb
from phipict_b200.grid import make_weights_tanh, rectilinear_vertices, span


def hartmann_2d(nx=16, ny=12, *, device="cuda", dtype=torch.float64, length=4.0, grading=1.5, nu=0.01, batch=1,
                channels=1):
    """Periodic x, no-slip insulating walls at y = +-1, tanh-graded in y; `channels` passive
    scalar channels (phiPICT's default is one)."""
    xs = np.linspace(0.0, length, nx + 1)
    ys = span(-1.0, 1.0, make_weights_tanh(ny, grading))
    dom = pb.Domain(2, torch.tensor([nu]), name="hartmann", device=device, dtype=dtype, passiveScalarChannels=channels)
    b = dom.CreateBlock(vertexCoordinates=rectilinear_vertices(xs, ys, dtype=dtype), name="channel")
    b.CloseBoundary("-y")
    b.CloseBoundary("+y")
    b.MakePeriodic("x")
    if batch > 1:
        dom.setBatchSize(batch)
    return dom


def duct_3d(nx=8, ny=6, nz=5, nblocks=2, *, device="cuda", dtype=torch.float64, grading=2.0, nu=0.05,
            seed=0, noise=1e-2, batch=1, channels=1):
    """nblocks blocks connected along x; inflow (u=1 + seeded noise, flux-balanced by a
    varying outflow) at -x, open-potential outflow at +x, insulating walls in y and z."""
    ws = make_weights_tanh(ny, grading)
    wz = make_weights_tanh(nz, grading)
    ys = span(-1.0, 1.0, ws)
    zs = span(-1.0, 1.0, wz)
    dom = pb.Domain(3, torch.tensor([nu]), name="duct", device=device, dtype=dtype, passiveScalarChannels=channels)
    blocks = []
    for i in range(nblocks):
        xs = np.linspace(i * 1.0, (i + 1) * 1.0, nx + 1)
        blocks.append(dom.CreateBlock(vertexCoordinates=rectilinear_vertices(xs, ys, zs, dtype=dtype), name=f"b{i}"))
    for i in range(nblocks - 1):
        blocks[i].ConnectBlock("+x", blocks[i + 1], "-x", "-y", "-z")
    g = torch.Generator(device="cpu").manual_seed(seed)
    inflow = torch.zeros(1, 3, nz, ny, 1, dtype=dtype)
    inflow[0, 0] = 1.0 + noise * torch.randn(nz, ny, 1, generator=g, dtype=dtype)
    first, last = blocks[0], blocks[-1]
    first.CloseBoundary("-x", inflow.to(device))
    # outflow: the same profile, so the boundary fluxes balance exactly on a rectilinear grid
    last.CloseBoundary("+x", inflow.clone().to(device))
    last.getBoundary("+x").setPotentialBC(pb.PotentialBC.OPEN)
    for b in blocks:
        for f in ("-y", "+y", "-z", "+z"):
            b.CloseBoundary(f)
    if batch > 1:
        dom.setBatchSize(batch)
    return dom


def rotated_pair_2d(n=6, *, device="cuda", dtype=torch.float64, nu=0.05):
    """Two 2D blocks without coordinates; block a's +x face is joined to block b's -y face
    with b's x axis inverted, exercising the connection axis mapping."""
    dom = pb.Domain(2, torch.tensor([nu]), name="rot", device=device, dtype=dtype)
    a = dom.CreateBlock(velocity=torch.zeros(1, 2, n, n, dtype=dtype), name="a")
    b = dom.CreateBlock(velocity=torch.zeros(1, 2, n, n, dtype=dtype), name="b")
    a.ConnectBlock("+x", b, "-y", "+x")
    a.CloseBoundary("-x")
    a.MakePeriodic("y")
    b.CloseBoundary("-x")
    b.CloseBoundary("+x")
    b.CloseBoundary("+y")
    return dom


def seeded_state(dom, seed=0, scale=0.3, base=(1.0,)):
    """Random block velocities (and a base flow along x)."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    for b in dom.getBlocks():
        v = scale * torch.randn(b.velocity.shape, generator=g, dtype=b.velocity.dtype)
        v[:, 0] += base[0]
        b.velocity.copy_(v.to(b.velocity.device))
