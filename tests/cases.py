"""Seeded domains shared by the tests: 2D Hartmann channel, 3D connected MHD duct, a
2D block pair joined with rotated axes, curvilinear (non-orthogonal) variants of the three,
and helpers to fill states.

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


def skewed_channel_2d(nx=14, ny=10, *, device="cuda", dtype=torch.float64, shear=0.35, wave=0.06, nu=0.02, channels=1,
                      length=4.0):
    """The periodic wall-bounded channel of hartmann_2d on a curvilinear grid: vertex x is
    sheared by shear * y and vertex y waves by wave sin(2 pi x / L) (1 - y^2), so every cell
    has metric cross terms while the walls stay at y = +-1 and the grid stays periodic in x."""
    xs = np.linspace(0.0, length, nx + 1)
    ys = span(-1.0, 1.0, make_weights_tanh(ny, 1.3))
    v = rectilinear_vertices(xs, ys, dtype=torch.float64)
    X, Y = v[0, 0].clone(), v[0, 1].clone()
    v[0, 0] = X + shear * Y
    v[0, 1] = Y + wave * torch.sin(2 * np.pi * X / length) * (1 - Y * Y)
    dom = pb.Domain(2, torch.tensor([nu]), name="skewed", device=device, dtype=dtype, passiveScalarChannels=channels)
    b = dom.CreateBlock(vertexCoordinates=v.to(dtype), name="channel")
    b.CloseBoundary("-y")
    b.CloseBoundary("+y")
    b.MakePeriodic("x")
    return dom


def skewed_duct_3d(nx=6, ny=5, nz=4, nblocks=2, *, device="cuda", dtype=torch.float64, nu=0.05, seed=0, noise=1e-2,
                   channels=1):
    """duct_3d on a curvilinear grid: x sheared by 0.3 y + 0.2 z, y and z waving with
    sin(pi x) inside the duct (the walls stay flat, the in- and outflow faces keep their
    rectilinear y-z grid, so the boundary fluxes still balance)."""
    ws, wz = make_weights_tanh(ny, 1.5), make_weights_tanh(nz, 1.5)
    ys, zs = span(-1.0, 1.0, ws), span(-1.0, 1.0, wz)
    dom = pb.Domain(3, torch.tensor([nu]), name="skewed_duct", device=device, dtype=dtype, passiveScalarChannels=channels)
    blocks = []
    for i in range(nblocks):
        xs = np.linspace(i * 1.0, (i + 1) * 1.0, nx + 1)
        v = rectilinear_vertices(xs, ys, zs, dtype=torch.float64)
        X, Y, Z = v[0, 0].clone(), v[0, 1].clone(), v[0, 2].clone()
        v[0, 0] = X + 0.3 * Y + 0.2 * Z
        v[0, 1] = Y + 0.05 * torch.sin(np.pi * X) * (1 - Y * Y)
        v[0, 2] = Z + 0.04 * torch.sin(np.pi * X) * (1 - Z * Z)
        blocks.append(dom.CreateBlock(vertexCoordinates=v.to(dtype), name=f"b{i}"))
    for i in range(nblocks - 1):
        blocks[i].ConnectBlock("+x", blocks[i + 1], "-x", "-y", "-z")
    g = torch.Generator(device="cpu").manual_seed(seed)
    inflow = torch.zeros(1, 3, nz, ny, 1, dtype=dtype)
    inflow[0, 0] = 1.0 + noise * torch.randn(nz, ny, 1, generator=g, dtype=dtype)
    blocks[0].CloseBoundary("-x", inflow.to(device))
    blocks[-1].CloseBoundary("+x", inflow.clone().to(device))
    blocks[-1].getBoundary("+x").setPotentialBC(pb.PotentialBC.OPEN)
    for b in blocks:
        for f in ("-y", "+y", "-z", "+z"):
            b.CloseBoundary(f)
    return dom


def skewed_pair_2d(n=6, *, device="cuda", dtype=torch.float64, nu=0.05, seed=1):
    """The block pair of rotated_pair_2d (a's +x joined to b's -y with b's x inverted) with
    seeded, distorted vertex coordinates: connections with an axis mapping on a grid with
    cross terms (an assembly case; the two blocks are not meant to fit together in space)."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    xs = np.linspace(0.0, 1.0, n + 1)

    def distorted(x0):
        v = rectilinear_vertices(xs + x0, xs, dtype=torch.float64)
        v[0, :, 1:-1, 1:-1] += 0.25 / n * (torch.rand(2, n - 1, n - 1, generator=g, dtype=torch.float64) - 0.5)
        v[0, 0] += 0.2 * v[0, 1]
        return v.to(dtype)

    dom = pb.Domain(2, torch.tensor([nu]), name="skewed_pair", device=device, dtype=dtype)
    a = dom.CreateBlock(vertexCoordinates=distorted(0.0), name="a")
    b = dom.CreateBlock(vertexCoordinates=distorted(2.0), name="b")
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
