"""Hand-written adjoint of the MHD PISO step (phipict_b200.adjoint).

- the transposed stencil built on the device is the transpose of the stencil matrix (host
  SciPy), across connected blocks with rotated axes;
- the rollout gradient with respect to a boundary velocity profile (shared by an inflow
  and the matching outflow, so mass stays balanced) and the Stuart number matches central
  finite differences in FP64 (the reference's check, core/piso_diff.py tests), through
  several steps and a checkpoint segment boundary."""
import ctypes as ct

import numpy as np
import pytest
import torch

import phipict_b200 as pb
from phipict_b200 import _C, _lib
from phipict_b200.adjoint import AdjointMHD, rollout
from cases import duct_3d, rotated_pair_2d, seeded_state
from test_gpu_amg import _dense

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["duct3d", "rotated2d"])
def test_transposed_stencil(cuda, case):
    dom = duct_3d(6, 5, 4, 2) if case == "duct3d" else rotated_pair_2d(6)
    seeded_state(dom, 3, scale=0.3)
    dom.PrepareSolve()
    _C.SetupAdvectionMatrix(dom, torch.tensor([0.01], dtype=torch.float64), 0)
    CT = torch.empty_like(dom._C_st)
    _lib.call("phb_transpose_stencil", ct.byref(dom.desc()), dom._C_st.data_ptr(), CT.data_ptr(), _lib.stream_ptr(dom.getDevice()))
    C = _dense(dom.desc(), dom._C_st).toarray()
    T = _dense(dom.desc(), CT).toarray()
    assert np.abs(T - C.T).max() <= 1e-14 * np.abs(C).max()


def _channel2d(nx=8, ny=6):
    """Two 2D blocks joined along x, inflow at -x and the same profile out at +x."""
    from phipict_b200.grid import make_weights_tanh, rectilinear_vertices, span
    dom = pb.Domain(2, torch.tensor([0.05]), name="ch", device="cuda", dtype=torch.float64)
    ys = span(-1.0, 1.0, make_weights_tanh(ny, 1.5))
    a = dom.CreateBlock(vertexCoordinates=rectilinear_vertices(np.linspace(0, 1, nx + 1), ys), name="a")
    b = dom.CreateBlock(vertexCoordinates=rectilinear_vertices(np.linspace(1, 2, nx + 1), ys), name="b")
    a.ConnectBlock("+x", b, "-x", "-y")
    prof = torch.zeros(1, 2, ny, 1, dtype=torch.float64)
    prof[0, 0] = 1.0
    a.CloseBoundary("-x", prof.cuda())
    b.CloseBoundary("+x", prof.clone().cuda())
    b.getBoundary("+x").setPotentialBC(pb.PotentialBC.OPEN)
    for blk in (a, b):
        blk.CloseBoundary("-y")
        blk.CloseBoundary("+y")
    return dom


@pytest.mark.parametrize("case", ["channel2d", "duct3d", "duct3d_upwind"])
def test_rollout_gradient_matches_finite_differences(cuda, case):
    dom = _channel2d() if case == "channel2d" else duct_3d(6, 5, 4, 2)
    if case.endswith("upwind"):
        dom.setAdvectionScheme(pb.AdvectionScheme.LINEAR_UPWIND)
    seeded_state(dom, 11, scale=0.1)
    dom.PrepareSolve()
    blocks = dom.getBlocks()
    faces = [(blocks[0], "-x"), (blocks[-1], "+x")]
    e_b = torch.tensor([0.0, 1.0, 0.0], dtype=torch.float64)
    model = AdjointMHD(dom, 0.01, torch.tensor([2.0]), e_b, steps=3, faces=faces, checkpoint_every=2)
    initial = model._state()
    p0 = model.faces[0]._velocity.detach().clone()
    g = torch.Generator().manual_seed(5)
    w = torch.randn(dom._u_block.numel(), generator=g, dtype=torch.float64).cuda()
    vp = torch.randn(p0.shape, generator=g, dtype=torch.float64).cuda()
    vp[:, 0] -= vp[:, 0].mean()  # keep the profile's net flux (the mass balance)
    if case == "channel2d":
        vp[:, 1] = 0
    vN = torch.tensor([0.7], dtype=torch.float64)

    def loss(profile, N):
        model.forward(profile, N, initial=[t.clone() for t in initial])
        return float((w * dom._u_block.reshape(-1)).sum())

    prof = p0.clone().requires_grad_(True)
    N = torch.tensor([2.0], dtype=torch.float64, requires_grad=True)
    u = rollout(model, prof, N, initial=[t.clone() for t in initial])
    (w * u).sum().backward()
    analytic = float((prof.grad * vp).sum()) + float((N.grad.cpu() * vN).sum())
    eps = 1e-4
    fd = (loss(p0 + eps * vp, torch.tensor([2.0]) + eps * vN) - loss(p0 - eps * vp, torch.tensor([2.0]) - eps * vN)) / (2 * eps)
    assert abs(analytic - fd) <= 1e-5 * max(abs(fd), 1e-12), (analytic, fd)
    # each parameter on its own, too
    fdN = (loss(p0, torch.tensor([2.0]) + eps * vN) - loss(p0, torch.tensor([2.0]) - eps * vN)) / (2 * eps)
    gN = float((N.grad.cpu() * vN).sum())
    assert abs(gN - fdN) <= 1e-5 * abs(fdN), (gN, fdN)
    fdp = (loss(p0 + eps * vp, torch.tensor([2.0])) - loss(p0 - eps * vp, torch.tensor([2.0]))) / (2 * eps)
    gp = float((prof.grad * vp).sum())
    assert abs(gp - fdp) <= 1e-5 * abs(fdp), (gp, fdp)
    print(f"{case}: d/dprofile {gp:.10e} (fd {fdp:.10e}), d/dN {gN:.10e} (fd {fdN:.10e})")
    assert abs(fdp) > 1e-6 and abs(fdN) > 1e-6  # both directions move the loss


def test_mixed_precision_adjoint_matches_fp64_adjoint(cuda):
    """FP32 multigrid-preconditioned solves inside FP64 refinement give the FP64 gradient."""
    grads = []
    for mixed in (False, True):
        dom = duct_3d(8, 6, 5, 2)
        seeded_state(dom, 12, scale=0.1)
        dom.PrepareSolve()
        blocks = dom.getBlocks()
        model = AdjointMHD(dom, 0.01, torch.tensor([1.5]), torch.tensor([0.0, 1.0, 0.0], dtype=torch.float64), steps=2,
                           faces=[(blocks[0], "-x"), (blocks[-1], "+x")], checkpoint_every=1, tol=1e-12,
                           mixed_precision=mixed)
        prof = model.faces[0]._velocity.detach().clone().requires_grad_(True)
        N = torch.tensor([1.5], dtype=torch.float64, requires_grad=True)
        u = rollout(model, prof, N)
        (u * u).sum().backward()
        grads.append((prof.grad.clone(), N.grad.clone()))
    rel = float((grads[1][0] - grads[0][0]).abs().max() / grads[0][0].abs().max())
    assert rel < 1e-7, rel
    assert abs(float(grads[1][1] - grads[0][1])) <= 1e-7 * abs(float(grads[0][1]))


def test_checkpointing_does_not_change_the_gradient(cuda):
    grads = []
    for every in (1, 4):
        dom = duct_3d(6, 5, 4, 2)
        seeded_state(dom, 11, scale=0.1)
        dom.PrepareSolve()
        blocks = dom.getBlocks()
        model = AdjointMHD(dom, 0.01, torch.tensor([2.0]), torch.tensor([0.0, 1.0, 0.0], dtype=torch.float64), steps=4,
                           faces=[(blocks[0], "-x"), (blocks[-1], "+x")], checkpoint_every=every)
        prof = model.faces[0]._velocity.detach().clone().requires_grad_(True)
        N = torch.tensor([2.0], dtype=torch.float64, requires_grad=True)
        u = rollout(model, prof, N)
        u.sum().backward()
        grads.append((prof.grad.clone(), N.grad.clone()))
    assert torch.allclose(grads[0][0], grads[1][0], rtol=1e-9, atol=1e-12)
    assert torch.allclose(grads[0][1], grads[1][1], rtol=1e-9)
