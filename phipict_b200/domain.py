"""Host model of a multi-block domain: the phipict_b200 mirror of phiPICT's ``Domain``,
``Block`` and boundary classes (csrc/phipict/bindings.cpp:92-620, domain/*.cpp).

The classes keep phiPICT's names, argument meaning and error behaviour. What differs is
the storage: after :meth:`Domain.PrepareSolve` every block field is a *view* into one flat
device buffer per field (``[B][dims][cells]`` for vectors, ``[B][cells]`` for scalars, the
layout of phiPICT's flat solve vectors), so copying results back to the blocks is a single
device copy and the kernels never gather from per-block tensors. The topology (block sizes,
face types, connection axes, fixed-face data offsets) is packed into int32 records that the
CUDA kernels read directly (``include/phipict_b200.h``).
"""
from __future__ import annotations

import ctypes as ct
import math
from enum import IntEnum
from typing import Sequence

import torch

from . import _lib
from ._lib import BREC, FREC, IREC, TILE


class BoundaryType(IntEnum):
    DIRICHLET = 0
    DIRICHLET_VARYING = 1
    NEUMANN = 10
    CONNECTED_GRID = 20
    PERIODIC = 21
    FIXED = 30


class BoundaryConditionType(IntEnum):
    DIRICHLET = 0
    NEUMANN = 1


class PotentialBC(IntEnum):
    """Electric potential condition of a fixed face (domain/domain_structs_gpu.h PotentialBC)."""
    INSULATING = 0
    OPEN = 1
    DIRICHLET = 2
    THIN_WALL = 3


class AdvectionScheme(IntEnum):
    CENTRAL = 0
    LINEAR_UPWIND = 1


_FACES = {"-x": 0, "+x": 1, "-y": 2, "+y": 3, "-z": 4, "+z": 5}
_AXES = {"x": 0, "y": 1, "z": 2}


def face_index(face: int | str) -> int:
    if isinstance(face, str):
        if face not in _FACES:
            raise ValueError(f"unknown face '{face}', expected one of {list(_FACES)}")
        return _FACES[face]
    return int(face)


def axis_index(axis: int | str) -> int:
    if isinstance(axis, str):
        if axis not in _AXES:
            raise ValueError(f"unknown axis '{axis}'")
        return _AXES[axis]
    return int(axis)


def _face_string(face: int) -> str:
    return [k for k, v in _FACES.items() if v == face][0]


class Boundary:
    type: BoundaryType

    def __init__(self, domain: "Domain"):
        self._domain = domain

    def getParentDomain(self) -> "Domain":
        return self._domain

    def __str__(self) -> str:
        return f"{type(self).__name__}()"


class PeriodicBoundary(Boundary):
    type = BoundaryType.PERIODIC


class ConnectedBoundary(Boundary):
    """Connection to another block. ``axes`` uses phiPICT's encoding
    (domain/boundaries.cpp:857-891): axes[0] is the connected face of the other block,
    axes[1], axes[2] the faces the tangential axes map to, the lowest bit meaning inversion."""
    type = BoundaryType.CONNECTED_GRID

    def __init__(self, domain: "Domain", block: "Block", axes: list[int]):
        super().__init__(domain)
        self.connectedBlock = block
        self.axes = list(axes)

    def getConnectedBlock(self) -> "Block":
        return self.connectedBlock

    def __str__(self) -> str:
        return f"ConnectedBoundary(block={self.connectedBlock.name}, axes={self.axes})"


class FixedBoundary(Boundary):
    """A prescribed face: a velocity condition plus the electric potential condition.

    Velocity is Dirichlet (a value) or Neumann (open, zero gradient); it is either static,
    shape ``[1 or B, dims]``, or varying, shape ``[1 or B, dims, *face]`` with size 1 along
    the face normal (domain/boundaries.cpp).
    """
    type = BoundaryType.FIXED

    def __init__(self, domain: "Domain", block: "Block", face: int, velocity: torch.Tensor | None,
                 velocity_type: BoundaryConditionType, passiveScalar: torch.Tensor | None = None,
                 passiveScalarType=None):
        super().__init__(domain)
        self._block = block
        self._face = face
        d = block.getSpatialDims()
        if velocity is None:
            velocity = torch.zeros(1, d, dtype=domain.getDtype(), device=domain.getDevice())
        # a differentiable simulation takes the boundary velocity as an input of the graph
        self._velocity_ag = velocity if velocity.requires_grad else None
        self._velocity = self._check_velocity(velocity.detach())
        self._velocityType = BoundaryConditionType(velocity_type)
        self._potentialType = PotentialBC.INSULATING
        self._potentialTypes: torch.Tensor | None = None
        self._potentialValues: torch.Tensor | None = None
        self._cw = 0.0
        # passive scalar (domain/boundaries.cpp:100-120): given values, or static zeros when the
        # domain carries scalars; the type defaults to the velocity type
        self._passiveScalar: torch.Tensor | None = None
        self._passiveScalarTypes: list[BoundaryConditionType] | None = None
        self._scalar_ag = passiveScalar if passiveScalar is not None and passiveScalar.requires_grad else None
        if passiveScalar is not None:
            self._passiveScalar = self._check_scalar(passiveScalar)
        elif domain.hasPassiveScalar():
            self._passiveScalar = torch.zeros(1, domain.getPassiveScalarChannels(), dtype=domain.getDtype(),
                                              device=domain.getDevice())
        if self._passiveScalar is not None:
            t = passiveScalarType if passiveScalarType is not None else self._velocityType
            self._passiveScalarTypes = [BoundaryConditionType(v) for v in (t if isinstance(t, (list, tuple)) else [t])]

    # --- geometry ---
    def getSpatialDims(self) -> int:
        return self._block.getSpatialDims()

    def face_shape(self) -> list[int]:
        """Spatial shape of the face cells, ``[(z,) y, x]`` with 1 along the normal."""
        sizes = list(self._block.getSizes()[: self.getSpatialDims()])
        sizes[self._face >> 1] = 1
        return list(reversed(sizes))

    def face_cells(self) -> int:
        return math.prod(self.face_shape())

    def getSizes(self) -> list[int]:
        return self.face_shape()

    def hasSize(self) -> bool:
        return True

    def getDevice(self) -> torch.device:
        return self._domain.getDevice()

    def hasTransform(self) -> bool:
        return self._block.hasVertexCoordinates()

    # --- velocity ---
    def _check_velocity(self, v: torch.Tensor) -> torch.Tensor:
        d = self.getSpatialDims()
        v = v.to(device=self._domain.getDevice(), dtype=self._domain.getDtype())
        if v.dim() == 1:
            v = v.view(1, -1)
        if v.dim() == 2:
            if v.shape[1] != d:
                raise RuntimeError(f"static boundary velocity must have shape [B, {d}], got {tuple(v.shape)}")
        else:
            want = self.face_shape()
            if v.dim() != d + 2 or v.shape[1] != d or list(v.shape[2:]) != want:
                raise RuntimeError(f"varying boundary velocity must have shape [B, {d}, {want}], got {tuple(v.shape)}")
        return v.contiguous()

    @property
    def velocity(self) -> torch.Tensor:
        return self._velocity

    def isVelocityStatic(self) -> bool:
        return self._velocity.dim() == 2

    def setVelocity(self, velocity: torch.Tensor) -> None:
        v = self._check_velocity(velocity)
        # a differentiable simulation takes the boundary velocity as an input of the graph
        self._velocity_ag = velocity if velocity.requires_grad else None
        v = v.detach()
        if v.shape == self._velocity.shape and self._domain._prepared_for(self):
            self._velocity.copy_(v)
        else:
            self._velocity = v
            self._domain._invalidate()
        self._domain._bump()

    @property
    def velocityType(self) -> BoundaryConditionType:
        return self._velocityType

    def setVelocityType(self, t: BoundaryConditionType) -> None:
        self._velocityType = BoundaryConditionType(t)
        self._domain._invalidate()

    def makeVelocityVarying(self, size=None) -> None:
        if not self.isVelocityStatic():
            return
        v = self._velocity
        shape = [v.shape[0], v.shape[1]] + self.face_shape()
        self._velocity = v.view(v.shape[0], v.shape[1], *([1] * self.getSpatialDims())).expand(shape).contiguous()
        self._domain._invalidate()

    def getVelocity(self, computational: bool = False) -> torch.Tensor:
        return self._velocity

    def getVelocityVarying(self, size=None) -> torch.Tensor:
        if self.isVelocityStatic():
            v = self._velocity
            return v.view(v.shape[0], v.shape[1], *([1] * self.getSpatialDims())).expand(
                [v.shape[0], v.shape[1]] + self.face_shape())
        return self._velocity

    def GetFluxes(self) -> torch.Tensor:
        """Contravariant normal fluxes of the face cells, ``[B, 1, *face]``."""
        return self._domain._boundary_fluxes(self)

    # --- passive scalar (domain/boundaries.cpp:372-440) ---
    def _check_scalar(self, ps: torch.Tensor) -> torch.Tensor:
        d, C = self.getSpatialDims(), self._domain.getPassiveScalarChannels()
        ps = ps.to(device=self._domain.getDevice(), dtype=self._domain.getDtype())
        if C < 1:
            raise RuntimeError("Passive scalars are not active.")
        if ps.dim() < 2 or ps.shape[0] < 1 or ps.shape[1] != C:
            raise RuntimeError("Passive scalar channels must match domain.")
        if ps.dim() not in (2, 2 + d):
            raise RuntimeError("Passive Scalar must be static (shape NC) or varying (shape NC + face spatial shape).")
        if ps.dim() == 2 + d and list(ps.shape[2:]) != self.face_shape():
            raise RuntimeError(f"varying passive scalar must have the face shape {self.face_shape()}")
        return ps.detach().contiguous()

    @property
    def passiveScalar(self) -> torch.Tensor | None:
        return self._passiveScalar

    @property
    def passiveScalarTypes(self) -> list[BoundaryConditionType] | None:
        return None if self._passiveScalarTypes is None else list(self._passiveScalarTypes)

    def hasPassiveScalar(self) -> bool:
        return self._passiveScalar is not None

    def getPassiveScalarChannels(self) -> int:
        return self._domain.getPassiveScalarChannels()

    def setPassiveScalar(self, passiveScalar: torch.Tensor) -> None:
        # a differentiable simulation takes the boundary scalar as an input of the graph
        self._scalar_ag = passiveScalar if passiveScalar.requires_grad else None
        ps = self._check_scalar(passiveScalar)
        if self._passiveScalar is not None and ps.shape == self._passiveScalar.shape and self._domain._prepared_for(self):
            self._passiveScalar.copy_(ps)
        else:
            self._passiveScalar = ps
            self._domain._invalidate()
        if self._passiveScalarTypes is None:
            self._passiveScalarTypes = [self._velocityType]
        self._domain._bump()

    def CreatePassiveScalar(self, createStatic: bool = True) -> None:
        C = self.getPassiveScalarChannels()
        shape = [1, C] if createStatic else [1, C] + self.face_shape()
        self.setPassiveScalar(torch.zeros(shape, dtype=self._domain.getDtype(), device=self._domain.getDevice()))

    def isPassiveScalarStatic(self) -> bool:
        return self._passiveScalar is None or self._passiveScalar.dim() == 2

    def setPassiveScalarType(self, types) -> None:
        """One type for every channel, or one per channel (Dirichlet: a value; Neumann: the
        physical gradient along the outward normal)."""
        if self._passiveScalar is None:
            raise RuntimeError("FixedBoundary has not passive scalar.")
        t = list(types) if isinstance(types, (list, tuple)) else [types]
        if len(t) not in (1, self.getPassiveScalarChannels()):
            raise RuntimeError("Passive scalar boundary conditions must be static or match channels.")
        self._passiveScalarTypes = [BoundaryConditionType(v) for v in t]
        self._domain._invalidate()

    def isPassiveScalarBoundaryTypeStatic(self) -> bool:
        return self._passiveScalarTypes is None or len(self._passiveScalarTypes) == 1

    def _scalar_types(self) -> list[int]:
        C = self.getPassiveScalarChannels()
        t = self._passiveScalarTypes or [BoundaryConditionType.DIRICHLET]
        return [int(t[0] if len(t) == 1 else t[c]) for c in range(C)]

    # --- electric potential (domain/boundaries.cpp:900-965) ---
    def setPotentialBC(self, type: PotentialBC, cw: float | None = None) -> None:
        type = PotentialBC(type)
        if type == PotentialBC.THIN_WALL:
            if cw is None or not cw > 0:
                raise RuntimeError("A THIN_WALL potential BC needs a wall conductance ratio cw > 0.")
            self._cw = float(cw)
        else:
            if cw not in (None, 0, 0.0):
                raise RuntimeError("cw is only valid for a THIN_WALL potential BC.")
            self._cw = 0.0
        self._potentialType = type
        self._potentialTypes = None
        self._domain._invalidate()

    def getPotentialBC(self) -> PotentialBC:
        return self._potentialType

    def getPotentialCw(self) -> float:
        return self._cw

    # legacy flag interface over the potential BC (domain/boundaries.cpp:968-991,
    # domain/domain_structs.h:244-249), used by files written before PotentialBC existed
    def setEpotCw(self, cw: float) -> None:
        if not cw >= 0.0:
            raise RuntimeError("Epot wall conductance Cw must be non-negative.")
        if cw > 0.0:
            self.setPotentialBC(PotentialBC.THIN_WALL, cw)
        elif self._potentialType == PotentialBC.THIN_WALL:
            self.setPotentialBC(PotentialBC.INSULATING)

    def setEpotDirichlet(self, dirichlet: bool) -> None:
        if dirichlet:
            self.setPotentialBC(PotentialBC.DIRICHLET)
        elif self._potentialType == PotentialBC.DIRICHLET:
            self.setPotentialBC(PotentialBC.INSULATING)

    def setEpotInsulating(self, insulating: bool) -> None:
        if not insulating:
            self.setPotentialBC(PotentialBC.OPEN)
        elif self._potentialType == PotentialBC.OPEN:
            self.setPotentialBC(PotentialBC.INSULATING)

    def hasEpotCw(self) -> bool:
        return self.hasPotentialThinWall() and self._cw > 0.0

    def getEpotCw(self) -> float:
        return self._cw if self.hasPotentialThinWall() else 0.0

    def hasEpotDirichlet(self) -> bool:
        return self.hasPotentialDirichlet()

    def isEpotInsulating(self) -> bool:
        return self._potentialType != PotentialBC.OPEN

    def setPotentialTypes(self, types: torch.Tensor, cw: float | None = None) -> None:
        d = self.getSpatialDims()
        if types.dim() != d + 2 or types.shape[0] != 1 or types.shape[1] != 1:
            raise RuntimeError("Potential BC types must have shape [1,1,(D),H,W] with size 1 along the face normal.")
        if types.is_floating_point() or types.dtype == torch.bool:
            raise RuntimeError("Potential BC types must be an integer tensor of PotentialBC values.")
        if types.numel() == 0:
            raise RuntimeError("Potential BC types must not be empty.")
        tmin, tmax = int(types.min()), int(types.max())
        if tmin < 0 or tmax > 3:
            raise RuntimeError("Potential BC types contain values that are not PotentialBC members.")
        if list(types.shape[2:]) != self.face_shape():
            raise RuntimeError(f"Potential BC types must cover the face {self.face_shape()}.")
        if bool((types == PotentialBC.THIN_WALL).any()):
            if cw is None or not cw > 0:
                raise RuntimeError("Potential BC types contain THIN_WALL cells but no wall conductance ratio cw was given.")
            self._cw = float(cw)
        else:
            if cw not in (None, 0, 0.0):
                raise RuntimeError("cw is only valid if some cells are THIN_WALL.")
            self._cw = 0.0
        self._potentialTypes = types.to(device=self._domain.getDevice(), dtype=torch.int8).contiguous()
        if tmin == tmax:
            self._potentialType = PotentialBC(tmin)
        self._domain._invalidate()

    def hasPotentialTypes(self) -> bool:
        return self._potentialTypes is not None

    def getPotentialTypes(self) -> torch.Tensor | None:
        return self._potentialTypes

    def clearPotentialTypes(self) -> None:
        self._potentialTypes = None
        self._domain._invalidate()

    def setPotentialValues(self, values: torch.Tensor) -> None:
        d = self.getSpatialDims()
        if values.dim() != d + 2 or values.shape[1] != 1:
            raise RuntimeError("Potential values must have shape [1 or batch,1,(D),H,W] with size 1 along the face normal.")
        if not values.is_floating_point():
            raise RuntimeError("Potential values must be a floating point tensor.")
        self._potentialValues = values.to(device=self._domain.getDevice(), dtype=self._domain.getDtype()).contiguous()
        self._domain._invalidate()

    def hasPotentialValues(self) -> bool:
        return self._potentialValues is not None

    def getPotentialValues(self) -> torch.Tensor | None:
        return self._potentialValues

    def clearPotentialValues(self) -> None:
        self._potentialValues = None
        self._domain._invalidate()

    def hasPotentialDirichlet(self) -> bool:
        if self._potentialTypes is not None:
            return bool((self._potentialTypes == PotentialBC.DIRICHLET).any())
        return self._potentialType == PotentialBC.DIRICHLET

    def hasPotentialThinWall(self) -> bool:
        if self._potentialTypes is not None:
            return bool((self._potentialTypes == PotentialBC.THIN_WALL).any())
        return self._potentialType == PotentialBC.THIN_WALL

    def __str__(self) -> str:
        kind = "static" if self.isVelocityStatic() else "varying"
        return (f"FixedBoundary(velocity={kind} {self._velocityType.name}, potential={self._potentialType.name}"
                f"{', mask' if self._potentialTypes is not None else ''})")


class Block:
    """A structured block of cells, x fastest (phiPICT domain/block.cpp)."""

    def __init__(self, domain: "Domain", name: str, sizes: list[int], velocity: torch.Tensor | None,
                 pressure: torch.Tensor | None, vertexCoordinates: torch.Tensor | None):
        self._domain = domain
        self.name = name
        d = domain.getSpatialDims()
        self._sizes = list(sizes) + [1] * (3 - len(sizes))  # x, y, z
        spatial = list(reversed(self._sizes[:d]))
        opts = dict(dtype=domain.getDtype(), device=domain.getDevice())
        B = domain.getBatchSize()
        self.velocity = velocity.detach().to(**opts).contiguous() if velocity is not None else torch.zeros(B, d, *spatial, **opts)
        self.pressure = pressure.detach().to(**opts).contiguous() if pressure is not None else torch.zeros(B, 1, *spatial, **opts)
        # inputs of a differentiable simulation's graph (set when a tensor that requires grad is
        # given; the block fields above hold their values)
        self._velocity_ag = velocity if velocity is not None and velocity.requires_grad else None
        self._source_ag: torch.Tensor | None = None
        self._epot_ag: torch.Tensor | None = None
        self._pressure_ag: torch.Tensor | None = None
        self._scalar_ag: torch.Tensor | None = None
        self.epot: torch.Tensor | None = None
        self.passiveScalar: torch.Tensor | None = None
        if domain.hasPassiveScalar():
            self.passiveScalar = torch.zeros(B, domain.getPassiveScalarChannels(), *spatial, **opts)
        self.velocitySource: torch.Tensor | None = None
        self.vertexCoordinates = vertexCoordinates.to(**opts).contiguous() if vertexCoordinates is not None else None
        self._boundaries: list[Boundary] = [PeriodicBoundary(domain) for _ in range(2 * d)]
        self.globalOffset = 0
        self.csrOffset = 0

    # --- geometry ---
    def getSpatialDims(self) -> int:
        return self._domain.getSpatialDims()

    def getSizes(self) -> list[int]:
        return list(self._sizes)

    def getStrides(self):
        nx, ny, nz = self._sizes
        return _Int4(1, nx, nx * ny, nx * ny * nz)

    def ncells(self) -> int:
        return math.prod(self._sizes)

    def getDevice(self) -> torch.device:
        return self._domain.getDevice()

    def getParentDomain(self) -> "Domain":
        return self._domain

    def hasVertexCoordinates(self) -> bool:
        return self.vertexCoordinates is not None

    def hasTransform(self) -> bool:
        return self.vertexCoordinates is not None

    def setVertexCoordinates(self, vertexCoordinates: torch.Tensor) -> None:
        self.vertexCoordinates = vertexCoordinates.to(dtype=self._domain.getDtype(), device=self._domain.getDevice()).contiguous()
        self._domain._invalidate()

    def getCellCoordinates(self) -> torch.Tensor:
        if self.vertexCoordinates is None:
            raise RuntimeError("block has no vertex coordinates")
        v = self.vertexCoordinates
        d = self.getSpatialDims()
        c = v
        for ax in range(d):
            dim = 2 + ax
            c = 0.5 * (c.narrow(dim, 0, c.shape[dim] - 1) + c.narrow(dim, 1, c.shape[dim] - 1))
        return c

    # --- fields ---
    def setVelocity(self, velocity: torch.Tensor) -> None:
        v = velocity.to(dtype=self._domain.getDtype(), device=self._domain.getDevice())
        if v.shape != self.velocity.shape:
            raise RuntimeError(f"velocity must have shape {tuple(self.velocity.shape)}, got {tuple(v.shape)}")
        self._domain._restore_block_views(self, ("velocity",))
        self._velocity_ag = velocity if velocity.requires_grad else None
        self.velocity.copy_(v.detach())

    def setPressure(self, pressure: torch.Tensor) -> None:
        self.pressure.copy_(pressure.to(dtype=self._domain.getDtype(), device=self._domain.getDevice()))

    def hasVelocitySource(self) -> bool:
        return self.velocitySource is not None

    def setVelocitySource(self, source: torch.Tensor) -> None:
        """Static ``[1 or B, dims]`` or per cell ``[1 or B, dims, *spatial]``."""
        d = self.getSpatialDims()
        s = source.to(dtype=self._domain.getDtype(), device=self._domain.getDevice())
        if s.dim() == 1:
            s = s.view(1, -1)
        if s.shape[1] != d or s.dim() not in (2, d + 2):
            raise RuntimeError(f"velocity source must be [B, {d}] or [B, {d}, *spatial], got {tuple(s.shape)}")
        self._source_ag = s if s.requires_grad else None
        self._domain._source_writes += 1
        self._domain._set_block_source(self, s.detach())

    def clearVelocitySource(self) -> None:
        self._source_ag = None
        self._domain._source_writes += 1
        self._domain._set_block_source(self, None)

    def setEpot(self, epot: torch.Tensor) -> None:
        """The electric potential [B, 1, *spatial]; before SetupEpotOnDomain it is kept and
        taken over when the potential fields are allocated."""
        self._epot_ag = epot if epot.requires_grad else None
        e = epot.detach().to(dtype=self._domain.getDtype(), device=self._domain.getDevice())
        if self.epot is None:
            self.epot = e.contiguous()
            return
        self.epot.copy_(e)

    def hasEpot(self) -> bool:
        return self.epot is not None

    # --- passive scalar (domain/block.cpp:347-377) ---
    def hasPassiveScalar(self) -> bool:
        return self._domain.hasPassiveScalar()

    def getPassiveScalarChannels(self) -> int:
        return self._domain.getPassiveScalarChannels()

    def setPassiveScalar(self, passiveScalar: torch.Tensor) -> None:
        C = self.getPassiveScalarChannels()
        if C < 1:
            raise RuntimeError("Passive scalars are not active.")
        d = self.getSpatialDims()
        s = passiveScalar.to(dtype=self._domain.getDtype(), device=self._domain.getDevice())
        want = [C] + list(reversed(self._sizes[:d]))
        if s.dim() != d + 2 or list(s.shape[1:]) != want:
            raise RuntimeError(f"passive scalar must have shape [B, {C}, *spatial], got {tuple(s.shape)}")
        if self._domain._prepared:
            self._domain._restore_block_views(self, ("passiveScalar",))
        self._scalar_ag = passiveScalar if passiveScalar.requires_grad else None
        s = s.detach()
        if self.passiveScalar is not None and s.shape == self.passiveScalar.shape:
            self.passiveScalar.copy_(s)
        else:
            self.passiveScalar = s.contiguous()
            self._domain._invalidate()

    def CreatePassiveScalar(self) -> None:
        C = self.getPassiveScalarChannels()
        if C < 1:
            raise RuntimeError("Passive scalars are not active.")
        d = self.getSpatialDims()
        self.setPassiveScalar(torch.zeros(self._domain.getBatchSize(), C, *reversed(self._sizes[:d]),
                                          dtype=self._domain.getDtype(), device=self._domain.getDevice()))

    @property
    def passiveScalarViscosity(self) -> torch.Tensor | None:
        return None

    def hasPassiveScalarViscosity(self) -> bool:
        return False

    def isAllFixedBoundariesPassiveScalarTypeStatic(self) -> bool:
        return all(b.isPassiveScalarBoundaryTypeStatic() for _, b in self.getFixedBoundaries())

    # --- boundaries ---
    def getBoundary(self, face: int | str) -> Boundary:
        return self._boundaries[face_index(face)]

    def getBoundaries(self) -> list[Boundary]:
        return list(self._boundaries)

    def getFixedBoundaries(self) -> list[tuple[int, FixedBoundary]]:
        return [(i, b) for i, b in enumerate(self._boundaries) if isinstance(b, FixedBoundary)]

    def hasPrescribedBoundary(self) -> bool:
        return any(isinstance(b, FixedBoundary) for b in self._boundaries)

    def _check_face(self, face: int) -> None:
        if not 0 <= face < 2 * self.getSpatialDims():
            raise RuntimeError(f"face index {face} out of range")

    def _close_connection(self, face: int) -> None:
        b = self._boundaries[face]
        if isinstance(b, ConnectedBoundary):
            other = b.connectedBlock
            oface = b.axes[0]
            ob = other._boundaries[oface]
            if isinstance(ob, ConnectedBoundary) and ob.connectedBlock is self:
                other._boundaries[oface] = FixedBoundary(self._domain, other, oface, None, BoundaryConditionType.DIRICHLET)

    def _set_boundary(self, face: int, b: Boundary) -> None:
        self._boundaries[face] = b
        self._domain._invalidate()

    def CloseBoundary(self, face: int | str, velocity: torch.Tensor | None = None, passiveScalar=None) -> None:
        """A no-slip (velocity given: Dirichlet) wall or inflow (domain/block.cpp:960-964); the
        passive scalar is Dirichlet (zero unless given)."""
        f = face_index(face)
        self._check_face(f)
        self._close_connection(f)
        self._set_boundary(f, FixedBoundary(self._domain, self, f, velocity, BoundaryConditionType.DIRICHLET,
                                            passiveScalar))

    def OpenBoundary(self, face: int | str, passiveScalar=None) -> None:
        """A zero-gradient (Neumann) velocity face (domain/block.cpp:969-977); the passive scalar
        is Neumann too (zero gradient unless given)."""
        f = face_index(face)
        self._check_face(f)
        self._close_connection(f)
        self._set_boundary(f, FixedBoundary(self._domain, self, f, None, BoundaryConditionType.NEUMANN, passiveScalar,
                                            BoundaryConditionType.NEUMANN))

    def CloseAllBoundaries(self) -> None:
        for f in range(2 * self.getSpatialDims()):
            self.CloseBoundary(f)

    def MakePeriodic(self, axis: int | str) -> None:
        a = axis_index(axis)
        if not 0 <= a < self.getSpatialDims():
            raise RuntimeError(f"axis {axis} out of range")
        for f in (2 * a, 2 * a + 1):
            self._close_connection(f)
            if not isinstance(self._boundaries[f], PeriodicBoundary):
                self._set_boundary(f, PeriodicBoundary(self._domain))

    def MakeAllPeriodic(self) -> None:
        for a in range(self.getSpatialDims()):
            self.MakePeriodic(a)

    def ConnectBlock(self, face: int | str, otherBlock: "Block", otherFace: int | str,
                     axis1: int | str = -1, axis2: int | str = -1) -> None:
        """Connect face ``face`` of this block to ``otherFace`` of ``otherBlock``; ``axis1``
        (and ``axis2`` in 3D) name the faces of the other block that this block's next
        tangential axes map to (ConnectBlocks, domain/boundaries.cpp:857-891)."""
        f1, f2 = face_index(face), face_index(otherFace)
        a1 = face_index(axis1) if isinstance(axis1, str) else int(axis1)
        a2 = face_index(axis2) if isinstance(axis2, str) else int(axis2)
        if otherBlock._domain is not self._domain:
            raise RuntimeError("The blocks must belong to the same domain.")
        d = self.getSpatialDims()
        self._check_face(f1)
        otherBlock._check_face(f2)
        self._close_connection(f1)
        otherBlock._close_connection(f2)
        axes1 = [f2]
        axes2 = [f1]
        if d > 1:
            axes1.append(a1)
            f1d, f2d = f1 >> 1, f2 >> 1
            swapped = False
            if d == 2 or (a1 >> 1) == (f2d + 1) % d:
                axes2.append((((f1d + 1) % d) << 1) | (a1 & 1))
            else:
                if (a2 >> 1) != (f2d + 1) % d:
                    raise RuntimeError("Invalid connection.")
                axes2.append((((f1d + 2) % d) << 1) | (a2 & 1))
                swapped = True
            if d > 2:
                axes1.append(a2)
                if not swapped:
                    axes2.append((((f1d + 2) % d) << 1) | (a2 & 1))
                else:
                    axes2.append((((f1d + 1) % d) << 1) | (a1 & 1))
        self._set_boundary(f1, ConnectedBoundary(self._domain, otherBlock, axes1))
        otherBlock._set_boundary(f2, ConnectedBoundary(self._domain, self, axes2))

    def __str__(self) -> str:
        return f"Block({self.name}, size={self._sizes[:self.getSpatialDims()]})"


class _Int4:
    def __init__(self, x, y, z, w):
        self.x, self.y, self.z, self.w = x, y, z, w

    def __getitem__(self, i):
        return (self.x, self.y, self.z, self.w)[i]

    def __len__(self):
        return 4


class CSRmatrix:
    """A CSR view (``row``, ``index``, ``value``) of a stencil matrix of a domain, or a plain
    CSR matrix (csrc/phipict/domain/csr_matrix.cpp). For domain matrices the values are
    gathered from the stencil on access, shape ``[B*nnz]`` in batch order."""

    def __init__(self, value: torch.Tensor | None = None, index: torch.Tensor | None = None,
                 row: torch.Tensor | None = None, *, _domain: "Domain | None" = None, _which: str = ""):
        self._domain = _domain
        self._which = _which
        self._value = value
        self.index = index
        self.row = row

    @property
    def value(self) -> torch.Tensor:
        if self._domain is not None:
            return self._domain._csr_values(self._which)
        return self._value

    @value.setter
    def value(self, v: torch.Tensor) -> None:
        if self._domain is not None:
            self._domain._set_csr_values(self._which, v)
        else:
            self._value = v

    def setValue(self, v: torch.Tensor) -> None:
        self.value = v

    def getRows(self) -> int:
        return int(self.row.numel() - 1)

    def getSize(self) -> int:
        return self.getNnz()

    def getNnz(self) -> int:
        return int(self.index.numel())

    def getBatchSize(self) -> int:
        return int(self.value.numel() // max(1, self.getNnz()))

    def getDevice(self) -> torch.device:
        return self.row.device

    def toType(self, dtype: torch.dtype) -> "CSRmatrix":
        return CSRmatrix(self.value.to(dtype), self.index, self.row)

    def clone(self) -> "CSRmatrix":
        return CSRmatrix(self.value.clone(), self.index, self.row)

    def detach(self) -> None:
        pass

    def stencil_source(self):
        """(domain, which) if this is a domain matrix the stencil solvers can use directly."""
        return (self._domain, self._which) if self._domain is not None else None

    def __str__(self) -> str:
        return f"CSRmatrix(rows={self.getRows()}, nnz={self.getNnz()})"


class Domain:
    """Multi-block domain (csrc/phipict/domain/domain.cpp), a drop-in for ``phipict.Domain``."""

    def __init__(self, spatialDims: int, viscosity: torch.Tensor | float, name: str = "Domain",
                 dtype: torch.dtype = torch.float32, device: torch.device | str = "cuda",
                 passiveScalarChannels: int = 1, scalarViscosity: torch.Tensor | None = None):
        if spatialDims not in (2, 3):
            raise RuntimeError("phipict_b200 supports 2D and 3D domains")
        self.name = name
        self._dims = int(spatialDims)
        self._dtype = dtype
        self._device = torch.device(device)
        if self._device.type == "cuda" and self._device.index is None:
            self._device = torch.device("cuda", torch.cuda.current_device() if torch.cuda.is_available() else 0)
        _lib.dtype_code(dtype)
        v = viscosity if isinstance(viscosity, torch.Tensor) else torch.tensor([float(viscosity)])
        self.viscosity = v.detach().to("cpu", torch.float64).reshape(-1).clone()
        # the autograd input of a differentiable simulation (phiPICT's tracked VISCOSITY)
        self._viscosity_ag = v if v.requires_grad else None
        self._blocks: list[Block] = []
        self._batch = 1
        self._prepared = False
        self._version = 0
        self._source_writes = 0  # velocity-source assignments (a differentiable step watches them)
        self._epot_on = False
        self._epot_flags = (0, False)
        self._advection_scheme = AdvectionScheme.CENTRAL
        self._timestep = torch.ones(1, dtype=torch.float64)
        if int(passiveScalarChannels) < 0:
            raise RuntimeError("passiveScalarChannels must not be negative")
        self._scalar_channels = int(passiveScalarChannels)
        self.passiveScalarViscosity: torch.Tensor | None = None
        if scalarViscosity is not None:
            self.setPassiveScalarViscosity(scalarViscosity)

    # --- basic accessors ---
    def getSpatialDims(self) -> int:
        return self._dims

    def getDtype(self) -> torch.dtype:
        return self._dtype

    def getDevice(self) -> torch.device:
        return self._device

    def getBlocks(self) -> list[Block]:
        return list(self._blocks)

    def getBlock(self, i: int) -> Block:
        return self._blocks[i]

    def getNumBlocks(self) -> int:
        return len(self._blocks)

    def getBatchSize(self) -> int:
        return self._batch

    def getTotalSize(self) -> int:
        return sum(b.ncells() for b in self._blocks)

    def numCells(self) -> int:
        """Cells of all batched environments (the length of a scalar field)."""
        return self.getTotalSize() * self._batch

    def IsInitialized(self) -> bool:
        return self._prepared

    def hasNonOrthogonalMetrics(self) -> bool:
        """Whether any cell transform has a cross term Minv[a] . Minv[b] != 0 (a != b), or a
        fixed-face transform one above 1e-10 of |Minv[a]| |Minv[b]|. The face transforms of a
        rectilinear block carry rounding-level cross terms (about 1e-14 relative) from their
        vertex averages; below that bound the cross terms are zero, or change a right-hand
        side by rounding only, and the step may leave them out. PrepareSolve() must have run."""
        if not self._prepared:
            raise RuntimeError("Domain is not initialized. Run domain.PrepareSolve() first.")
        key = (self._metrics.data_ptr(), self._face_metrics.data_ptr(), self._version)
        cached = self.__dict__.get("_cross_terms")
        if cached is not None and cached[0] == key:
            return cached[1]
        d = self._dims
        found = False
        for m, rtol in ((self._metrics, 0.0), (self._face_metrics, 1e-10)):
            rows = m[d * d:2 * d * d].view(d, d, -1)
            for a in range(d):
                for b in range(a + 1, d):
                    cross = (rows[a] * rows[b]).sum(0).abs()
                    bound = rtol * rows[a].norm(dim=0) * rows[b].norm(dim=0)
                    if bool((cross > bound).any()):
                        found = True
        self._cross_terms = (key, found)
        return found

    # --- passive scalar (domain/domain.cpp:618-636) ---
    def hasPassiveScalar(self) -> bool:
        return self._scalar_channels > 0

    def getPassiveScalarChannels(self) -> int:
        return self._scalar_channels

    def setPassiveScalarViscosity(self, scalarViscosity) -> None:
        """The scalar diffusivity: one value for every channel, or one per channel."""
        v = scalarViscosity if isinstance(scalarViscosity, torch.Tensor) else torch.tensor([float(scalarViscosity)])
        v = v.detach().to("cpu", torch.float64).reshape(-1).clone()
        if v.numel() not in (1, max(1, self._scalar_channels)):
            raise RuntimeError("scalar viscosity must have 1 or one-per-channel entries")
        self.passiveScalarViscosity = v
        if getattr(self, "_prepared", False):
            self._upload_scalar_viscosity()

    def hasPassiveScalarViscosity(self) -> bool:
        return self.passiveScalarViscosity is not None

    def isPassiveScalarViscosityStatic(self) -> bool:
        return self.passiveScalarViscosity is None or self.passiveScalarViscosity.numel() == 1

    def hasPassiveScalarBlockViscosity(self) -> bool:
        return False

    def isAllFixedBoundariesPassiveScalarTypeStatic(self) -> bool:
        return all(b.isAllFixedBoundariesPassiveScalarTypeStatic() for b in self._blocks)

    def CreatePassiveScalarOnBlocks(self) -> None:
        if self.hasPassiveScalar():
            for b in self._blocks:
                b.CreatePassiveScalar()

    def setScalarResult(self, result: torch.Tensor) -> None:
        r = result.detach().reshape(-1)
        if r.numel() != self.scalarResult.numel():
            raise RuntimeError(f"scalar result must have {self.scalarResult.numel()} values")
        self.scalarResult.copy_(r)

    def CreateScalarResult(self) -> None:
        self.scalarResult.zero_()

    def _set_vector(self, name: str, value: torch.Tensor) -> None:
        """Domain::set<Vector> (domain.cpp:644-760): the values of a solve vector, [B*comp*n]
        in the domain's dtype on its device. They are copied into the domain's own buffer,
        whose address the prepared descriptors and cached solver graphs hold."""
        cur = getattr(self, name, None)
        if cur is None:
            raise RuntimeError(f"{name}: the domain is not prepared (PrepareSolve)")
        if not isinstance(value, torch.Tensor) or value.device != cur.device or value.dtype != cur.dtype:
            raise RuntimeError(f"{name} must be a {cur.dtype} tensor on {cur.device}")
        if value.numel() != cur.numel():
            raise RuntimeError(f"{name} must have {cur.numel()} values, got {value.numel()}")
        if value.data_ptr() != cur.data_ptr():
            cur.copy_(value.detach().reshape(-1))

    def setA(self, a: torch.Tensor) -> None:
        self._set_vector("A", a)

    def setVelocityRHS(self, v: torch.Tensor) -> None:
        self._set_vector("velocityRHS", v)

    def setVelocityResult(self, v: torch.Tensor) -> None:
        self._set_vector("velocityResult", v)

    def setPressureRHS(self, v: torch.Tensor) -> None:
        self._set_vector("pressureRHS", v)

    def setPressureRHSdiv(self, v: torch.Tensor) -> None:
        self._set_vector("pressureRHSdiv", v)

    def setPressureResult(self, v: torch.Tensor) -> None:
        self._set_vector("pressureResult", v)

    def setScalarRHS(self, v: torch.Tensor) -> None:
        self._set_vector("scalarRHS", v)

    def setEpotRHS(self, v: torch.Tensor) -> None:
        self._set_vector("epotRHS", v)

    def setEpotResult(self, v: torch.Tensor) -> None:
        self._set_vector("epotResult", v)

    def GetCoordinateOrientation(self) -> int:
        """Domain/Block::GetCoordinateOrientation (domain.cpp:265-276, block.cpp:1091-1105):
        the sign of the cell volumes (det M) when all cells of all blocks share it, else 0; a
        block without vertex coordinates counts as +1."""
        signs = set()
        for b in self._blocks:
            if b.vertexCoordinates is None:
                signs.add(1)
                continue
            met = getattr(self, "_metrics", None)
            if met is None:
                raise RuntimeError("GetCoordinateOrientation needs a prepared domain (PrepareSolve)")
            det = met[-1, b.globalOffset:b.globalOffset + b.ncells()]
            lo, hi = int(torch.sign(det).min().item()), int(torch.sign(det).max().item())
            signs.add(lo if lo == hi else 0)
        if not signs:
            raise RuntimeError("Domain does not contain any blocks.")
        return signs.pop() if len(signs) == 1 else 0

    def getMaxVelocityMagnitude(self, withBounds: bool = True, computational: bool = False) -> torch.Tensor:
        """Largest velocity magnitude |u|_2 over cells (and, withBounds, fixed faces), all
        environments (domain.cpp:234-243, block.cpp:578-612)."""
        d = self._dims
        u = self._u_block
        if computational:
            u = _to_computational(u, self._metrics, d)
        m = torch.linalg.vector_norm(u, 2, dim=1).max()
        if withBounds:
            for k, (_, _, bd) in enumerate(self._fixed):
                v = bd._velocity
                if computational:
                    fc, to = self._fixed_cells[k], self._fixed_toff[k]
                    vv = v.reshape(v.shape[0], d, -1).expand(v.shape[0], d, fc) if v.dim() == 2 else v.reshape(v.shape[0], d, fc)
                    v = _to_computational(vv, self._face_metrics[:, to:to + fc], d)
                m = torch.maximum(m, torch.linalg.vector_norm(v.reshape(v.shape[0], d, -1), 2, dim=1).max())
        return m

    def hasVertexCoordinates(self) -> bool:
        return all(b.hasVertexCoordinates() for b in self._blocks)

    def getVertexCoordinates(self) -> list[torch.Tensor]:
        return [b.vertexCoordinates for b in self._blocks]

    def hasPrescribedBoundary(self) -> bool:
        return any(b.hasPrescribedBoundary() for b in self._blocks)

    def hasBlockViscosity(self) -> bool:
        return False

    def setViscosity(self, viscosity) -> None:
        v = viscosity if isinstance(viscosity, torch.Tensor) else torch.tensor([float(viscosity)])
        self.viscosity = v.detach().to("cpu", torch.float64).reshape(-1).clone()
        self._viscosity_ag = v if v.requires_grad else None
        if self._prepared:
            self._upload_viscosity()

    def setAdvectionScheme(self, scheme: AdvectionScheme) -> None:
        """CENTRAL (implicit central fluxes) or LINEAR_UPWIND (first-order upwind in the matrix
        with the linear-upwind part as a lagged explicit correction, where the far-upwind cell
        lies in the same block; domain_structs_gpu.h:65-68)."""
        self._advection_scheme = AdvectionScheme(scheme)
        if getattr(self, "_prepared", False):
            self._desc.scheme = int(self._advection_scheme)
            self._version += 1

    def getAdvectionScheme(self) -> AdvectionScheme:
        return self._advection_scheme

    def _bump(self) -> None:
        self._version += 1

    def _invalidate(self) -> None:
        self._prepared = False
        self._version += 1

    def _prepared_for(self, bound: FixedBoundary) -> bool:
        return self._prepared

    # --- construction ---
    def CreateBlock(self, velocity: torch.Tensor | None = None, pressure: torch.Tensor | None = None,
                    passiveScalar: torch.Tensor | None = None, vertexCoordinates: torch.Tensor | None = None,
                    name: str = "Block") -> Block:
        d = self._dims
        if vertexCoordinates is not None:
            if vertexCoordinates.dim() != d + 2 or vertexCoordinates.shape[0] != 1 or vertexCoordinates.shape[1] != d:
                raise RuntimeError(f"vertexCoordinates must have shape [1, {d}, *vertices]")
            sizes = [int(s) - 1 for s in reversed(vertexCoordinates.shape[2:])]
        elif velocity is not None:
            if velocity.dim() != d + 2 or velocity.shape[1] != d:
                raise RuntimeError(f"velocity must have shape [B, {d}, *spatial]")
            sizes = [int(s) for s in reversed(velocity.shape[2:])]
        elif pressure is not None:
            sizes = [int(s) for s in reversed(pressure.shape[2:])]
        else:
            raise RuntimeError("CreateBlock needs velocity, pressure or vertexCoordinates to know its size")
        if velocity is not None and [int(s) for s in reversed(velocity.shape[2:])] != sizes:
            raise RuntimeError("velocity and vertexCoordinates sizes do not match")
        if any(s < 1 for s in sizes):
            raise RuntimeError("block sizes must be positive")
        if velocity is not None and velocity.shape[0] != self._batch:
            if self._batch == 1:
                self._batch = int(velocity.shape[0])
            else:
                raise RuntimeError("velocity batch size does not match the domain")
        blk = Block(self, name, sizes, velocity, pressure, vertexCoordinates)
        if passiveScalar is not None:
            blk.setPassiveScalar(passiveScalar)
        self._blocks.append(blk)
        self._invalidate()
        return blk

    def CreateBlockWithSize(self, size, name: str = "Block") -> Block:
        s = [int(v) for v in (list(size) if not hasattr(size, "x") else [size.x, size.y, size.z])]
        d = self._dims
        spatial = list(reversed(s[:d]))
        vel = torch.zeros(self._batch, d, *spatial, dtype=self._dtype, device=self._device)
        return self.CreateBlock(velocity=vel, name=name)

    def setBatchSize(self, batchSize: int) -> None:
        """Repeat every block's state from batch size 1 to ``batchSize`` (domain.cpp:1348-1368)."""
        B = int(batchSize)
        if B < 1:
            raise RuntimeError("batch size must be positive")
        for b in self._blocks:
            for name in ("velocity", "pressure"):
                t = getattr(b, name)
                if t.shape[0] == B:
                    continue
                if t.shape[0] != 1:
                    raise RuntimeError("setBatchSize repeats fields of batch size 1 only")
                setattr(b, name, t.expand(B, *t.shape[1:]).contiguous())
            if b.velocitySource is not None and b.velocitySource.shape[0] == 1 and B > 1:
                s = b.velocitySource
                b.velocitySource = s.expand(B, *s.shape[1:]).contiguous()
            if b.passiveScalar is not None and b.passiveScalar.shape[0] == 1 and B > 1:
                s = b.passiveScalar
                b.passiveScalar = s.expand(B, *s.shape[1:]).contiguous()
        self._batch = B
        self._invalidate()

    # --- PrepareSolve: flat buffers, metrics, topology records -----------------------------
    def PrepareSolve(self) -> None:
        _lib.require_cuda(self._device)
        _lib.load()
        d, B = self._dims, self._batch
        if not self._blocks:
            raise RuntimeError("Domain does not contain blocks.")
        opts = dict(dtype=self._dtype, device=self._device)
        # block offsets
        off = 0
        for b in self._blocks:
            b.globalOffset = off
            off += b.ncells()
        N = off
        self._N = N
        nb = len(self._blocks)
        bidx = {id(b): i for i, b in enumerate(self._blocks)}
        for b in self._blocks:
            for f, bd in enumerate(b._boundaries):
                if isinstance(bd, ConnectedBoundary) and id(bd.connectedBlock) not in bidx:
                    raise RuntimeError(f"block {b.name} is connected to a block of another domain")
        # flat state buffers; blocks become views
        u = torch.empty(B, d, N, **opts)
        p = torch.empty(B, N, **opts)
        for b in self._blocks:
            n = b.ncells()
            u[:, :, b.globalOffset:b.globalOffset + n] = b.velocity.reshape(B, d, n)
            p[:, b.globalOffset:b.globalOffset + n] = b.pressure.reshape(B, n)
        self._u_block = u
        self._p_block = p
        for b in self._blocks:
            n = b.ncells()
            spatial = list(reversed(b._sizes[:d]))
            b.velocity = u[:, :, b.globalOffset:b.globalOffset + n].view(B, d, *spatial)
            b.pressure = p[:, b.globalOffset:b.globalOffset + n].view(B, 1, *spatial)
        # passive scalar: one flat [B][channels][cells] buffer, blocks are views
        C = self._scalar_channels
        if C > 0:
            phi = torch.zeros(B, C, N, **opts)
            for b in self._blocks:
                n = b.ncells()
                spatial = list(reversed(b._sizes[:d]))
                if b.passiveScalar is not None:
                    phi[:, :, b.globalOffset:b.globalOffset + n] = b.passiveScalar.expand(B, C, *spatial).reshape(B, C, n)
                b.passiveScalar = phi[:, :, b.globalOffset:b.globalOffset + n].view(B, C, *spatial)
            self._phi_block = phi
            self.scalarRHS = torch.zeros(B * C * N, **opts)
            self.scalarResult = torch.zeros(B * C * N, **opts)
        else:
            self._phi_block = None
        # velocity sources: one per-cell buffer when any block has a per-cell source,
        # otherwise static [B, d] per block (all equal) or none
        self._rebuild_sources()
        # solve vectors (domain.cpp:517-561)
        self.velocityRHS = torch.zeros(B * d * N, **opts)
        self.velocityResult = torch.zeros(B * d * N, **opts)
        self.pressureRHS = torch.zeros(B * d * N, **opts)
        self.pressureRHSdiv = torch.zeros(B * N, **opts)
        self.pressureResult = torch.zeros(B * N, **opts)
        self.A = torch.zeros(B * N, **opts)
        S = 2 * d + 1
        self._C_st = torch.zeros(S, B * N, **opts)
        self._P_st = torch.zeros(S, B * N, **opts)
        # metrics (SoA [TS, N]) and fixed faces
        TS = 2 * d * d + 1
        met = torch.zeros(TS, N, **opts)
        stream = _lib.stream_ptr(self._device)
        dc = _lib.dtype_code(self._dtype)
        itemsize = torch.finfo(self._dtype).bits // 8
        for b in self._blocks:
            if b.vertexCoordinates is not None:
                nx, ny, nz = b._sizes
                _lib.call("phb_cell_metrics", d, dc, nx, ny, nz, b.vertexCoordinates.data_ptr(),
                          met.data_ptr() + b.globalOffset * itemsize, N, stream)
            else:
                _identity_metrics(met[:, b.globalOffset:b.globalOffset + b.ncells()], d)
        self._metrics = met
        fixed = []  # (block index, face, boundary)
        for i, b in enumerate(self._blocks):
            for f, bd in enumerate(b._boundaries):
                if isinstance(bd, FixedBoundary):
                    fixed.append((i, f, bd))
        self._fixed = fixed
        fcells = [bd.face_cells() for _, _, bd in fixed]
        toff = [sum(fcells[:k]) for k in range(len(fixed))]
        FM = max(1, sum(fcells))
        fmet = torch.zeros(TS, FM, **opts)
        for k, (i, f, bd) in enumerate(fixed):
            b = self._blocks[i]
            if b.vertexCoordinates is not None:
                nx, ny, nz = b._sizes
                _lib.call("phb_face_metrics", d, dc, nx, ny, nz, b.vertexCoordinates.data_ptr(), f,
                          fmet.data_ptr() + toff[k] * itemsize, FM, stream)
            else:
                _identity_metrics(fmet[:, toff[k]:toff[k] + fcells[k]], d)
        self._face_metrics = fmet
        self._fixed_toff = toff
        self._fixed_cells = fcells
        # fixed-face data buffers (velocity, potential values, masks) with boundary views
        self._pack_fixed()
        # records
        self._build_records()
        self._pack_scalar_faces()
        self._dt_dev = torch.ones(B, dtype=torch.float64, device=self._device)
        self._nu_dev = torch.zeros(B, dtype=torch.float64, device=self._device)
        self._upload_viscosity()
        self._snu_dev = torch.zeros(max(1, self._scalar_channels), dtype=torch.float64, device=self._device)
        self._upload_scalar_viscosity()
        self._scratch = torch.zeros(int(_lib.load().phb_scratch_doubles(ct.byref(self._desc_struct()), 3)) + 64,
                                    dtype=torch.float64, device=self._device)
        self._rms_out = torch.zeros(B, dtype=torch.float64, device=self._device)
        self._csr_cache = {}
        self._csr_pattern = None
        self._solvers = {}
        self._prepared = True
        self._version += 1
        self._desc = self._desc_struct()
        # CSR views of the domain matrices
        self.C = CSRmatrix(_domain=self, _which="C")
        self.P = CSRmatrix(_domain=self, _which="P")
        self._attach_csr_pattern()
        if self._epot_on:
            self.SetupEpotOnDomain(*self._epot_flags)

    def _upload_scalar_viscosity(self) -> None:
        v = self.passiveScalarViscosity
        if v is not None:
            self._snu_dev[: v.numel()].copy_(v)

    def _pack_scalar_faces(self) -> None:
        """Fixed-face passive-scalar data per fixed record (one per environment and face):
        values (boundary tensors become views of the packed buffer), offsets, static flags
        and per-channel types, the layout phb_scalar describes."""
        B, C = self._batch, self._scalar_channels
        nf = len(self._fixed)
        opts = dict(dtype=self._dtype, device=self._device)
        if C == 0:
            self._fscal = None
            return
        chunks, offs, stat, types = [], [0] * max(1, B * nf), [0] * max(1, B * nf), [0] * max(1, B * nf * C)
        off = 0
        for k, (i, f, bd) in enumerate(self._fixed):
            ps = bd._passiveScalar
            if ps is None:
                ps = torch.zeros(1, C, **opts)
                bd._passiveScalar = ps
                bd._passiveScalarTypes = [bd._velocityType]
            if ps.shape[0] not in (1, B):
                raise RuntimeError("boundary passive scalar batch size must be 1 or the domain batch size")
            static = ps.dim() == 2
            esize = C if static else C * self._fixed_cells[k]
            tv = bd._scalar_types()
            for e in range(B):
                r = e * nf + k
                offs[r] = off + (e if ps.shape[0] == B else 0) * esize
                stat[r] = 1 if static else 0
                for c in range(C):
                    types[r * C + c] = tv[c]
            chunks.append(ps.reshape(-1))
            off += ps.numel()
        self._fscal = torch.cat(chunks) if chunks else torch.zeros(1, **opts)
        self._fscal_off = torch.tensor(offs, dtype=torch.int64, device=self._device)
        self._fscal_static = torch.tensor(stat, dtype=torch.int8, device=self._device)
        self._fscal_types = torch.tensor(types, dtype=torch.int8, device=self._device)
        o = 0
        for k, (i, f, bd) in enumerate(self._fixed):
            ps = bd._passiveScalar
            bd._passiveScalar = self._fscal[o:o + ps.numel()].view(ps.shape)
            o += ps.numel()

    def _scalar_struct(self) -> _lib.PhbScalar:
        """The phb_scalar description of this domain's passive scalar."""
        if not self.hasPassiveScalar():
            raise RuntimeError("the domain has no passive scalar")
        s = _lib.PhbScalar()
        s.channels = self._scalar_channels
        v = self.passiveScalarViscosity
        s.nu_count = 0 if v is None else int(v.numel())
        s.nu = self._snu_dev.data_ptr()
        s.types = self._fscal_types.data_ptr()
        s.values = self._fscal.data_ptr()
        s.offsets = self._fscal_off.data_ptr()
        s.statics = self._fscal_static.data_ptr()
        return s

    def _upload_viscosity(self) -> None:
        v = self.viscosity
        vals = v.expand(self._batch) if v.numel() == 1 else v
        if vals.numel() != self._batch:
            raise RuntimeError("viscosity must have 1 or batch-size entries")
        self._nu_dev.copy_(vals.to(torch.float64))

    def _rebuild_sources(self) -> None:
        d, B, N = self._dims, self._batch, self._N
        opts = dict(dtype=self._dtype, device=self._device)
        srcs = [b.velocitySource for b in self._blocks]
        if all(s is None for s in srcs):
            self._src = None
            self._src_mode = 0
            return
        static = all(s is not None and s.dim() == 2 for s in srcs)
        if static and all(torch.equal(s, srcs[0]) for s in srcs[1:]):
            self._src = srcs[0].expand(B, d).contiguous()
            self._src_mode = 1
            for b in self._blocks:
                b.velocitySource = self._src
            return
        buf = torch.zeros(B, d, N, **opts)
        for b, s in zip(self._blocks, srcs):
            n = b.ncells()
            spatial = list(reversed(b._sizes[:d]))
            if s is not None:
                view = buf[:, :, b.globalOffset:b.globalOffset + n].view(B, d, *spatial)
                if s.dim() == 2:
                    view.copy_(s.view(s.shape[0], d, *([1] * d)).expand(B, d, *spatial))
                else:
                    view.copy_(s.expand(B, d, *spatial))
        self._src = buf
        self._src_mode = 2
        for b in self._blocks:
            n = b.ncells()
            spatial = list(reversed(b._sizes[:d]))
            b.velocitySource = buf[:, :, b.globalOffset:b.globalOffset + n].view(B, d, *spatial)

    def _set_block_source(self, blk: Block, s: torch.Tensor | None) -> None:
        if not self._prepared:
            blk.velocitySource = s
            return
        d, B = self._dims, self._batch
        if s is not None and s.shape[0] not in (1, B):
            raise RuntimeError("velocity source batch size must be 1 or the domain batch size")
        if s is None:
            blk.velocitySource = None
            self._rebuild_sources()
            return
        if self._src_mode == 2:
            spatial = list(reversed(blk._sizes[:d]))
            view = self._src[:, :, blk.globalOffset:blk.globalOffset + blk.ncells()].view(B, d, *spatial)
            if s.dim() == 2:
                view.copy_(s.view(s.shape[0], d, *([1] * d)).expand(B, d, *spatial))
            else:
                view.copy_(s.expand(B, d, *spatial))
            blk.velocitySource = view
            return
        if self._src_mode == 1 and s.dim() == 2 and len(self._blocks) == 1:
            self._src.copy_(s.expand(B, d))
            return
        blk.velocitySource = s
        self._rebuild_sources()

    def _pack_fixed(self) -> None:
        d, B = self._dims, self._batch
        opts = dict(dtype=self._dtype, device=self._device)
        vel_chunks, pot_chunks, mask_chunks = [], [], []
        vel_off, pot_off, mask_off = 0, 0, 0
        self._fixed_layout = []
        for k, (i, f, bd) in enumerate(self._fixed):
            fc = self._fixed_cells[k]
            v = bd._velocity
            if v.shape[0] not in (1, B):
                raise RuntimeError("boundary velocity batch size must be 1 or the domain batch size")
            per_env = v.shape[0]
            static = v.dim() == 2
            esize = d if static else d * fc
            vel_chunks.append(v.reshape(-1))
            venv = [vel_off + (e if per_env == B else 0) * esize for e in range(B)]
            vel_off += per_env * esize
            pv = bd._potentialValues
            if pv is not None:
                if pv.shape[0] not in (1, B):
                    raise RuntimeError("potential values batch size must be 1 or the domain batch size")
                pot_chunks.append(pv.reshape(-1))
                penv = [pot_off + (e if pv.shape[0] == B else 0) * fc for e in range(B)]
                pot_off += pv.shape[0] * fc
            else:
                penv = [-1] * B
            if bd._potentialTypes is not None:
                mask_chunks.append(bd._potentialTypes.reshape(-1))
                moff = mask_off
                mask_off += fc
            else:
                moff = -1
            self._fixed_layout.append((static, venv, penv, moff, per_env, pv.shape[0] if pv is not None else 0))
        self._fvel = torch.cat(vel_chunks) if vel_chunks else torch.zeros(1, **opts)
        self._fpot = torch.cat(pot_chunks) if pot_chunks else torch.zeros(1, **opts)
        self._fmask = torch.cat(mask_chunks) if mask_chunks else torch.zeros(1, dtype=torch.int8, device=self._device)
        # wall conductance per fixed record (one record per environment and face)
        self._fcw = torch.tensor([bd._cw for _ in range(B) for _, _, bd in self._fixed] or [0.0], **opts)
        # boundary tensors become views of the packed buffers
        vo, po, mo = 0, 0, 0
        for k, (i, f, bd) in enumerate(self._fixed):
            v = bd._velocity
            bd._velocity = self._fvel[vo:vo + v.numel()].view(v.shape)
            vo += v.numel()
            if bd._potentialValues is not None:
                pv = bd._potentialValues
                bd._potentialValues = self._fpot[po:po + pv.numel()].view(pv.shape)
                po += pv.numel()
            if bd._potentialTypes is not None:
                pt = bd._potentialTypes
                bd._potentialTypes = self._fmask[mo:mo + pt.numel()].view(pt.shape)
                mo += pt.numel()

    def _build_records(self) -> None:
        d, B, N = self._dims, self._batch, self._N
        nb = len(self._blocks)
        bidx = {id(b): i for i, b in enumerate(self._blocks)}
        fidx = {(i, f): k for k, (i, f, _) in enumerate(self._fixed)}
        nf = len(self._fixed)
        blocks = torch.zeros(B * nb, BREC, dtype=torch.int32)
        fixed = torch.zeros(max(1, B * nf), FREC, dtype=torch.int32)
        insts = torch.zeros(B, IREC, dtype=torch.int32)
        tiles = []
        for e in range(B):
            inst_tile0 = len(tiles)
            for i, b in enumerate(self._blocks):
                r = blocks[e * nb + i]
                nx, ny, nz = b._sizes
                r[0], r[1], r[2] = nx, ny, nz
                r[3] = e * N + b.globalOffset
                r[4] = b.globalOffset
                r[5] = e
                r[6] = e * N
                r[7] = N
                for f in range(6):
                    base = 8 + f * 6
                    if f >= 2 * d:
                        r[base] = 1  # unused axes: periodic of size 1 (never reached)
                        continue
                    bd = b._boundaries[f]
                    if isinstance(bd, FixedBoundary):
                        r[base] = 0
                        r[base + 5] = e * nf + fidx[(i, f)]
                    elif isinstance(bd, PeriodicBoundary):
                        r[base] = 1
                    else:
                        r[base] = 2
                        r[base + 1] = e * nb + bidx[id(bd.connectedBlock)]
                        ax = bd.axes + [0] * (3 - len(bd.axes))
                        r[base + 2], r[base + 3], r[base + 4] = ax[0], ax[1], ax[2]
                r[44] = len(tiles)
                n = b.ncells()
                for t0 in range(0, n, TILE):
                    tiles.append((e * nb + i, t0))
            ins = insts[e]
            ins[0] = e * N
            ins[1] = N
            ins[2] = inst_tile0
            ins[3] = len(tiles) - inst_tile0
            ins[4] = e * nb
            ins[5] = nb
            for k, (i, f, bd) in enumerate(self._fixed):
                static, venv, penv, moff, _, _ = self._fixed_layout[k]
                r = fixed[e * nf + k]
                r[0] = e * nb + i
                r[1] = f
                r[2] = 1 if static else 0
                r[3] = int(bd._velocityType)
                r[4] = int(bd._potentialType)
                r[5] = moff
                r[6] = penv[e]
                r[7] = venv[e]
                r[8] = self._fixed_cells[k]
                r[9] = self._fixed_toff[k]
        self._blocks_host, self._insts_host = blocks, insts
        self._blocks_dev = blocks.to(self._device)
        self._fixed_dev = fixed.to(self._device)
        self._insts_dev = insts.to(self._device)
        self._tiles_dev = torch.tensor(tiles, dtype=torch.int32).reshape(-1, 2).to(self._device)
        self._ntiles = len(tiles)
        self._nrec_fixed = B * nf

    def _desc_struct(self) -> _lib.PhbDomain:
        s = _lib.PhbDomain()
        s.dims = self._dims
        s.dtype = _lib.dtype_code(self._dtype)
        s.nblocks = self._batch * len(self._blocks)
        s.ninst = self._batch
        s.ntiles = self._ntiles
        s.nfixed = self._nrec_fixed
        s.ncells = self._batch * self._N
        s.metric_stride = self._N
        s.face_metric_stride = self._face_metrics.shape[1]
        s.blocks = self._blocks_dev.data_ptr()
        s.tiles = self._tiles_dev.data_ptr()
        s.fixed = self._fixed_dev.data_ptr()
        s.insts = self._insts_dev.data_ptr()
        s.metrics = self._metrics.data_ptr()
        s.face_metrics = self._face_metrics.data_ptr()
        s.fvel = self._fvel.data_ptr()
        s.fpot = self._fpot.data_ptr()
        s.fcw = self._fcw.data_ptr()
        s.fmask = self._fmask.data_ptr()
        s.dt = self._dt_dev.data_ptr()
        s.nu = self._nu_dev.data_ptr()
        s.scheme = int(self._advection_scheme)
        return s

    def desc(self) -> _lib.PhbDomain:
        """The device descriptor (phb_domain) of this domain; PrepareSolve() must have run."""
        if not self._prepared:
            raise RuntimeError("Domain is not initialized. Run domain.PrepareSolve() first.")
        return self._desc

    # --- differentiable simulations -------------------------------------------------------
    def _block_view(self, b: "Block", field: str) -> torch.Tensor | None:
        """The view of the flat state buffer that a block field normally is."""
        d, B = self._dims, self._batch
        spatial = list(reversed(b._sizes[:d]))
        o, n = b.globalOffset, b.ncells()
        if field == "velocity":
            return self._u_block[:, :, o:o + n].view(B, d, *spatial)
        if field == "pressure":
            return self._p_block[:, o:o + n].view(B, 1, *spatial)
        if field == "epot":
            e = getattr(self, "_epot_block", None)
            return None if e is None else e[:, o:o + n].view(B, 1, *spatial)
        if field == "velocitySource":
            return self._src[:, :, o:o + n].view(B, d, *spatial) if self._src_mode == 2 else b.velocitySource
        if field == "passiveScalar":
            ph = getattr(self, "_phi_block", None)
            return None if ph is None else ph[:, :, o:o + n].view(B, ph.shape[1], *spatial)
        raise KeyError(field)

    _AG_FIELDS = (("velocity", "_velocity_ag"), ("pressure", "_pressure_ag"), ("epot", "_epot_ag"),
                  ("velocitySource", "_source_ag"), ("passiveScalar", "_scalar_ag"))

    def _restore_block_views(self, b: "Block", fields=None) -> None:
        """Point fields that a differentiable step replaced by graph outputs back at the flat
        buffers (their values are equal) and forget their graph inputs."""
        if not self._prepared:
            return
        for field, ag in self._AG_FIELDS:
            if fields is not None and field not in fields:
                continue
            t = getattr(b, field)
            if t is not None and t.requires_grad:
                setattr(b, field, self._block_view(b, field))
            setattr(b, ag, None)

    def Detach(self) -> None:
        """Drop the autograd history of every field (reference Domain::Detach): the block fields
        become plain views of the domain's buffers again, with their current values."""
        for b in self._blocks:
            self._restore_block_views(b)
            for bd in b._boundaries:
                if isinstance(bd, FixedBoundary):
                    bd._velocity_ag = None
                    bd._scalar_ag = None
        self._viscosity_ag = None

    def UpdateDomainData(self) -> None:
        """Re-pack after structural changes (new boundaries, sizes or data shapes). Values
        written into the field and boundary views need no update."""
        if not self._prepared:
            self.PrepareSolve()
        self._version += 1

    UpdateDomain = UpdateDomainData

    def setTimeStep(self, timeStep) -> None:
        """1-element (shared) or batch-size host tensor (domain.cpp:370-400)."""
        t = timeStep if isinstance(timeStep, torch.Tensor) else torch.tensor([float(timeStep)])
        t = t.detach().reshape(-1)
        if t.numel() not in (1, self._batch):
            raise RuntimeError("time step must have 1 or batch-size entries")
        if t.device.type != "cpu":
            if self._prepared:
                self._dt_dev.copy_(t.to(torch.float64).expand(self._batch))
            self._timestep = None
            return
        vals = t.to(torch.float64).expand(self._batch).clone()
        # the device copy is issued only when the value changes, so a run with a constant
        # time step does not pay a host-to-device copy per kernel
        if self._prepared and (self._timestep is None or self._timestep.numel() != vals.numel()
                               or not torch.equal(self._timestep, vals)):
            self._dt_dev.copy_(vals)
        self._timestep = vals

    # --- epot ---------------------------------------------------------------------------
    def SetupEpotOnDomain(self, nonOrthoFlags: int = 0, useFaceTransform: bool = False) -> None:
        """Allocate the electric potential fields and build its matrix (mhd.py:511-514)."""
        if nonOrthoFlags or useFaceTransform:
            raise NotImplementedError("phipict_b200 assembles the orthogonal potential matrix without face transforms")
        self._epot_on = True
        self._epot_flags = (nonOrthoFlags, useFaceTransform)
        if not self._prepared:
            return
        d, B, N = self._dims, self._batch, self._N
        opts = dict(dtype=self._dtype, device=self._device)
        self._E_st = torch.zeros(2 * d + 1, B * N, **opts)
        # existing vectors are kept (domain.cpp:755-775): a second call rebuilds the matrix
        # only, and the potential of the last solve survives it
        if getattr(self, "epotRHS", None) is None or self.epotRHS.numel() != B * N:
            self.epotRHS = torch.zeros(B * N, **opts)
        had_result = getattr(self, "epotResult", None) is not None and self.epotResult.numel() == B * N
        if not had_result:
            self.epotResult = torch.zeros(B * N, **opts)
        all_blocks_had = all(b.epot is not None for b in self._blocks)
        self._attach_epot_blocks(copy_old=True)
        if not had_result and all_blocks_had:
            self.epotResult.copy_(self._epot_block.view(-1))
        _lib.call("phb_epot_matrix", ct.byref(self._desc), self._E_st.data_ptr(), None, _lib.stream_ptr(self._device))
        self._bump_matrix("E")
        self.Epot = CSRmatrix(_domain=self, _which="E")
        self.Epot.row, self.Epot.index = self._csr_row, self._csr_col
        self._csr_cache.pop("E", None)

    def hasEpot(self) -> bool:
        return self._epot_on and self._prepared

    def _attach_epot_blocks(self, copy_old: bool) -> None:
        """A fresh potential buffer [B, n] whose slices are the blocks' epot views (with the
        blocks' previous values when copy_old)."""
        d, B, N = self._dims, self._batch, self._N
        e = torch.zeros(B, N, dtype=self._dtype, device=self._device)
        for b in self._blocks:
            old = b.epot
            spatial = list(reversed(b._sizes[:d]))
            b.epot = e[:, b.globalOffset:b.globalOffset + b.ncells()].view(B, 1, *spatial)
            if copy_old and old is not None and old.shape == b.epot.shape:
                b.epot.copy_(old)
        self._epot_block = e

    def CreateEpotOnBlocks(self) -> None:
        """Domain::CreateEpotOnBlocks (domain.cpp:607-611): every block gets a new zero
        potential field; the domain's potential vectors and matrix stay as they are."""
        if getattr(self, "_epot_block", None) is None:
            self.SetupEpotOnDomain(*self._epot_flags)
            return
        self._attach_epot_blocks(copy_old=False)

    # --- CSR views ----------------------------------------------------------------------
    def _attach_csr_pattern(self) -> None:
        """Row pointers and columns of one instance (PrepareSolve, domain.cpp:426-561)."""
        B, N = self._batch, self._N
        stream = _lib.stream_ptr(self._device)
        rowsize = torch.zeros(B * N, dtype=torch.int32, device=self._device)
        _lib.call("phb_csr_row_sizes", ct.byref(self._desc), rowsize.data_ptr(), stream)
        row = torch.zeros(B * N + 1, dtype=torch.int32, device=self._device)
        row[1:] = torch.cumsum(rowsize, 0, dtype=torch.int32)
        nnz_all = int(row[-1])
        col = torch.zeros(max(1, nnz_all), dtype=torch.int32, device=self._device)
        perm = torch.zeros(max(1, nnz_all), dtype=torch.int32, device=self._device)
        _lib.call("phb_csr_pattern", ct.byref(self._desc), row.data_ptr(), col.data_ptr(), perm.data_ptr(), stream)
        nnz = nnz_all // B
        self._csr_perm = perm[:nnz_all]
        self._csr_row = row[: N + 1].contiguous()
        self._csr_col = col[:nnz].contiguous()
        self._csr_nnz = nnz
        for b in self._blocks:
            b.csrOffset = int(self._csr_row[b.globalOffset])
        for m in (self.C, self.P):
            m.row, m.index = self._csr_row, self._csr_col
        if getattr(self, "Epot", None) is not None:
            self.Epot.row, self.Epot.index = self._csr_row, self._csr_col

    def _stencil(self, which: str) -> torch.Tensor:
        return {"C": self._C_st, "P": self._P_st, "E": getattr(self, "_E_st", None)}[which]

    def _csr_values(self, which: str) -> torch.Tensor:
        st = self._stencil(which)
        nnz_all = self._csr_perm.numel()
        out = torch.empty(nnz_all, dtype=self._dtype, device=self._device)
        _lib.call("phb_csr_gather", _lib.dtype_code(self._dtype), nnz_all, self._csr_perm.data_ptr(), st.data_ptr(),
                  out.data_ptr(), _lib.stream_ptr(self._device))
        return out

    def _set_csr_values(self, which: str, v: torch.Tensor) -> None:
        st = self._stencil(which)
        st.view(-1).scatter_(0, self._csr_perm.long(), v.to(self._dtype).reshape(-1))
        self._bump_matrix(which)

    def _bump_matrix(self, which: str) -> int:
        """A new version of stencil ``which`` (its float32 copy and multigrid operators
        follow on their next use)."""
        ver = self.__dict__.setdefault("_mver", {})
        ver[which] = ver.get(which, 0) + 1
        return ver[which]

    def _matrix_version(self, which: str) -> int:
        return self.__dict__.get("_mver", {}).get(which, 0)

    # --- per-instance vector helpers ------------------------------------------------------
    def _subtract_mean(self, x: torch.Tensor, comps: int) -> None:
        """x[B][comps][cells] -= each environment's mean (subtract_env_mean)."""
        _lib.call("phb_subtract_mean", ct.byref(self.desc()), x.data_ptr(), comps, self._scratch.data_ptr(),
                  _lib.stream_ptr(self._device))

    def _rms(self, v: torch.Tensor, comps: int) -> torch.Tensor:
        """||v_env||_2 / sqrt(n_env) per environment, [B] float64 (device)."""
        _lib.call("phb_rms", ct.byref(self.desc()), v.data_ptr(), comps, self._scratch.data_ptr(),
                  self._rms_out.data_ptr(), _lib.stream_ptr(self._device))
        return self._rms_out

    def _ensure_cell_source(self) -> None:
        """Switch the velocity source to the per-cell buffer ([B][dims][cells]), keeping its
        values; the Lorentz force writes there."""
        if self._src_mode == 2:
            return
        d, B, N = self._dims, self._batch, self._N
        buf = torch.zeros(B, d, N, dtype=self._dtype, device=self._device)
        if self._src_mode == 1:
            buf.copy_(self._src.view(B, d, 1).expand(B, d, N))
        self._src = buf
        self._src_mode = 2
        for b in self._blocks:
            n = b.ncells()
            spatial = list(reversed(b._sizes[:d]))
            b.velocitySource = buf[:, :, b.globalOffset:b.globalOffset + n].view(B, d, *spatial)

    # --- boundary flux balance (domain.cpp:296-337) ---------------------------------------
    def _boundary_fluxes(self, bd: FixedBoundary) -> torch.Tensor:
        """Contravariant normal flux of each face cell: det_f * Minv_f[n] . u_b, [B, 1, *face]."""
        if not self._prepared:
            raise RuntimeError("Domain is not initialized.")
        k = [i for i, (_, _, b) in enumerate(self._fixed) if b is bd][0]
        d, B = self._dims, self._batch
        fc = self._fixed_cells[k]
        t0 = self._fixed_toff[k]
        ax = self._fixed[k][1] >> 1
        fm = self._face_metrics[:, t0:t0 + fc]
        minv = fm[d * d + ax * d: d * d + ax * d + d]  # [d, fc]
        det = fm[2 * d * d]
        v = bd.getVelocityVarying().reshape(bd._velocity.shape[0], d, fc)
        if bd.velocityType != BoundaryConditionType.DIRICHLET:
            v = torch.zeros_like(v)
        flux = det * (minv.unsqueeze(0) * v).sum(1)
        return flux.expand(B, fc).reshape(B, 1, *bd.face_shape())

    def GetBoundaryFluxBalance(self) -> torch.Tensor:
        """Net outflow of each batched environment, ``[B]``."""
        if not self._prepared:
            raise RuntimeError("Domain is not initialized.")
        total = torch.zeros(self._batch, dtype=torch.float64, device=self._device)
        for k, (i, f, bd) in enumerate(self._fixed):
            sign = 1.0 if (f & 1) else -1.0
            total += sign * self._boundary_fluxes(bd).reshape(self._batch, -1).sum(1).to(torch.float64)
        return total

    def CheckBoundaryFluxBalance(self, eps: float = 1e-5) -> bool:
        return bool(self.GetBoundaryFluxBalance().abs().max() <= eps)

    # --- misc ---------------------------------------------------------------------------
    def getMaxVelocity(self, withBounds: bool = True, computational: bool = False) -> torch.Tensor:
        """Largest velocity component magnitude over all environments (block.cpp:505-535)."""
        return self.getMaxVelocityPerEnv(withBounds, computational).max()

    def getMaxVelocityPerEnv(self, withBounds: bool = True, computational: bool = False) -> torch.Tensor:
        """Largest velocity component magnitude per environment, [B] (block.cpp:537-575):
        cell velocities and, withBounds, the fixed faces' velocities; computational: the
        velocities in computational space, Minv u per cell (grid/transform_vectors.cu:42-72),
        as the CFL bound of adaptive substeps uses them."""
        d = self._dims
        u = self._u_block
        if computational:
            u = _to_computational(u, self._metrics, d)
        m = u.abs().amax(dim=(1, 2))
        if withBounds:
            for k, (_, _, bd) in enumerate(self._fixed):
                v = bd._velocity
                if computational:
                    fc, to = self._fixed_cells[k], self._fixed_toff[k]
                    vv = v.reshape(v.shape[0], d, -1).expand(v.shape[0], d, fc) if v.dim() == 2 else v.reshape(v.shape[0], d, fc)
                    v = _to_computational(vv, self._face_metrics[:, to:to + fc], d)
                mb = v.abs().reshape(v.shape[0], -1).amax(1)
                m = torch.maximum(m, mb.expand_as(m))
        return m

    def __str__(self) -> str:
        return f"Domain({self.name}, dims={self._dims}, blocks={len(self._blocks)}, batch={self._batch})"


def _to_computational(u: torch.Tensor, metrics: torch.Tensor, d: int) -> torch.Tensor:
    """Minv u per cell: u [B, d, n] with metrics [2d^2+1, n] (Minv rows at d^2 + i d + j)."""
    rows = [sum(metrics[d * d + i * d + j] * u[:, j] for j in range(d)) for i in range(d)]
    return torch.stack(rows, dim=1)


def _identity_metrics(view: torch.Tensor, d: int) -> None:
    """M = Minv = I, det = 1: the metrics of a block without vertex coordinates, for which
    phiPICT's kernels take the untransformed branch (same values)."""
    view.zero_()
    for i in range(d):
        view[i * d + i] = 1
        view[d * d + i * d + i] = 1
    view[2 * d * d] = 1
