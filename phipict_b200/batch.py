"""Heterogeneous instance batches: several prepared domains with different grids, viscosities
and time steps advanced together, every kernel and solve one launch over all of them.

phiPICT batches only copies of one domain (one grid, one Stuart number,
docs/source/batching.rst:4-6, simulation/mhd.py:478-479). The device records here already
describe every instance separately (its blocks, tiles, cell offset and size), so a
:class:`DomainBatch` packs the records, metrics and boundary data of its member domains into
one descriptor and owns one set of flat field buffers (``[inst][comp][cells_inst]``
concatenated). ``Simulation`` and ``MHDSimulation`` run on it unchanged; per-instance Stuart
numbers and fields go in as ``(B,)`` / ``(B, 3)`` tensors, per-instance viscosities come from
the members and per-instance time steps through ``setTimeStep``.

The members keep their own buffers: :meth:`DomainBatch.gather` copies their state in,
:meth:`DomainBatch.scatter` copies the batch state back (the serving loop does both when the
membership changes). Boundary data are packed at construction: change a member's boundaries,
then build a new batch.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch

from . import _lib
from .domain import Domain, FixedBoundary

_FIELDS_SCALAR = ("pressureResult", "pressureRHSdiv", "A")
_FIELDS_VECTOR = ("velocityRHS", "velocityResult", "pressureRHS")


class DomainBatch:
    """Prepared single-environment domains of the same dimensionality, dtype and device,
    packed as the instances of one device descriptor."""

    def __init__(self, domains: list[Domain]):
        if not domains:
            raise ValueError("DomainBatch needs at least one domain")
        d0 = domains[0]
        for m in domains:
            if not m.IsInitialized():
                m.PrepareSolve()
            if m.getBatchSize() != 1:
                raise NotImplementedError("DomainBatch packs single-environment domains")
            if (m.getSpatialDims(), m.getDtype(), m.getDevice()) != (d0.getSpatialDims(), d0.getDtype(), d0.getDevice()):
                raise ValueError("the domains of a batch must share dimensionality, dtype and device")
        self.members = list(domains)
        self._dims = d0.getSpatialDims()
        self._dtype = d0.getDtype()
        self._device = d0.getDevice()
        self._batch = len(domains)
        self._version = 1
        self._prepared = True
        self._mixed = False
        self._epot_on = False
        self._pack()
        self.gather()

    # --- packing ------------------------------------------------------------------------
    def _pack(self) -> None:
        d, dev = self._dims, self._device
        opts = dict(dtype=self._dtype, device=dev)
        blocks, tiles, fixed, insts = [], [], [], []
        metrics, fmetrics, fvel, fpot, fmask, fcw = [], [], [], [], [], []
        self._cell_off, self._ncells = [], []
        cell = blk = tile = fix = fm = vel = pot = mask = 0
        for e, m in enumerate(self.members):
            N = m._N
            b = m._blocks_host.clone().numpy()
            nb = b.shape[0]
            nf = m._nrec_fixed
            t = m._tiles_dev.cpu().numpy().copy()
            f = m._fixed_dev.cpu().numpy()[:nf].copy()
            b[:, 3] += cell
            b[:, 4] += cell
            b[:, 5] = e
            b[:, 6] = cell
            b[:, 7] = N
            for face in range(6):
                base = 8 + 6 * face
                conn = b[:, base] == 2
                b[conn, base + 1] += blk
                fixd = (b[:, base] == 0) & (face < 2 * d)
                b[fixd, base + 5] += fix
            b[:, 44] += tile
            t[:, 0] += blk
            if nf:
                f[:, 0] += blk
                f[:, 5] = np.where(f[:, 5] >= 0, f[:, 5] + mask, f[:, 5])
                f[:, 6] = np.where(f[:, 6] >= 0, f[:, 6] + pot, f[:, 6])
                f[:, 7] += vel
                f[:, 9] += fm
            blocks.append(b)
            tiles.append(t)
            fixed.append(f)
            rec = np.zeros(_lib.IREC, dtype=np.int32)
            rec[:6] = (cell, N, tile, t.shape[0], blk, nb)
            insts.append(rec)
            metrics.append(m._metrics[:, :N])
            fmetrics.append(m._face_metrics)
            fvel.append(m._fvel)
            fpot.append(m._fpot)
            fmask.append(m._fmask)
            fcw.append(m._fcw[:nf] if nf else m._fcw[:0])
            self._cell_off.append(cell)
            self._ncells.append(N)
            cell += N
            blk += nb
            tile += t.shape[0]
            fix += nf
            fm += m._face_metrics.shape[1]
            vel += m._fvel.numel()
            pot += m._fpot.numel()
            mask += m._fmask.numel()
        self._total = cell
        self._blocks_host = torch.from_numpy(np.concatenate(blocks).astype(np.int32))
        self._insts_host = torch.from_numpy(np.stack(insts).astype(np.int32))
        self._blocks_dev = self._blocks_host.to(dev)
        self._insts_dev = self._insts_host.to(dev)
        self._tiles_dev = torch.from_numpy(np.concatenate(tiles).astype(np.int32)).to(dev)
        fx = np.concatenate(fixed) if fix else np.zeros((1, _lib.FREC), dtype=np.int32)
        self._fixed_dev = torch.from_numpy(fx.astype(np.int32)).to(dev)
        self._nrec_fixed = fix
        self._ntiles = tile
        self._metrics = torch.cat(metrics, dim=1).contiguous()
        self._face_metrics = torch.cat(fmetrics, dim=1).contiguous()
        self._fvel = torch.cat([v.reshape(-1) for v in fvel]).contiguous()
        self._fpot = torch.cat([v.reshape(-1) for v in fpot]).contiguous()
        self._fmask = torch.cat([v.reshape(-1) for v in fmask]).contiguous()
        self._fcw = torch.cat(fcw).contiguous() if fix else torch.zeros(1, **opts)
        B, T = self._batch, self._total
        self._dt_dev = torch.cat([m._dt_dev for m in self.members]).contiguous()
        self._nu_dev = torch.cat([m._nu_dev for m in self.members]).contiguous()
        self._timestep = None
        self._u_block = torch.zeros(d * T, **opts)
        self._p_block = torch.zeros(T, **opts)
        for name in _FIELDS_VECTOR:
            setattr(self, name, torch.zeros(d * T, **opts))
        for name in _FIELDS_SCALAR:
            setattr(self, name, torch.zeros(T, **opts))
        S = 2 * d + 1
        self._C_st = torch.zeros(S, T, **opts)
        self._P_st = torch.zeros(S, T, **opts)
        self._src, self._src_mode = None, 0
        self._desc = self._desc_struct()
        self._scratch = torch.zeros(int(_lib.load().phb_scratch_doubles(ct.byref(self._desc), 3)) + 64,
                                    dtype=torch.float64, device=dev)
        self._rms_out = torch.zeros(B, dtype=torch.float64, device=dev)
        self._solvers = {}

    def _desc_struct(self) -> _lib.PhbDomain:
        s = _lib.PhbDomain()
        s.dims = self._dims
        s.dtype = _lib.dtype_code(self._dtype)
        s.nblocks = int(self._blocks_host.shape[0])
        s.ninst = self._batch
        s.ntiles = self._ntiles
        s.nfixed = self._nrec_fixed
        s.ncells = self._total
        s.metric_stride = self._total
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
        schemes = {int(m.getAdvectionScheme()) for m in self.members}
        if len(schemes) != 1:
            raise NotImplementedError("the instances of a DomainBatch must share the advection scheme")
        s.scheme = schemes.pop()
        return s

    # --- state in and out -------------------------------------------------------------
    def _vec(self, e: int, comps: int) -> slice:
        c, n = self._cell_off[e], self._ncells[e]
        return slice(comps * c, comps * (c + n))

    def gather(self) -> None:
        """Copy the members' state (velocity, pressure, potential, solver warm starts and
        velocity sources) into the batch buffers."""
        d = self._dims
        cell_src = any(m._src_mode != 0 for m in self.members)
        if cell_src:
            self._ensure_cell_source()
        for e, m in enumerate(self.members):
            self._u_block[self._vec(e, d)].copy_(m._u_block.reshape(-1))
            self._p_block[self._vec(e, 1)].copy_(m._p_block.reshape(-1))
            self.velocityResult[self._vec(e, d)].copy_(m.velocityResult)
            self.pressureResult[self._vec(e, 1)].copy_(m.pressureResult)
            if self._epot_on and getattr(m, "epotResult", None) is not None:
                self.epotResult[self._vec(e, 1)].copy_(m.epotResult)
                self._epot_block[self._vec(e, 1)].copy_(m._epot_block.reshape(-1))
            if cell_src:
                dst = self._src[self._vec(e, d)].view(d, -1)
                if m._src_mode == 1:
                    dst.copy_(m._src.reshape(d, 1).expand(d, m._N))
                elif m._src_mode == 2:
                    dst.copy_(m._src.reshape(d, -1))
                else:
                    dst.zero_()

    def scatter(self) -> None:
        """Copy the batch state back into the members."""
        d = self._dims
        for e, m in enumerate(self.members):
            m._u_block.view(-1).copy_(self._u_block[self._vec(e, d)])
            m._p_block.view(-1).copy_(self._p_block[self._vec(e, 1)])
            m.velocityResult.copy_(self.velocityResult[self._vec(e, d)])
            m.pressureResult.copy_(self.pressureResult[self._vec(e, 1)])
            if self._epot_on and getattr(m, "epotResult", None) is not None:
                m.epotResult.copy_(self.epotResult[self._vec(e, 1)])
                m._epot_block.view(-1).copy_(self._epot_block[self._vec(e, 1)])
            if self._src_mode == 2:
                m._ensure_cell_source()
                m._src.view(-1).copy_(self._src[self._vec(e, d)])

    def instance_slice(self, e: int, comps: int = 1) -> slice:
        """Range of instance e in a flat field with `comps` components per cell."""
        return self._vec(e, comps)

    # --- the Domain interface the step uses ---------------------------------------------
    def desc(self) -> _lib.PhbDomain:
        return self._desc

    def getDevice(self) -> torch.device:
        return self._device

    def getDtype(self) -> torch.dtype:
        return self._dtype

    def getSpatialDims(self) -> int:
        return self._dims

    def getBatchSize(self) -> int:
        return self._batch

    def numCells(self) -> int:
        return self._total

    def getTotalSize(self) -> int:
        raise NotImplementedError("the instances of a DomainBatch differ in size: use numCells() or the members")

    def IsInitialized(self) -> bool:
        return True

    def hasNonOrthogonalMetrics(self) -> bool:
        return any(m.hasNonOrthogonalMetrics() for m in self.members)

    def hasPassiveScalar(self) -> bool:
        """Passive scalars are not transported in a batch: the members' scalar fields stay as
        they are (a batched step advances velocity, pressure and potential)."""
        return False

    def getPassiveScalarChannels(self) -> int:
        return 0

    def hasBlockViscosity(self) -> bool:
        return False

    def PrepareSolve(self) -> None:
        pass

    def getBlocks(self):
        return [b for m in self.members for b in m.getBlocks()]

    def getNumBlocks(self) -> int:
        return len(self.getBlocks())

    def GetBoundaryFluxBalance(self) -> torch.Tensor:
        return torch.cat([m.GetBoundaryFluxBalance().reshape(-1) for m in self.members])

    def getMaxVelocity(self, withBounds: bool = True, computational: bool = False) -> torch.Tensor:
        return torch.stack([m.getMaxVelocity(withBounds, computational) for m in self.members]).max()

    def setTimeStep(self, timeStep) -> None:
        t = timeStep if isinstance(timeStep, torch.Tensor) else torch.tensor([float(timeStep)])
        t = t.detach().reshape(-1).to("cpu", torch.float64)
        if t.numel() not in (1, self._batch):
            raise RuntimeError("time step must have 1 or one entry per instance")
        vals = t.expand(self._batch).clone()
        if self._timestep is None or not torch.equal(self._timestep, vals):
            self._dt_dev.copy_(vals)
        self._timestep = vals

    def _stencil(self, which: str) -> torch.Tensor:
        return {"C": self._C_st, "P": self._P_st, "E": getattr(self, "_E_st", None)}[which]

    def _bump_matrix(self, which: str) -> int:
        ver = self.__dict__.setdefault("_mver", {})
        ver[which] = ver.get(which, 0) + 1
        return ver[which]

    def _matrix_version(self, which: str) -> int:
        return self.__dict__.get("_mver", {}).get(which, 0)

    def _subtract_mean(self, x: torch.Tensor, comps: int) -> None:
        _lib.call("phb_subtract_mean", ct.byref(self._desc), x.data_ptr(), comps, self._scratch.data_ptr(),
                  _lib.stream_ptr(self._device))

    def _rms(self, v: torch.Tensor, comps: int) -> torch.Tensor:
        _lib.call("phb_rms", ct.byref(self._desc), v.data_ptr(), comps, self._scratch.data_ptr(),
                  self._rms_out.data_ptr(), _lib.stream_ptr(self._device))
        return self._rms_out

    def _ensure_cell_source(self) -> None:
        if self._src_mode == 2:
            return
        self._src = torch.zeros(self._dims * self._total, dtype=self._dtype, device=self._device)
        self._src_mode = 2

    def SetupEpotOnDomain(self, nonOrthoFlags: int = 0, useFaceTransform: bool = False) -> None:
        if nonOrthoFlags or useFaceTransform:
            raise NotImplementedError("phipict_b200 assembles the orthogonal potential matrix without face transforms")
        opts = dict(dtype=self._dtype, device=self._device)
        first = not self._epot_on
        self._epot_on = True
        for m in self.members:  # so that scatter() has somewhere to put the potential
            if getattr(m, "epotResult", None) is None:
                m.SetupEpotOnDomain(nonOrthoFlags, useFaceTransform)
        self._E_st = torch.zeros(2 * self._dims + 1, self._total, **opts)
        if first:
            self.epotRHS = torch.zeros(self._total, **opts)
            self.epotResult = torch.zeros(self._total, **opts)
            self._epot_block = torch.zeros(self._total, **opts)
            for e, m in enumerate(self.members):
                if getattr(m, "epotResult", None) is not None:
                    self.epotResult[self._vec(e, 1)].copy_(m.epotResult)
                    self._epot_block[self._vec(e, 1)].copy_(m._epot_block.reshape(-1))
        _lib.call("phb_epot_matrix", ct.byref(self._desc), self._E_st.data_ptr(), None, _lib.stream_ptr(self._device))
        self._bump_matrix("E")

    def hasEpot(self) -> bool:
        return self._epot_on

    def __repr__(self) -> str:
        return f"DomainBatch(instances={self._batch}, cells={self._ncells})"


def potential_anchoring(batch: DomainBatch) -> bool:
    """Whether the potential systems of the batch have a Dirichlet anchor; the instances of one
    batch must agree (the mean projection is applied to all or none of them)."""
    flags = {any(bd.hasPotentialDirichlet() for blk in m.getBlocks() for _, bd in blk.getFixedBoundaries())
             for m in batch.members}
    if len(flags) != 1:
        raise NotImplementedError("the instances of a batch must all have, or all lack, Dirichlet potential faces")
    return flags.pop()


__all__ = ["DomainBatch", "FixedBoundary", "potential_anchoring"]
