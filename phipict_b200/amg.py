"""Aggregation multigrid hierarchy of a domain: the preconditioner of the pressure and
potential CG solves (phiPICT's solvers/amg.py: ``hierarchy_for`` :450, ``galerkin_refresh``,
``amg_pcg_solve`` :1544, and the device V-cycle of solvers/krylov/krylov.cu:1248-1546).

phiPICT sets the hierarchy up on the host with pyamg (Ruge-Stueben or smoothed aggregation
on the CSR matrix) and keeps only the Galerkin products on the GPU. Here the whole
hierarchy follows the block structure, so nothing but a few hundred integers of level
records is built on the host, once per grid:

- level l+1 halves every block of level l along each axis longer than one cell (an odd
  size leaves one single-cell aggregate at the end), keeps the blocks' faces (periodic and
  connected ones included) and so stays a multi-block stencil grid;
- ``phb_amg_setup`` forms the coarse operators P^T A P (times ``coarse_scale``) on the
  device whenever the fine matrix changes, plus a dense FP64 generalised inverse of the
  coarsest operator of every instance;
- one V-cycle is damped Jacobi from zero, restriction, the coarse cycle, prolongation and
  a second damped Jacobi sweep: a symmetric preconditioner for CG.

Coarsening stops at ``coarse_cells`` cells per instance or when a connection that reverses
a tangential axis meets an odd size (its aggregates would not line up across the face).
Options of phiPICT's pyamg setup (``method``, ``strength``, ...) do not apply and are
recorded in :attr:`AmgHierarchy.ignored_options`.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch

from . import _lib

# omega 0.8 and the unscaled Galerkin product gave the fewest iterations on the graded
# 3D duct's pressure and potential systems (omega 1 is not a convergent Jacobi smoother,
# scaled coarse operators over-correct on the deeper levels)
# dense_cells / dense_bytes: the cycle below the first level with at most dense_cells cells per
# instance (and dense operators of at most dense_bytes for all instances) is applied as one
# dense operator, which saves two grid-wide phases per folded level; 0 folds nothing (the
# cycle runs down to the coarsest inverse)
DEFAULT_OPTIONS = {"omega": 0.8, "coarse_scale": 1.0, "coarse_cells": 128, "max_levels": _lib.AMG_MAX_LEVELS,
                   "dense_cells": 1024, "dense_bytes": 32 << 20}
MAX_COARSE_CELLS = 1024  # largest dense coarsest operator per instance (phb_amg::coarse_n)


def require_amg() -> None:
    """The multigrid entry points are part of the CUDA library (raises if it is missing)."""
    lib = _lib.load()
    for name in ("phb_amg_setup", "phb_amg_vcycle"):
        getattr(lib, name)


def coarsen_records(blocks: np.ndarray, insts: np.ndarray, dims: int):
    """Block, tile and instance records of the next coarser level, or None when the level
    cannot be coarsened (nothing left to halve, or an odd size across a connection that
    reverses a tangential axis)."""
    sizes = blocks[:, 0:3].astype(np.int64)
    new = sizes.copy()
    for a in range(dims):
        new[:, a] = np.where(sizes[:, a] >= 2, (sizes[:, a] + 1) // 2, sizes[:, a])
    if np.array_equal(new, sizes):
        return None
    for i in range(blocks.shape[0]):
        for f in range(2 * dims):
            base = 8 + 6 * f
            if blocks[i, base] != 2:
                continue
            bdim = f >> 1
            for t in range(1, dims):
                axis = (bdim + t) % dims
                if blocks[i, base + 2 + t] & 1 and sizes[i, axis] > 1 and sizes[i, axis] % 2:
                    return None
    out = blocks.copy()
    out[:, 0:3] = new
    tiles: list[tuple[int, int]] = []
    insts2 = np.zeros_like(insts)
    off = 0
    for e in range(insts.shape[0]):
        bs, bc = int(insts[e, 4]), int(insts[e, 5])
        t0, ioff = len(tiles), off
        for i in range(bs, bs + bc):
            n = int(np.prod(new[i]))
            out[i, 3] = off
            out[i, 4] = off - ioff
            out[i, 6] = ioff
            out[i, 44] = len(tiles)
            tiles.extend((i, t) for t in range(0, n, _lib.TILE))
            off += n
        out[bs:bs + bc, 7] = off - ioff
        insts2[e, :6] = (ioff, off - ioff, t0, len(tiles) - t0, bs, bc)
    return out, np.asarray(tiles, dtype=np.int32).reshape(-1, 2), insts2


class AmgHierarchy:
    """Level records and device buffers of one domain's hierarchy; :meth:`setup` fills the
    coarse operators from a float32 fine stencil, :meth:`vcycle` applies one cycle, and
    :meth:`struct` is the ``phb_amg`` that a solve takes."""

    def __init__(self, domain, **options):
        opts = dict(DEFAULT_OPTIONS)
        self.ignored_options = {k: v for k, v in options.items() if k not in DEFAULT_OPTIONS}
        opts.update({k: v for k, v in options.items() if k in DEFAULT_OPTIONS})
        self.options = opts
        self.domain = domain
        self.version = None  # the matrix version the operators were set up from
        # setups since the last full one, the coarse operators marked stale, the baseline
        # iterations of the solves after the last full setup, full setups so far
        self.refreshes, self.stale, self.baseline_iterations, self.full_setups = 0, False, None, 0
        dev = domain.getDevice()
        dims = domain.getSpatialDims()
        blocks, insts = domain._blocks_host.numpy(), domain._insts_host.numpy()
        records = [(blocks, None, insts)]
        max_levels = max(2, min(int(opts["max_levels"]), _lib.AMG_MAX_LEVELS))
        # at least one coarse level, then down to coarse_cells cells per instance
        while len(records) < max_levels and (len(records) == 1 or int(records[-1][2][:, 1].max()) > int(opts["coarse_cells"])):
            nxt = coarsen_records(records[-1][0], records[-1][2], dims)
            if nxt is None:
                break
            records.append((nxt[0], nxt[1], nxt[2]))
        if len(records) < 2:
            raise ValueError("the domain is too small (or shaped so) that no coarser level exists")
        cn = int(records[-1][2][:, 1].max())
        if cn > MAX_COARSE_CELLS:
            raise ValueError(f"the coarsest level keeps {cn} cells per instance (more than {MAX_COARSE_CELLS}); "
                             "raise max_levels or use plain CG")
        s = _lib.PhbAmg()
        s.nlevels = len(records)
        s.coarse_n = cn
        s.omega = float(opts["omega"])
        s.coarse_scale = float(opts["coarse_scale"])
        # the dense level T: the first small enough one below level 0 (else the coarsest)
        inst_max = [int(r[2][:, 1].max()) for r in records]
        ninst = insts.shape[0]
        T = len(records) - 1
        if int(opts["dense_cells"]) > 0:
            for t in range(1, len(records)):
                n_t = inst_max[t]
                if n_t <= min(int(opts["dense_cells"]), MAX_COARSE_CELLS) and ninst * n_t * n_t * 8 <= int(opts["dense_bytes"]):
                    T = t
                    break
        s.tail_level = T
        self.tail_level = T
        cn = inst_max[T]
        s.coarse_n = cn
        self.coarse_inv = torch.zeros(ninst * cn * cn, dtype=torch.float64, device=dev)
        s.coarse_inv = self.coarse_inv.data_ptr()
        self._keep: list[torch.Tensor] = []
        self.sizes: list[int] = []
        self.records = records  # host (blocks, tiles, insts) of every level
        self.level_A: list[torch.Tensor | None] = [None]  # coarse operators (level 0: the fine matrix)
        self.level_wdinv: list[torch.Tensor] = []  # omega / diagonal per level (0 on zero rows)
        fine = domain.desc()
        N0 = int(fine.ncells)
        self.z = torch.zeros(N0, dtype=torch.float32, device=dev)
        for l, (blk, tiles, ins) in enumerate(records):
            lv = s.levels[l]
            lv.inst_cells = inst_max[l]
            if l == 0:
                lv.dom = _lib.PhbDomain.from_buffer_copy(fine)
                lv.x = self.z.data_ptr()
                wd = torch.zeros(N0, dtype=torch.float32, device=dev)
                self._keep.append(wd)
                self.level_wdinv.append(wd)
                lv.wdinv = wd.data_ptr()
                self.sizes.append(N0)
                continue
            n = int(ins[:, 1].sum())
            self.sizes.append(n)
            bt = torch.from_numpy(np.ascontiguousarray(blk, dtype=np.int32)).to(dev)
            tt = torch.from_numpy(np.ascontiguousarray(tiles, dtype=np.int32)).to(dev)
            it = torch.from_numpy(np.ascontiguousarray(ins, dtype=np.int32)).to(dev)
            A = torch.zeros((2 * dims + 1) * n, dtype=torch.float32, device=dev)
            b = torch.zeros(n, dtype=torch.float32, device=dev)
            x = torch.zeros(n, dtype=torch.float32, device=dev)
            wd = torch.zeros(n, dtype=torch.float32, device=dev)
            self._keep += [bt, tt, it, A, b, x, wd]
            self.level_wdinv.append(wd)
            lv.wdinv = wd.data_ptr()
            self.level_A.append(A)
            d = _lib.PhbDomain()
            d.dims = dims
            d.dtype = _lib.PHB_F32
            d.nblocks = blk.shape[0]
            d.ninst = ninst
            d.ntiles = tiles.shape[0]
            d.nfixed = fine.nfixed
            d.ncells = n
            d.metric_stride = n
            d.blocks, d.tiles, d.insts, d.fixed = bt.data_ptr(), tt.data_ptr(), it.data_ptr(), fine.fixed
            lv.dom = d
            lv.A, lv.b, lv.x = A.data_ptr(), b.data_ptr(), x.data_ptr()
        self._struct = s
        self.coarse_n = cn
        wd = int(_lib.load().phb_amg_work_doubles(ct.byref(s)))
        self.work = torch.zeros(max(1, wd), dtype=torch.float64, device=dev)
        s.work = self.work.data_ptr()
        s.work_doubles = self.work.numel()
        self._fine_blocks = domain._blocks_dev
        self._A0 = None

    @property
    def nlevels(self) -> int:
        return self._struct.nlevels

    def struct(self) -> _lib.PhbAmg:
        return self._struct

    def address(self) -> int:
        return ct.addressof(self._struct)

    def setup(self, A32: torch.Tensor, version=None, coarse: bool = True) -> None:
        """Coarse operators of the float32 fine stencil ``A32`` [2d+1][ncells] (on the
        domain's current stream; the hierarchy keeps a reference to ``A32``). With
        ``coarse=False`` only the finest level follows ``A32`` (its smoother); the coarse
        operators of the last full setup are kept (phiPICT's galerkin_refresh(..., coarse=False),
        solvers/amg.py:749)."""
        if A32.dtype != torch.float32 or not A32.is_contiguous():
            raise TypeError("the multigrid hierarchy is built from a contiguous float32 stencil")
        if A32.numel() != (2 * self.domain.getSpatialDims() + 1) * self.sizes[0]:
            raise ValueError("stencil size does not match the domain")
        coarse = coarse or self._A0 is not A32 or self.version is None
        self._A0 = A32
        self.level_A[0] = A32
        self._struct.levels[0].A = A32.data_ptr()
        name = "phb_amg_setup" if coarse else "phb_amg_refresh_fine"
        _lib.call(name, ct.byref(self._struct), _lib.stream_ptr(self.domain.getDevice()))
        self.version = version
        if coarse:
            self.refreshes, self.stale, self.baseline_iterations = 0, False, None
            self.full_setups += 1
        self.refreshes += 1

    def note_iterations(self, iterations: int) -> None:
        """Iterations of a solve with this hierarchy (core/piso_simulation.py:2376-2392): the
        solves after a full setup set the baseline, and a later solve needing more than twice
        the baseline plus 5 marks the coarse operators stale, so that the next change of the
        matrix sets the whole hierarchy up again."""
        if self.baseline_iterations is None or self.refreshes <= 1:
            b = self.baseline_iterations
            self.baseline_iterations = iterations if b is None else max(b, iterations)
        elif iterations > 2 * self.baseline_iterations + 5:
            self.stale = True

    def vcycle(self, r: torch.Tensor, z: torch.Tensor | None = None) -> torch.Tensor:
        """z = one V-cycle applied to the float32 residual r."""
        if z is None:
            z = torch.empty_like(r)
        if r.dtype != torch.float32 or z.dtype != torch.float32 or r.numel() != self.sizes[0]:
            raise TypeError("the V-cycle takes float32 vectors of the domain's size")
        _lib.call("phb_amg_vcycle", ct.byref(self._struct), r.data_ptr(), z.data_ptr(),
                  _lib.stream_ptr(self.domain.getDevice()))
        return z

    def __repr__(self) -> str:
        return f"AmgHierarchy(levels={self.sizes}, coarse_n={self.coarse_n}, options={self.options})"


def hierarchy_for(domain, which: str, A32: torch.Tensor, version, cache: dict, options: dict | None = None,
                  coarse_refresh_interval: int = 1) -> AmgHierarchy:
    """The cached hierarchy of matrix ``which`` of ``domain``, rebuilt for a new grid and
    set up again when the matrix version changed (phiPICT's fingerprint refresh,
    core/piso_simulation.py:2222-2300). ``options["coarse_refresh_interval"]`` (else the
    argument) n > 1: the whole hierarchy is set up on every n-th change of the matrix and
    when its coarse operators were marked stale; in between only the finest level follows
    (core/piso_simulation.py:1042-1046,2268-2297)."""
    options = dict(options or {})
    interval = int(options.pop("coarse_refresh_interval", coarse_refresh_interval))
    h = cache.get(which)
    # PrepareSolve re-creates the domain's records, which level 0 points at
    if h is None or h.domain is not domain or h._fine_blocks is not domain._blocks_dev:
        h = AmgHierarchy(domain, **options)
        cache[which] = h
    if h.version != version or h._A0 is not A32:
        coarse = interval <= 1 or h.refreshes % interval == 0 or h.stale
        h.setup(A32, version, coarse=coarse)
    return h


def auto_rows() -> int:
    """Unknowns from which ``pressure_use_amg=None`` turns the preconditioner on
    (PRESSURE_AMG_AUTO_MIN_ROWS, core/piso_simulation.py:1118)."""
    return 200_000


def levels_of(domain, coarse_cells: int = DEFAULT_OPTIONS["coarse_cells"]) -> list[int]:
    """Cells per level of the hierarchy the domain would get (no device work)."""
    dims = domain.getSpatialDims()
    blocks, insts = domain._blocks_host.numpy(), domain._insts_host.numpy()
    out = [int(insts[:, 1].sum())]
    while len(out) < _lib.AMG_MAX_LEVELS and int(insts[:, 1].max()) > coarse_cells:
        nxt = coarsen_records(blocks, insts, dims)
        if nxt is None:
            break
        blocks, _, insts = nxt
        out.append(int(insts[:, 1].sum()))
    return out


__all__ = ["AmgHierarchy", "DEFAULT_OPTIONS", "coarsen_records", "hierarchy_for", "levels_of", "require_amg",
           "auto_rows"]
