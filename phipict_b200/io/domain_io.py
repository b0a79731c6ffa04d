"""Domain checkpoints as a ``<name>.json`` + ``<name>.npz`` pair, in phiPICT's file layout
(src/phipict/io/domain_io.py, format version 2), so that a domain saved by either
implementation loads in the other.

The JSON holds the structure (name, dimensionality, passive-scalar channels, blocks and their
six face descriptions) and names every tensor by a string index into the NPZ; ``data_info``
records each tensor's shape, dtype and device. A tensor shared by several objects (same
storage, shape and strides) is stored once. Both files carry the same random ``save_id`` and
are each written atomically (temporary file, fsync, rename; tensors first, JSON last), so a
pair left by an interrupted save is refused on load instead of mixing two saves. Files of
format version 1 (no version, no save id) still load.
"""
from __future__ import annotations

import json
import os
import tempfile
import uuid
from pathlib import Path
from typing import Any

import numpy as np
import torch

from ..domain import (BoundaryConditionType, ConnectedBoundary, Domain, FixedBoundary, PeriodicBoundary,
                      PotentialBC)

FORMAT_VERSION = 2
_SUFFIXES = (".json", ".npz")
_SAVE_ID = "save_id"
_FACES = ("-x", "+x", "-y", "+y", "-z", "+z")
_DTYPES = {torch.float32: "float32", torch.float64: "float64", torch.int8: "int8"}


def _dtype_name(dtype: torch.dtype) -> str:
    if dtype not in _DTYPES:
        raise TypeError(f"Unsupported tensor dtype {dtype}.")
    return _DTYPES[dtype]


def _bc_name(t) -> str:
    return BoundaryConditionType(t).name


def _pair(path: Path) -> tuple[Path, Path]:
    """The .json and .npz paths of a pair; a .json/.npz extension on `path` is dropped (and a
    dot inside the name is kept)."""
    if not isinstance(path, Path):
        raise TypeError(f"path must be a pathlib.Path, got {type(path).__name__}: {path!r}.")
    if path.suffix in _SUFFIXES:
        path = path.with_suffix("")
    return path.with_name(path.name + ".json"), path.with_name(path.name + ".npz")


def _atomic_write(target: Path, write) -> None:
    fd, tmp = tempfile.mkstemp(dir=target.parent, prefix=f".{target.name}.", suffix=".tmp")
    try:
        with os.fdopen(fd, "wb") as f:
            write(f)
            f.flush()
            os.fsync(f.fileno())
        os.replace(tmp, target)
    except BaseException:
        Path(tmp).unlink(missing_ok=True)
        raise


def save_domain(domain: Domain, path: Path) -> None:
    """Save `domain` to ``<path>.json`` and ``<path>.npz`` (parent directories created)."""
    json_path, npz_path = _pair(path)
    data: list[torch.Tensor] = []
    index: dict[tuple, int] = {}

    def add(t: torch.Tensor, into: dict, name: str) -> None:
        key = (t.device, t.dtype, t.data_ptr(), tuple(t.shape), tuple(t.stride()))
        if key not in index:
            index[key] = len(data)
            data.append(t)
        into[name] = str(index[key])

    out: dict[str, Any] = {"format_version": FORMAT_VERSION, "name": domain.name,
                           "spatialDims": domain.getSpatialDims()}
    # the viscosity in the domain's dtype: its saved dtype is the default dtype on load
    add(domain.viscosity.to(domain.getDtype()), out, "viscosity")
    out["passiveScalarChannels"] = domain.getPassiveScalarChannels()
    if domain.hasPassiveScalarViscosity():
        add(domain.passiveScalarViscosity.to(domain.getDtype()), out, "passiveScalarViscosity")
    blocks = domain.getBlocks()
    out["blocks"] = []
    for blk in blocks:
        bd: dict[str, Any] = {"name": blk.name}
        add(blk.velocity, bd, "velocity")
        add(blk.pressure, bd, "pressure")
        if blk.hasPassiveScalar() and blk.passiveScalar is not None:
            add(blk.passiveScalar, bd, "scalar")
        if blk.hasEpot():
            add(blk.epot, bd, "epot")
        if blk.hasVelocitySource():
            add(blk.velocitySource, bd, "velocitySource")
        if blk.hasVertexCoordinates():
            add(blk.vertexCoordinates, bd, "vertexCoordinates")
        bd["boundaries"] = []
        for f in range(2 * blk.getSpatialDims()):
            b = blk.getBoundary(f)
            fd: dict[str, Any] = {}
            if isinstance(b, FixedBoundary):
                fd["type"] = "FIXED"
                fd["velocityType"] = _bc_name(b.velocityType)
                add(b.velocity, fd, "velocity")
                if b.hasPassiveScalar():
                    fd["passiveScalarType"] = [_bc_name(t) for t in b.passiveScalarTypes]
                    add(b.passiveScalar, fd, "scalar")
                if b.hasPotentialTypes():
                    add(b.getPotentialTypes(), fd, "potentialTypes")
                if b.hasPotentialTypes() or b.getPotentialBC() != PotentialBC.INSULATING:
                    fd["potentialBC"] = PotentialBC(b.getPotentialBC()).name
                if b.hasPotentialThinWall():
                    fd["potentialCw"] = b.getPotentialCw()
                if b.hasPotentialValues():
                    add(b.getPotentialValues(), fd, "potentialValues")
            elif isinstance(b, ConnectedBoundary):
                fd["type"] = "CONNECTED"
                fd["connectedBlock"] = blocks.index(b.getConnectedBlock())
                fd["axes"] = list(b.axes)
            elif isinstance(b, PeriodicBoundary):
                fd["type"] = "PERIODIC"
            else:
                raise TypeError(f"Block '{blk.name}' face {_FACES[f]}: unknown boundary type {type(b).__name__}.")
            bd["boundaries"].append(fd)
        out["blocks"].append(bd)
    save_id = uuid.uuid4().hex
    out[_SAVE_ID] = save_id
    out["data_info"] = {str(i): {"shape": list(t.shape), "dtype": _dtype_name(t.dtype), "device": t.device.type}
                        for i, t in enumerate(data)}
    arrays = {str(i): t.detach().cpu().numpy() for i, t in enumerate(data)}
    arrays[_SAVE_ID] = np.array(save_id)
    json_path.parent.mkdir(parents=True, exist_ok=True)
    _atomic_write(npz_path, lambda f: np.savez_compressed(f, **arrays))
    _atomic_write(json_path, lambda f: f.write(json.dumps(out, indent=1).encode()))


def _read(path: Path) -> tuple[dict, dict[str, np.ndarray]]:
    json_path, npz_path = _pair(path)
    missing = [str(p) for p in (json_path, npz_path) if not p.is_file()]
    if missing:
        raise FileNotFoundError(f"Saved domain incomplete, missing: {', '.join(missing)}.")
    try:
        desc = json.loads(json_path.read_text())
    except json.JSONDecodeError as e:
        raise ValueError(f"{json_path} is not valid JSON: {e}.") from e
    version = int(desc.get("format_version", 1))
    if version > FORMAT_VERSION:
        raise ValueError(f"{json_path} has format version {version}; this reader reads up to {FORMAT_VERSION}.")
    for key in ("spatialDims", "name", "blocks", "data_info", "viscosity"):
        if key not in desc:
            raise ValueError(f"{json_path} is missing the '{key}' entry.")
    info = desc["data_info"]
    try:
        with np.load(npz_path) as npz:
            if _SAVE_ID in desc:
                npz_id = str(npz[_SAVE_ID]) if _SAVE_ID in npz else None
                if npz_id != desc[_SAVE_ID]:
                    raise ValueError(f"{json_path} and {npz_path} belong to different saves (interrupted save?).")
            absent = [k for k in info if k not in npz]
            if absent:
                raise ValueError(f"{npz_path} lacks tensors {absent} listed in {json_path}.")
            arrays = {k: npz[k] for k in info}
    except (OSError, EOFError) as e:
        raise ValueError(f"{npz_path} is not a readable .npz file: {e}.") from e
    for key, i in info.items():
        if "shape" in i and list(arrays[key].shape) != list(i["shape"]):
            raise ValueError(f"Tensor {key} in {npz_path} has shape {list(arrays[key].shape)}, "
                             f"{json_path} expects {i['shape']}.")
    return desc, arrays


def load_domain(path: Path, dtype: torch.dtype | None = None, device: torch.device | str | None = None,
                with_scalar: bool = True) -> Domain:
    """Load a domain saved by :func:`save_domain` (or by phiPICT). dtype / device default to
    the saved ones; host tensors (the domain viscosity) stay on the host. Call
    ``PrepareSolve()`` before simulating."""
    desc, arrays = _read(path)
    info = desc["data_info"]
    if dtype is None:
        dtype = getattr(torch, info[desc["viscosity"]].get("dtype", "float32"))
    if device is None:
        bl = desc["blocks"]
        vk = bl[0].get("velocity") if bl else None
        device = info[vk].get("device", "cuda") if vk else "cuda"
    target = torch.device(device)
    tensors: dict[str, torch.Tensor] = {}
    for key, arr in arrays.items():
        t = torch.from_numpy(np.ascontiguousarray(arr))
        host = info[key].get("device", "cuda") == "cpu"
        tensors[key] = t.to(device="cpu" if host else target, dtype=dtype if t.is_floating_point() else None)

    def get(d: dict, name: str):
        return tensors[d[name]] if name in d else None

    dom = Domain(desc["spatialDims"], get(desc, "viscosity"), desc["name"], dtype=dtype, device=target,
                 passiveScalarChannels=desc.get("passiveScalarChannels", 1) if with_scalar else 0,
                 scalarViscosity=get(desc, "passiveScalarViscosity") if with_scalar else None)
    nb = 2 * desc["spatialDims"]
    for bd in desc["blocks"]:
        if len(bd.get("boundaries", [])) != nb:
            raise ValueError(f"Block '{bd.get('name')}' lists {len(bd.get('boundaries', []))} boundaries, expected {nb}.")
        if "viscosity" in bd:
            raise NotImplementedError(f"Block '{bd['name']}': per-block viscosity is not supported")
        if "vertexCoordinates" not in bd and "transform" in bd:
            raise NotImplementedError(f"Block '{bd['name']}': blocks given by transforms instead of vertex coordinates")
        blk = dom.CreateBlock(get(bd, "velocity"), get(bd, "pressure"), get(bd, "scalar") if with_scalar else None,
                              vertexCoordinates=get(bd, "vertexCoordinates"), name=bd["name"])
        if "velocitySource" in bd:
            blk.setVelocitySource(get(bd, "velocitySource"))
        if "epot" in bd:
            blk.setEpot(get(bd, "epot"))
    blocks = dom.getBlocks()
    for bd, blk in zip(desc["blocks"], blocks, strict=True):
        for f, fd in enumerate(bd["boundaries"]):
            t = fd["type"]
            if t == "FIXED":
                _load_fixed(blk, f, fd, get, with_scalar)
            elif t == "CONNECTED":
                blk.ConnectBlock(_FACES[f], blocks[fd["connectedBlock"]], *[_FACES[a] for a in fd["axes"]])
            elif t == "PERIODIC":
                blk.MakePeriodic(f // 2)
            elif t in ("NEUMANN", "DIRICHLET", "DIRICHLET_VARYING"):
                raise NotImplementedError(f"Block '{blk.name}' face {_FACES[f]}: {t} boundaries (old format) cannot be loaded.")
            else:
                raise TypeError(f"Block '{blk.name}' face {_FACES[f]}: unknown boundary type {t!r}.")
    return dom


def _load_fixed(blk, f: int, fd: dict, get, with_scalar: bool) -> None:
    """A closed or open face with its velocity, scalar and potential conditions."""
    has_scalar = with_scalar and "scalar" in fd
    if fd.get("velocityType", "DIRICHLET") == "NEUMANN":
        st = fd.get("passiveScalarType", "NEUMANN")
        dirichlet = any(x == "DIRICHLET" for x in st) if isinstance(st, list) else st == "DIRICHLET"
        blk.OpenBoundary(f, get(fd, "scalar") if has_scalar and dirichlet else None)
    else:
        blk.CloseBoundary(f, get(fd, "velocity"), get(fd, "scalar") if has_scalar else None)
        if has_scalar:
            st = fd["passiveScalarType"]
            blk.getBoundary(f).setPassiveScalarType([BoundaryConditionType[x] for x in st] if isinstance(st, list)
                                                     else BoundaryConditionType[st])
    b = blk.getBoundary(f)
    values, types = get(fd, "potentialValues"), get(fd, "potentialTypes")
    if values is not None:
        b.setPotentialValues(values)
    cw = fd.get("potentialCw")
    if types is not None:
        if types.is_floating_point():
            types = types.round()
        b.setPotentialTypes(types.to(torch.int8), cw=cw)
    elif "potentialBC" in fd:
        b.setPotentialBC(PotentialBC[fd["potentialBC"]], cw=cw)
    else:
        # files written before PotentialBC existed hold independent flags (reference
        # io/domain_io.py:200-207), applied through the legacy setters in the same order
        if "epotCw" in fd:
            b.setEpotCw(fd["epotCw"])
        if "epotInsulating" in fd:
            b.setEpotInsulating(fd["epotInsulating"])
        if fd.get("epotDirichlet", False):
            b.setEpotDirichlet(True)


__all__ = ["FORMAT_VERSION", "load_domain", "save_domain"]
