"""Domain checkpoints in phiPICT's .json + .npz layout (src/phipict/io/domain_io.py), on the
CPU: round trips of every field and face setting (velocity, pressure, passive scalar with
types, potential conditions, connections, periodic faces, sources, vertex coordinates), dtype
conversion, path handling, atomic overwrites, and refusal of missing, mismatched,
inconsistent and newer files (the behaviours tests/test_domain_io.py of phiPICT checks)."""
import json
import shutil
from pathlib import Path

import numpy as np
import pytest
import torch

import phipict_b200 as pb
from phipict_b200.domain import BoundaryConditionType as BC
from phipict_b200.io import load_domain, save_domain
from cases import duct_3d, hartmann_2d


def _mhd_duct():
    dom = duct_3d(6, 5, 4, 2, device="cpu", channels=2)
    g = torch.Generator().manual_seed(0)
    dom.setPassiveScalarViscosity(torch.tensor([0.01, 0.03]))
    blocks = dom.getBlocks()
    for b in blocks:
        b.setVelocity(torch.randn(b.velocity.shape, generator=g, dtype=torch.float64))
        b.setPassiveScalar(torch.rand(b.passiveScalar.shape, generator=g, dtype=torch.float64))
        b.setEpot(torch.randn(b.velocity.shape[0], 1, *b.velocity.shape[2:], generator=g, dtype=torch.float64))
    blocks[0].getBoundary("-x").setPassiveScalar(torch.rand(1, 2, 4, 5, 1, generator=g, dtype=torch.float64))
    blocks[0].getBoundary("-y").setPassiveScalarType([BC.DIRICHLET, BC.NEUMANN])
    wall = blocks[1].getBoundary("+z")
    mask = torch.zeros(1, 1, 1, 5, 6, dtype=torch.int8)
    mask[..., ::2] = int(pb.PotentialBC.THIN_WALL)
    wall.setPotentialTypes(mask, cw=0.25)
    d = blocks[0].getBoundary("-z")
    d.setPotentialBC(pb.PotentialBC.DIRICHLET)
    d.setPotentialValues(torch.randn(1, 1, 1, 5, 6, generator=g, dtype=torch.float64))
    blocks[1].setVelocitySource(torch.tensor([[0.5, 0.0, -0.25]], dtype=torch.float64))
    return dom


def _assert_same(a, b):
    assert a.name == b.name and a.getSpatialDims() == b.getSpatialDims()
    assert a.getPassiveScalarChannels() == b.getPassiveScalarChannels()
    assert torch.equal(a.viscosity.to(b.viscosity.dtype), b.viscosity)
    if a.hasPassiveScalarViscosity():
        assert torch.equal(a.passiveScalarViscosity.to(b.passiveScalarViscosity.dtype), b.passiveScalarViscosity)
    for x, y in zip(a.getBlocks(), b.getBlocks(), strict=True):
        assert x.name == y.name and x.getSizes() == y.getSizes()
        for name in ("velocity", "pressure", "passiveScalar", "epot", "velocitySource", "vertexCoordinates"):
            tx, ty = getattr(x, name), getattr(y, name)
            assert (tx is None) == (ty is None), name
            if tx is not None:
                assert tx.dtype == ty.dtype and torch.equal(tx, ty), name
        for f, (bx, by) in enumerate(zip(x.getBoundaries(), y.getBoundaries(), strict=True)):
            assert type(bx) is type(by), (x.name, f)
            if isinstance(bx, pb.FixedBoundary):
                assert bx.velocityType == by.velocityType and torch.equal(bx.velocity, by.velocity)
                assert bx.passiveScalarTypes == by.passiveScalarTypes
                assert (bx.passiveScalar is None) == (by.passiveScalar is None)
                if bx.passiveScalar is not None:
                    assert torch.equal(bx.passiveScalar, by.passiveScalar)
                assert bx.getPotentialBC() == by.getPotentialBC() and bx.getPotentialCw() == by.getPotentialCw()
                for g in ("getPotentialTypes", "getPotentialValues"):
                    px, py = getattr(bx, g)(), getattr(by, g)()
                    assert (px is None) == (py is None) and (px is None or torch.equal(px, py)), g
            elif isinstance(bx, pb.domain.ConnectedBoundary):
                assert bx.axes == by.axes
                assert x.getParentDomain().getBlocks().index(bx.getConnectedBlock()) == \
                    y.getParentDomain().getBlocks().index(by.getConnectedBlock())


def test_roundtrip_of_every_setting(tmp_path: Path):
    dom = _mhd_duct()
    save_domain(dom, tmp_path / "duct")
    loaded = load_domain(tmp_path / "duct")
    _assert_same(dom, loaded)
    # saving the loaded domain gives the same description (apart from the save id)
    save_domain(loaded, tmp_path / "again")
    j1, j2 = (json.loads((tmp_path / f"{n}.json").read_text()) for n in ("duct", "again"))
    j1.pop("save_id"), j2.pop("save_id")
    assert j1 == j2


def test_roundtrip_of_a_periodic_channel_and_dtype_conversion(tmp_path: Path):
    dom = hartmann_2d(7, 5, device="cpu", dtype=torch.float32)
    dom.getBlocks()[0].setVelocity(torch.randn(1, 2, 5, 7, generator=torch.Generator().manual_seed(1)))
    save_domain(dom, tmp_path / "ch")
    _assert_same(dom, load_domain(tmp_path / "ch"))
    wide = load_domain(tmp_path / "ch", dtype=torch.float64)
    assert wide.getBlock(0).velocity.dtype == torch.float64
    assert torch.equal(wide.getBlock(0).velocity, dom.getBlock(0).velocity.double())


def test_loaded_domain_prepares_and_packs_its_scalar_faces(tmp_path: Path):
    save_domain(_mhd_duct(), tmp_path / "duct")
    loaded = load_domain(tmp_path / "duct")
    b0 = loaded.getBlocks()[0]
    assert b0.getBoundary("-y").passiveScalarTypes == [BC.DIRICHLET, BC.NEUMANN]
    assert not loaded.isAllFixedBoundariesPassiveScalarTypeStatic()


def test_paths(tmp_path: Path):
    dom = hartmann_2d(4, 3, device="cpu")
    with pytest.raises(TypeError, match="pathlib.Path"):
        save_domain(dom, str(tmp_path / "d"))
    with pytest.raises(TypeError, match="pathlib.Path"):
        load_domain(str(tmp_path / "d"))
    base = tmp_path / "new" / "dirs" / "Re2.5_domain"
    save_domain(dom, base.with_name(base.name + ".json"))
    assert sorted(p.name for p in base.parent.iterdir()) == ["Re2.5_domain.json", "Re2.5_domain.npz"]
    _assert_same(dom, load_domain(base.with_name(base.name + ".npz")))
    for _ in range(2):
        save_domain(dom, tmp_path / "d")
    assert sorted(p.name for p in tmp_path.iterdir() if p.is_file()) == ["d.json", "d.npz"]


def test_refuses_broken_pairs(tmp_path: Path):
    dom = hartmann_2d(4, 3, device="cpu")
    save_domain(dom, tmp_path / "a")
    save_domain(dom, tmp_path / "b")
    shutil.copy(tmp_path / "b.npz", tmp_path / "a.npz")
    with pytest.raises(ValueError, match="different saves"):
        load_domain(tmp_path / "a")
    save_domain(dom, tmp_path / "c")
    saved = json.loads((tmp_path / "c.json").read_text())
    saved["data_info"]["0"]["shape"] = [123]
    (tmp_path / "c.json").write_text(json.dumps(saved))
    with pytest.raises(ValueError, match="shape"):
        load_domain(tmp_path / "c")
    save_domain(dom, tmp_path / "v")
    saved = json.loads((tmp_path / "v.json").read_text())
    saved["format_version"] = 99
    (tmp_path / "v.json").write_text(json.dumps(saved))
    with pytest.raises(ValueError, match="format version 99"):
        load_domain(tmp_path / "v")
    (tmp_path / "b.npz").unlink()
    with pytest.raises(FileNotFoundError, match=r"b\.npz"):
        load_domain(tmp_path / "b")


def test_reads_version_1_files_and_stores_shared_tensors_once(tmp_path: Path):
    dom = hartmann_2d(4, 3, device="cpu")
    blk = dom.getBlock(0)
    blk.setVelocitySource(blk.velocity)  # the same storage twice
    save_domain(dom, tmp_path / "d")
    saved = json.loads((tmp_path / "d.json").read_text())
    assert saved["blocks"][0]["velocity"] == saved["blocks"][0]["velocitySource"]
    del saved["format_version"], saved["save_id"]
    (tmp_path / "d.json").write_text(json.dumps(saved))
    with np.load(tmp_path / "d.npz") as npz:
        arrays = {k: npz[k] for k in npz.files if k != "save_id"}
    np.savez_compressed(tmp_path / "d.npz", **arrays)
    _assert_same(dom, load_domain(tmp_path / "d"))


def test_reads_the_legacy_potential_flags_of_old_files(tmp_path: Path):
    """Files written before PotentialBC existed stored epotCw / epotInsulating /
    epotDirichlet per face (phiPICT io/domain_io.py:200-207); they map onto the potential BC
    as the legacy setters do (domain/boundaries.cpp:968-991)."""
    dom = duct_3d(6, 5, 4, 2, device="cpu")
    save_domain(dom, tmp_path / "d")
    saved = json.loads((tmp_path / "d.json").read_text())
    flags = {(0, 2): {"epotCw": 0.3}, (0, 3): {"epotDirichlet": True}, (1, 1): {"epotInsulating": False},
             (1, 2): {"epotCw": 0.0, "epotInsulating": True, "epotDirichlet": False}}
    for bi, bd in enumerate(saved["blocks"]):
        for f, fd in enumerate(bd["boundaries"]):
            fd.pop("potentialBC", None)
            fd.pop("potentialCw", None)
            fd.update(flags.get((bi, f), {}))
    del saved["format_version"], saved["save_id"]
    (tmp_path / "d.json").write_text(json.dumps(saved))
    with np.load(tmp_path / "d.npz") as npz:
        arrays = {k: npz[k] for k in npz.files if k != "save_id"}
    np.savez_compressed(tmp_path / "d.npz", **arrays)
    got = load_domain(tmp_path / "d")
    b0, b1 = got.getBlocks()
    P = pb.PotentialBC
    assert b0.getBoundary("-y").getPotentialBC() == P.THIN_WALL and b0.getBoundary("-y").getEpotCw() == 0.3
    assert b0.getBoundary("+y").getPotentialBC() == P.DIRICHLET and b0.getBoundary("+y").hasEpotDirichlet()
    assert b1.getBoundary("+x").getPotentialBC() == P.OPEN and not b1.getBoundary("+x").isEpotInsulating()
    assert b1.getBoundary("-y").getPotentialBC() == P.INSULATING
    # faces without flags keep the default
    assert b0.getBoundary("-x").getPotentialBC() == P.INSULATING
