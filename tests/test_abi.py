"""The C ABI library loads and exports every entry point include/phipict_b200.h declares
(no compute calls: these run without a GPU)."""
import ctypes as ct
import re
from pathlib import Path

from phipict_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> set[str]:
    text = (ROOT / "include" / "phipict_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"^\s*(?:const\s+)?[a-z0-9_]+\s*\*?\s*(phb_[a-z0-9_]+)\s*\(", text, flags=re.M))


def test_header_declares_what_the_binding_lists():
    assert declared_functions() == set(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_version_and_error_text():
    lib = _lib.load()
    assert lib.phb_version() >= 1
    # a rejected argument leaves a message and does not touch the device
    rc = lib.phb_advection_matrix(None, None, None, None, None, None)
    assert rc == -1
    assert b"null" in lib.phb_last_error()
    rc = lib.phb_nonortho_rhs(None, 0, None, None, None, None, None)
    assert rc == -1 and b"phb_nonortho_rhs" in lib.phb_last_error()


def test_struct_layouts_match_header():
    assert ct.sizeof(_lib.PhbTolerance) == 48
    assert ct.sizeof(_lib.PhbSolveResult) == 32
    assert _lib.PhbSolve.tol.offset == 32
    assert _lib.PhbDomain.blocks.offset == 48
    assert _lib.PhbDomain.nonortho.offset == 148 and ct.sizeof(_lib.PhbDomain) == 152
    assert ct.sizeof(_lib.PhbScalar) == 48 and _lib.PhbScalar.nu.offset == 8
    assert ct.sizeof(_lib.PhbCsrLevel) == 96 and _lib.PhbCsrLevel.n.offset == 88
    assert _lib.PhbCsrPcg.tol.offset == 56 and _lib.PhbCsrPcg.levels.offset == 112
    assert ct.sizeof(_lib.PhbCsrPcg) == 152


def test_csr_pcg_rejects_bad_arguments_without_a_gpu():
    lib = _lib.load()
    a = _lib.PhbCsrPcg()
    assert lib.phb_csr_pcg_work_bytes(ct.byref(a)) == -1
    assert b"phb_csr_pcg" in lib.phb_last_error()
    assert lib.phb_csr_pcg_solve(ct.byref(a), None, None) == -1
