"""Build recipe of the reference itself, for parity fixtures only (test infrastructure).

Compiles phiPICT's ``_C`` extension from the reference's C++/CUDA sources where they lie
(``csrc/phipict/**``, the source list and flags of the reference's ``setup.py:62-112``) with
``torch.utils.cpp_extension.load`` for sm_100, and lays the reference's pure-Python package
(``src/phipict``) beside it, so that ``import phipict`` with ``oracle/_ref`` on ``sys.path`` is the
unmodified reference (the same result ``pip install --target`` would give).

Outputs go to ``oracle/_ref/`` only (git-ignored, so the built files never enter the history,
but they travel with the repository snapshot to a GPU machine). Object files are built in
``oracle/_ref/build`` and removed after a successful link. Nothing in ``phipict_b200`` imports
or links any of this: it is used by ``tests/golden/make_ref_fields.py`` on a GPU machine to
produce the committed field fixtures, and by nothing else.

Usage: ``python -m oracle.build_ref --reference <reference root>`` (the root that holds
``csrc/`` and ``src/``; default: the ``PHIPICT_REFERENCE`` environment variable). Takes about
ten minutes on eight cores.
"""
from __future__ import annotations

import argparse
import os
import shutil
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
PKG = OUT / "phipict"

# setup.py:62-87 of the reference: the sources of phipict._C
SOURCES = [
    "bindings.cpp",
    "domain/csr_matrix.cpp", "domain/boundaries.cpp", "domain/block.cpp", "domain/domain.cpp",
    "piso/launch.cu", "piso/advection.cu", "piso/pressure.cu", "piso/velocity_correction.cu",
    "piso/analysis.cu", "piso/result_copy.cu", "piso/sgs.cu",
    "mhd/potential.cu",
    "solvers/linear_solve.cu", "solvers/krylov/krylov.cu", "solvers/legacy_cg.cu",
    "solvers/legacy_bicgstab.cu",
    "grid/grid_gen.cu", "grid/resampling.cu", "grid/transform_vectors.cu",
    "math/eigenvalue.cu", "math/ortho_basis.cu", "math/matrix_vector_ops.cu",
    "math/matrix_vector_ops_grads.cu",
]


def built() -> bool:
    return PKG.is_dir() and any(PKG.glob("_C*.so")) and (PKG / "__init__.py").exists()


def build(reference: Path, force: bool = False, jobs: int | None = None) -> Path:
    if built() and not force:
        return PKG
    reference = Path(reference).resolve()
    csrc = reference / "csrc" / "phipict"
    src = reference / "src" / "phipict"
    if not csrc.is_dir() or not src.is_dir():
        raise FileNotFoundError(f"no reference sources under {reference}")
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0")
    os.environ.setdefault("MAX_JOBS", str(jobs or os.cpu_count() or 8))
    from torch.utils import cpp_extension

    if PKG.exists():
        shutil.rmtree(PKG)
    shutil.copytree(src, PKG, ignore=shutil.ignore_patterns("__pycache__", "*.pyc", "*.so"))
    for path in [PKG, *PKG.rglob("*")]:  # the sources may be read-only; the copy stays removable
        path.chmod(path.stat().st_mode | 0o200)
    bdir = OUT / "build"
    bdir.mkdir(parents=True, exist_ok=True)
    t0 = time.time()
    # setup.py:89-110: same macro and optimisation flags
    mod = cpp_extension.load(
        name="_C",
        sources=[str(csrc / s) for s in SOURCES],
        extra_include_paths=[str(csrc)],
        extra_cflags=["-DPYTHON_EXTENSION_BUILD=1", "-fvisibility=hidden", "-Ofast", "-w"],
        extra_cuda_cflags=["-DPYTHON_EXTENSION_BUILD=1", "--threads=2", "-O3", "--use_fast_math",
                           "--compiler-options=-w"],
        build_directory=str(bdir),
        verbose=False,
        is_python_module=True,
    )
    so = Path(mod.__file__)
    shutil.copy2(so, PKG / so.name)
    shutil.rmtree(bdir, ignore_errors=True)
    print(f"built {PKG / so.name} in {time.time() - t0:.0f} s", flush=True)
    return PKG


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PHIPICT_REFERENCE"))
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args()
    if not a.reference:
        sys.exit("give --reference <root> or set PHIPICT_REFERENCE")
    build(Path(a.reference), force=a.force, jobs=a.jobs)


if __name__ == "__main__":
    main()
