"""Build recipe for ``oracle/_ref``: the reference itself, compiled here.

Test infrastructure only.  The reference (``offline_particles``) keeps its hot
loops in eight Cython modules (``CMakeLists.txt:14-23``).  This script compiles
them from the sources where they lie -- nothing is copied into this repository --
with the flags the reference's CMake build uses (``cython -3 -X
boundscheck=False``, ``CMakeLists.txt:26``; C at ``-O3 -DNDEBUG`` with OpenMP,
``CMakeLists.txt:66-68``), in a temporary folder, and keeps only the compiled
extension modules.  Its pure-Python modules (the fields' time blend, the
launcher, the steppers, ``Simulation``) are compiled to bytecode (``.pyc``,
``py_compile``) into one zip beside them (``offline_particles_py.zip``).  Outputs go only to ``oracle/_ref/``
(git-ignored, never committed); there the compiled package imports without
the reference's sources (``oracle/ref_import.py: import_compiled``), which is
how the CPU baseline runs the reference's own code on a machine that has no
reference checkout.  It also pins the oracle and generates the committed
golden fixtures under ``tests/golden/``.

The sources are read from ``$OFFLINE_PARTICLES_REF_SRC``, else from
``reference/src`` beside this repository's folder.

Usage: ``python oracle/build_ref.py [--src REF_SRC_DIR]``.
"""

from __future__ import annotations

import argparse
import os
import py_compile
import subprocess
import sys
import sysconfig
import tempfile
import zipfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
PY_ZIP = OUT / "offline_particles_py.zip"
DEFAULT_SRC = Path(os.environ.get("OFFLINE_PARTICLES_REF_SRC", HERE.parent.parent / "reference" / "src"))

# (module path relative to the package root) -- CMakeLists.txt:14-23
MODULES = (
    "kernels/_core",
    "kernels/status",
    "kernels/validation",
    "kernels/output/linear_interpolation",
    "kernels/roms/_roms_core",
    "kernels/roms/ab3_w_advection",
    "kernels/roms/ab3_isopycnal_following",
    "kernels/roms/rk2_w_advection",
)

# x86-64 gcc without -march: no FMA contraction, strict IEEE double (the
# reference's release build); the oracle restatement is compiled the same way.
CFLAGS = ["-O3", "-DNDEBUG", "-fPIC", "-fopenmp", "-shared", "-w"]


def _gcc() -> str:
    # /usr/bin/gcc ships libgomp.spec; another gcc on PATH may not.
    return "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc"


def _empty_pyc(path: Path) -> bytes:
    path.write_text("")
    out = path.with_suffix(".pyc")
    py_compile.compile(str(path), cfile=str(out), doraise=True,
                       invalidation_mode=py_compile.PycInvalidationMode.UNCHECKED_HASH)
    return out.read_bytes()


def build(src: Path = DEFAULT_SRC, force: bool = False) -> Path:
    pkg = src / "offline_particles"
    if not pkg.is_dir():
        raise FileNotFoundError(f"reference package not found under {src}")
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    inc = sysconfig.get_paths()["include"]
    with tempfile.TemporaryDirectory(prefix="opb_ref_") as tmp:
        for mod in MODULES:
            pyx = pkg / f"{mod}.pyx"
            c_file = Path(tmp) / f"{mod}.c"
            so = OUT / "offline_particles" / f"{mod}{ext}"
            if so.exists() and not force and so.stat().st_mtime >= pyx.stat().st_mtime:
                continue
            c_file.parent.mkdir(parents=True, exist_ok=True)
            so.parent.mkdir(parents=True, exist_ok=True)
            # the .pxd files next to the .pyx are found through the include path
            subprocess.run(
                [sys.executable, "-m", "cython", "-3", "-X", "boundscheck=False",
                 "-I", str(src), "-o", str(c_file), str(pyx)],
                check=True, cwd=str(src),
            )
            subprocess.run([_gcc(), *CFLAGS, f"-I{inc}", str(c_file), "-o", str(so)], check=True)
    # the pure-Python modules as sourceless bytecode in one zip (zipimport loads .pyc without sources)
    sources = sorted(pkg.rglob("*.py"))
    if force or not PY_ZIP.exists() or any(py.stat().st_mtime > PY_ZIP.stat().st_mtime for py in sources):
        tmp_zip = PY_ZIP.with_suffix(f".{os.getpid()}.tmp")
        with tempfile.TemporaryDirectory(prefix="opb_ref_pyc_") as tmp, \
                zipfile.ZipFile(tmp_zip, "w", zipfile.ZIP_DEFLATED) as zf:
            for py in sources:
                rel = py.relative_to(pkg)
                pyc = Path(tmp) / rel.with_suffix(".pyc")
                pyc.parent.mkdir(parents=True, exist_ok=True)
                py_compile.compile(str(py), cfile=str(pyc), dfile=f"offline_particles/{rel}", doraise=True,
                                   invalidation_mode=py_compile.PycInvalidationMode.UNCHECKED_HASH)
                zf.write(pyc, f"offline_particles/{rel.with_suffix('.pyc')}")
            # folders the reference leaves as namespace packages (no __init__.py, e.g. models/) get an
            # empty package module: zipimport does not resolve namespace packages
            dirs = {py.parent for py in sources} | {d for py in sources for d in py.parents if pkg in d.parents}
            for d in sorted(dirs):
                if d != pkg and pkg in d.parents and not (d / "__init__.py").exists():
                    zf.writestr(f"offline_particles/{d.relative_to(pkg)}/__init__.pyc",
                                _empty_pyc(Path(tmp) / "empty.py"))
        os.replace(tmp_zip, PY_ZIP)
    import shutil

    for stale in [OUT / "csrc", *(p for p in (OUT / "offline_particles").rglob("*.pyc"))]:
        if stale.is_dir():  # older builds kept the generated C here
            shutil.rmtree(stale)
        elif stale.exists():  # older builds kept loose bytecode
            stale.unlink()
    return OUT


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--src", type=Path, default=DEFAULT_SRC)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    out = build(a.src, a.force)
    print(f"reference kernels built into {out}")


if __name__ == "__main__":
    main()
