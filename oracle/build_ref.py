"""Build recipe for ``oracle/_ref``: the reference's own Cython kernels, compiled here.

Test infrastructure only.  The reference (``offline_particles``) keeps its hot
loops in eight Cython modules (``CMakeLists.txt:14-23``).  This script compiles
them from the sources where they lie -- nothing is copied into this repository --
with the flags the reference's CMake build uses (``cython -3 -X
boundscheck=False``, ``CMakeLists.txt:26``; C at ``-O3 -DNDEBUG`` with OpenMP,
``CMakeLists.txt:66-68``).  Outputs go only to ``oracle/_ref/`` (git-ignored).

The reference's pure-Python modules are *not* copied: ``oracle/ref_import.py``
imports them from the reference checkout and takes the compiled extension
modules from ``oracle/_ref``.  The result therefore exists only on a machine
that has the reference checkout; it is used to pin the oracle and to generate
the committed golden fixtures under ``tests/golden/``.

Usage: ``python oracle/build_ref.py [--src REF_SRC_DIR]``.
"""

from __future__ import annotations

import argparse
import os
import subprocess
import sys
import sysconfig
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
DEFAULT_SRC = Path(os.environ.get("OFFLINE_PARTICLES_REF_SRC", "/root/reference/src"))

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


def build(src: Path = DEFAULT_SRC, force: bool = False) -> Path:
    pkg = src / "offline_particles"
    if not pkg.is_dir():
        raise FileNotFoundError(f"reference package not found under {src}")
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    inc = sysconfig.get_paths()["include"]
    cdir = OUT / "csrc"
    for mod in MODULES:
        pyx = pkg / f"{mod}.pyx"
        c_file = cdir / f"{mod}.c"
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
