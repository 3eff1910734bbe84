"""Build liboffline_particles_b200.so for sm_100a.

The repository's ``CMakeLists.txt`` is the build description; this module
drives it (``cmake`` + ``ninja``).  Where CMake is unavailable it runs the same
``nvcc`` commands directly.  The library is written into
``offline_particles_b200/_lib/`` next to the package, never installed elsewhere.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
LIB_DIR = PKG / "_lib"
LIB_PATH = LIB_DIR / "liboffline_particles_b200.so"
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"

GENCODE = "-gencode=arch=compute_100a,code=sm_100a"
# per-file flags, as CMakeLists.txt sets them: the float64 path contracts no
# multiply-add (bit parity with the reference); the float32 path may
SOURCE_FLAGS = {"opb_roms.cu": ["-fmad=false"], "opb_batched.cu": ["-fmad=false"], "opb_fast.cu": ["-prec-div=false", "-ftz=true"]}


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _deps() -> list[Path]:
    return _sources() + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h")) + [ROOT / "CMakeLists.txt"]


def up_to_date() -> bool:
    if not LIB_PATH.exists():
        return False
    t = LIB_PATH.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in _deps() if p.exists())


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(cuda) / "bin" / "nvcc"
    return str(cand) if cand.exists() else "nvcc"


def _build_nvcc(build_dir: Path) -> None:
    build_dir.mkdir(parents=True, exist_ok=True)
    objs = []
    for src in _sources():
        obj = build_dir / (src.stem + ".o")
        flags = [GENCODE, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
                 f"-I{INCLUDE}", f"-I{CSRC}"]
        flags += SOURCE_FLAGS.get(src.name, [])
        subprocess.run([_nvcc(), *flags, "-c", str(src), "-o", str(obj)], check=True)
        objs.append(str(obj))
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    tmp = LIB_PATH.with_suffix(f".{os.getpid()}.tmp")
    subprocess.run([_nvcc(), GENCODE, "-shared", "-cudart", "static", *objs, "-o", str(tmp)], check=True)
    os.replace(tmp, LIB_PATH)


def _build_cmake(build_dir: Path) -> None:
    gen = ["-G", "Ninja"] if shutil.which("ninja") else []
    subprocess.run(["cmake", "-S", str(ROOT), "-B", str(build_dir), *gen, f"-DCMAKE_CUDA_COMPILER={_nvcc()}",
                    "-DCMAKE_BUILD_TYPE=Release"], check=True, stdout=subprocess.DEVNULL)
    subprocess.run(["cmake", "--build", str(build_dir), "--parallel"], check=True, stdout=subprocess.DEVNULL)


def build_library(force: bool = False, use_cmake: bool | None = None) -> Path:
    """Compile the CUDA library if any source is newer than it; return its path."""
    if not force and up_to_date():
        return LIB_PATH
    build_dir = ROOT / "_build"
    if use_cmake is None:
        use_cmake = shutil.which("cmake") is not None
    if use_cmake:
        try:
            _build_cmake(build_dir / "cmake")
        except (subprocess.CalledProcessError, FileNotFoundError):
            _build_nvcc(build_dir / "nvcc")
    else:
        _build_nvcc(build_dir / "nvcc")
    if not LIB_PATH.exists():
        raise RuntimeError(f"build did not produce {LIB_PATH}")
    os.utime(LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build_library(force=True))
