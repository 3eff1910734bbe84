"""Import the reference package (``offline_particles``) for pinning the oracle and timing it.

Test infrastructure only.  ``import_reference``: the pure-Python modules are
read from the reference checkout, the eight Cython extension modules come from
``oracle/_ref`` (built by ``oracle/build_ref.py``).  ``import_compiled``: the
whole package from ``oracle/_ref`` (the extension modules and the bytecode of
the pure-Python modules), on a machine without the reference's sources -- the
CPU baseline's way of running the reference's own code.  ``dask`` and ``zarr``
are not installed here, and the
reference's numpy path touches them only in annotations and in ``from_dask`` /
the zarr writer (``fields.py:6,443-458``; ``spatial_arrays.py:9,228-295``;
``output/_zarr_writer.py:7-8``), so empty stand-in modules satisfy its imports.
"""

from __future__ import annotations

import importlib.machinery
import importlib.util
import os
import sys
import types
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_OUT = HERE / "_ref"
DEFAULT_SRC = Path(os.environ.get("OFFLINE_PARTICLES_REF_SRC", HERE.parent.parent / "reference" / "src"))


def available(src: Path = DEFAULT_SRC) -> bool:
    return (src / "offline_particles" / "__init__.py").exists()


class _ExtFinder:
    """Resolve ``offline_particles.*`` extension modules to ``oracle/_ref``."""

    def __init__(self, root: Path) -> None:
        self.root = root
        self.suffix = importlib.machinery.EXTENSION_SUFFIXES[0]

    def find_spec(self, fullname, path=None, target=None):
        if not fullname.startswith("offline_particles."):
            return None
        rel = fullname.split(".")[1:]
        so = self.root.joinpath("offline_particles", *rel[:-1], rel[-1] + self.suffix)
        if not so.exists():
            return None
        loader = importlib.machinery.ExtensionFileLoader(fullname, str(so))
        return importlib.util.spec_from_file_location(fullname, str(so), loader=loader)


def _stub_getattr(attr: str):
    if attr.startswith("__"):
        raise AttributeError(attr)
    return type(attr, (), {})


def _stub_missing_deps() -> None:
    for name in ("dask", "dask.array", "zarr", "zarr.storage"):
        if name in sys.modules:
            continue
        try:
            __import__(name)
        except ImportError:
            mod = types.ModuleType(name)
            mod.Array = object  # used only in annotations / isinstance on the dask path
            mod.__getattr__ = _stub_getattr  # type: ignore[attr-defined]
            sys.modules[name] = mod
    if "dask" in sys.modules and "dask.array" in sys.modules:
        sys.modules["dask"].array = sys.modules["dask.array"]  # type: ignore[attr-defined]
    if "zarr" in sys.modules and "zarr.storage" in sys.modules:
        sys.modules["zarr"].storage = sys.modules["zarr.storage"]  # type: ignore[attr-defined]


def import_reference(src: Path = DEFAULT_SRC, build: bool = True):
    """Return the imported reference package ``offline_particles``."""
    if "offline_particles" in sys.modules:
        return sys.modules["offline_particles"]
    if not available(src):
        raise ImportError(f"reference checkout not found under {src}")
    if build:
        from oracle import build_ref

        build_ref.build(src)
    _stub_missing_deps()
    sys.meta_path.insert(0, _ExtFinder(REF_OUT))
    sys.path.insert(0, str(src))
    try:
        import offline_particles  # noqa: F401
    finally:
        sys.path.remove(str(src))
    return sys.modules["offline_particles"]


PY_ZIP = REF_OUT / "offline_particles_py.zip"


def compiled_available() -> bool:
    """``oracle/_ref`` holds the whole compiled package (``oracle/build_ref.py`` ran): the bytecode zip of
    the pure-Python modules and the extension modules."""
    pkg = REF_OUT / "offline_particles"
    return PY_ZIP.exists() and any((pkg / "kernels" / "roms").glob("ab3_w_advection*.so"))


def import_compiled():
    """Return the reference package imported from ``oracle/_ref`` alone (no sources needed): its
    pure-Python modules from the bytecode zip, its extension modules from ``oracle/_ref``."""
    if "offline_particles" in sys.modules:
        return sys.modules["offline_particles"]
    if not compiled_available():
        raise ImportError(f"no compiled reference under {REF_OUT}; run oracle/build_ref.py where the sources are")
    _stub_missing_deps()
    sys.meta_path.insert(0, _ExtFinder(REF_OUT))
    sys.path.insert(0, str(PY_ZIP))
    try:
        import offline_particles  # noqa: F401
    finally:
        sys.path.remove(str(PY_ZIP))
    return sys.modules["offline_particles"]
