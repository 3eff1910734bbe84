"""The C-ABI boundary without a GPU: exports, struct layouts, argument checks."""

from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from offline_particles_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions() -> list[str]:
    names = []
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(opb_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 16
    for name in names:
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\sT\s(opb_\w+)", out))
    assert set(names) == exported, f"exports differ from the header: {set(names) ^ exported}"


def test_every_declared_symbol_is_bound():
    bound = set(_lib.SIGNATURES) | set(_lib.SIGNATURES_OTHER)
    assert set(declared_functions()) - {"opb_last_error", "opb_abi_version"} == bound


LAYOUT_PROBE = r"""
#include <stddef.h>
#include <stdio.h>
#include "opb200.h"
#define F(T, m) printf(#T "." #m " %zu\n", offsetof(T, m))
#define S(T) printf(#T " %zu\n", sizeof(T))
int main(void) {
    S(opb_field); F(opb_field, data); F(opb_field, dtype); F(opb_field, ndim); F(opb_field, shape);
    F(opb_field, offset); F(opb_field, is_static); F(opb_field, nslots); F(opb_field, scale);
    S(opb_roms_fields); F(opb_roms_fields, zeta); F(opb_roms_fields, C);
    S(opb_time); F(opb_time, ft); F(opb_time, gt);
    S(opb_particles); F(opb_particles, status); F(opb_particles, z); F(opb_particles, dz2); F(opb_particles, err);
    F(opb_particles, rho_t);
    S(opb_scalars); F(opb_scalars, NZ); F(opb_scalars, dt); F(opb_scalars, alpha); F(opb_scalars, bounds);
    F(opb_scalars, w_max); F(opb_scalars, rho_scale);
    S(opb_experiment); F(opb_experiment, count); F(opb_experiment, first_chunk); F(opb_experiment, scheme);
    F(opb_experiment, nsteps); F(opb_experiment, table_offset); F(opb_experiment, validate);
    F(opb_experiment, dt); F(opb_experiment, alpha);
    S(opb_batch_header); F(opb_batch_header, nchunks); F(opb_batch_header, next_chunk);
    return 0;
}
"""


def test_struct_layouts_match_ctypes(tmp_path):
    src = tmp_path / "probe.c"
    src.write_text(LAYOUT_PROBE)
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c99", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    lines = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    c = dict(line.rsplit(" ", 1) for line in lines if line)
    types = {"opb_field": _lib.opb_field, "opb_roms_fields": _lib.opb_roms_fields, "opb_time": _lib.opb_time,
             "opb_particles": _lib.opb_particles, "opb_scalars": _lib.opb_scalars,
             "opb_experiment": _lib.opb_experiment, "opb_batch_header": _lib.opb_batch_header}
    for key, val in c.items():
        if "." in key:
            t, m = key.split(".")
            assert getattr(types[t], m).offset == int(val), key
        else:
            assert ctypes.sizeof(types[key]) == int(val), key


def test_argument_errors_need_no_gpu():
    lib = _lib.load()
    assert lib.opb_validation(None, None, None) == _lib.EINVAL
    assert b"particles is NULL" in lib.opb_last_error()
    p = _lib.opb_particles()
    p.n = -1
    assert lib.opb_finite_indices(ctypes.byref(p), None) == _lib.EINVAL
    p.n = 0
    assert lib.opb_finite_indices(ctypes.byref(p), None) == _lib.OK  # nothing to launch
    p.n = 4
    assert lib.opb_finite_indices(ctypes.byref(p), None) == _lib.EINVAL  # status NULL
    # a field with one point along a dimension cannot be interpolated
    f = _lib.opb_field()
    f.ndim, f.is_static, f.dtype = 1, 1, _lib.F64
    f.data[0] = 16
    f.shape[0] = 1
    p.status = p.zidx = p.yidx = p.xidx = 16
    assert lib.opb_linear_interpolation(ctypes.byref(p), 16, ctypes.byref(f), None, 16, None) == _lib.EINVAL
    assert b"size 1" in lib.opb_last_error()
    # mixed storage dtypes across time-dependent fields are rejected
    rf = _lib.opb_roms_fields()
    for name, nd in (("u", 3), ("v", 3), ("w", 3), ("dx", 2), ("dy", 2), ("h", 2), ("zeta", 2), ("C", 1)):
        g = getattr(rf, name)
        g.ndim = nd
        for d in range(nd):
            g.shape[d] = 4
        g.data[0] = g.data[1] = 16
        if name in ("u", "v", "w", "zeta"):
            g.nslots, g.dtype = 2, _lib.F32
        else:
            g.is_static, g.dtype = 1, _lib.F64
    rf.v.dtype = _lib.F64
    s = _lib.opb_scalars()
    t = _lib.opb_time(0, 1, 0.0, 1.0)
    p.z = p.dxidx1 = p.dyidx1 = p.dz1 = 16
    rc = lib.opb_rk2_w_advection_step_1(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), ctypes.byref(t), None)
    assert rc == _lib.EINVAL and b"share one storage dtype" in lib.opb_last_error()
    rf.v.dtype = _lib.F32
    t.next = 5
    rc = lib.opb_rk2_w_advection_step_1(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), ctypes.byref(t), None)
    assert rc == _lib.EINVAL and b"slot out of range" in lib.opb_last_error()
    # the isopycnal follower needs the particles' target density
    t.next = 1
    p.dxidx0 = p.dyidx0 = p.dz0 = p.dxidx2 = p.dyidx2 = p.dz2 = 16
    rc = lib.opb_ab3_isopycnal_following(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), ctypes.byref(t), None)
    assert rc == _lib.EINVAL and b"rho_t" in lib.opb_last_error()
    rc = lib.opb_ab3_isopycnal_following_steps(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), 16, 1, 1, None)
    assert rc == _lib.EINVAL and b"rho_t" in lib.opb_last_error()
    # snapshot quads come with x-pairs of h, dx and dy, all four time-dependent fields quads, float32 only
    for name in ("u", "v", "w", "zeta"):
        getattr(rf, name).dtype = _lib.F32_QUADS
    rc = lib.opb_ab3_w_advection_steps(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), 16, 1, 1, None)
    assert rc == _lib.EINVAL and b"static x-pairs" in lib.opb_last_error()
    rf.zeta.dtype = _lib.F32_PAIRS
    for name in ("h", "dx", "dy"):
        getattr(rf, name).dtype = _lib.F64_XPAIRS
    rc = lib.opb_ab3_w_advection_steps(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), 16, 1, 1, None)
    assert rc == _lib.EINVAL and b"every time-dependent field" in lib.opb_last_error()
    for name in ("u", "v", "w", "zeta"):
        getattr(rf, name).dtype = _lib.F32
    rc = lib.opb_ab3_w_advection_steps(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), 16, 1, 1, None)
    assert rc == _lib.EINVAL and b"come with snapshot quads only" in lib.opb_last_error()
    # a vector layout's buffers must be aligned to its load width
    for name in ("u", "v", "w", "zeta"):
        getattr(rf, name).dtype = _lib.F32_QUADS
    rf.h.data[0] = 24
    rc = lib.opb_ab3_w_advection_steps(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), 16, 1, 1, None)
    assert rc == _lib.EINVAL and b"not 16-byte aligned" in lib.opb_last_error()
    rf.h.data[0] = 16
    rf.u.data[1] = 8
    rc = lib.opb_ab3_w_advection_steps(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), 16, 1, 1, None)
    assert rc == _lib.EINVAL and b"not 16-byte aligned" in lib.opb_last_error()
    rf.u.data[1] = 16
    # octets come with yx-pairs, 32-byte aligned
    for name in ("u", "v", "w", "zeta"):
        g = getattr(rf, name)
        g.dtype, g.data[0], g.data[1] = _lib.F32_OCTS, 32, 32
    rc = lib.opb_ab3_w_advection_steps(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), 16, 1, 1, None)
    assert rc == _lib.EINVAL and b"static yx-pairs" in lib.opb_last_error()
    for name in ("h", "dx", "dy"):
        getattr(rf, name).dtype = _lib.F64_YXPAIRS
    rc = lib.opb_ab3_w_advection_steps(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), 16, 1, 1, None)
    assert rc == _lib.EINVAL and b"not 32-byte aligned" in lib.opb_last_error()
    assert lib.opb_interleave_octets(16, 16, 48, 4, 2, None) == _lib.EINVAL
    assert b"32-byte aligned" in lib.opb_last_error()
    # 2-D bundles: all four codes together, shapes and offsets shared, with float32 pairs or quads
    for name in ("u", "v", "w"):
        g = getattr(rf, name)
        g.dtype, g.data[0], g.data[1] = _lib.F32_PAIRS, 32, 32
    rf.zeta.dtype, rf.zeta.data[0], rf.zeta.data[1] = _lib.F32_ZETA_H, 32, 32
    rf.h.dtype = _lib.F64_IN_ZETA
    rf.dx.dtype, rf.dx.data[0] = _lib.F64_DX_DY, 32
    rf.dy.dtype = _lib.F64
    rc = lib.opb_ab3_w_advection_steps(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), 16, 1, 1, None)
    assert rc == _lib.EINVAL and b"together" in lib.opb_last_error()
    rf.dy.dtype = _lib.F64_IN_DX
    rf.dy.offset[0] = 0.5
    rc = lib.opb_ab3_w_advection_steps(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), 16, 1, 1, None)
    assert rc == _lib.EINVAL and b"share their shape and offsets" in lib.opb_last_error()
    rf.dy.offset[0] = 0.0
    rf.dx.data[0] = 48
    rc = lib.opb_ab3_w_advection_steps(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), 16, 1, 1, None)
    assert rc == _lib.EINVAL and b"not 32-byte aligned" in lib.opb_last_error()
    rf.dx.data[0] = 32
    for name in ("u", "v", "w"):
        getattr(rf, name).dtype = _lib.F32_OCTS
    rc = lib.opb_ab3_w_advection_steps(ctypes.byref(p), ctypes.byref(s), ctypes.byref(rf), 16, 1, 1, None)
    assert rc == _lib.EINVAL and b"float32 snapshot pairs or quads" in lib.opb_last_error()
    assert lib.opb_interleave_quads(16, 16, 20, 4, None) == _lib.EINVAL
    assert b"16-byte aligned" in lib.opb_last_error()


def test_call_raises_value_error():
    with pytest.raises(ValueError, match="NULL"):
        _lib.call("opb_validation", None, None, None)


CONSTANT_PROBE = r"""
#include <stdio.h>
#include "opb200.h"
#define C(name) printf(#name " %d\n", (int)(name))
int main(void) {
    C(OPB_ABI_VERSION); C(OPB_MAX_SLOTS); C(OPB_F64); C(OPB_F32); C(OPB_BF16); C(OPB_F16); C(OPB_F64_PAIRS);
    C(OPB_F32_PAIRS); C(OPB_F32_QUADS); C(OPB_F64_XPAIRS); C(OPB_F32_OCTS); C(OPB_F64_YXPAIRS);
    C(OPB_INLINE_TABLE); C(OPB_EINVAL); C(OPB_ECUDA); C(OPB_F32_ZETA_H); C(OPB_F64_IN_ZETA); C(OPB_F64_DX_DY);
    C(OPB_F64_IN_DX); C(OPB_NOALLOC_MAX_PARTICLES); C(OPB_NOALLOC_SORT_TEMP_BYTES); C(OPB_NOALLOC_SCRATCH_BYTES);
    return 0;
}
"""


def test_header_constants_match_the_binding(tmp_path):
    src = tmp_path / "consts.c"
    src.write_text(CONSTANT_PROBE)
    exe = tmp_path / "consts"
    subprocess.run(["gcc", "-std=c99", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    c = {k: int(v) for k, v in (line.split() for line in out if line)}
    py = {"OPB_ABI_VERSION": _lib.ABI_VERSION, "OPB_MAX_SLOTS": _lib.MAX_SLOTS, "OPB_F64": _lib.F64,
          "OPB_F32": _lib.F32, "OPB_BF16": _lib.BF16, "OPB_F16": _lib.F16, "OPB_F64_PAIRS": _lib.F64_PAIRS,
          "OPB_F32_PAIRS": _lib.F32_PAIRS, "OPB_F32_QUADS": _lib.F32_QUADS, "OPB_F64_XPAIRS": _lib.F64_XPAIRS,
          "OPB_F32_OCTS": _lib.F32_OCTS, "OPB_F64_YXPAIRS": _lib.F64_YXPAIRS,
          "OPB_INLINE_TABLE": _lib.INLINE_TABLE, "OPB_EINVAL": _lib.EINVAL, "OPB_ECUDA": _lib.ECUDA,
          "OPB_F32_ZETA_H": _lib.F32_ZETA_H, "OPB_F64_IN_ZETA": _lib.F64_IN_ZETA, "OPB_F64_DX_DY": _lib.F64_DX_DY,
          "OPB_F64_IN_DX": _lib.F64_IN_DX}
    noalloc = {k: c.pop(k) for k in ("OPB_NOALLOC_MAX_PARTICLES", "OPB_NOALLOC_SORT_TEMP_BYTES",
                                     "OPB_NOALLOC_SCRATCH_BYTES")}
    assert c == py
    # the static scratch of opb_sort_particles_noalloc: two key buffers and one id buffer of the maximum count,
    # then the radix passes' tile counts, which fit its temporary part at the maximum count
    assert noalloc["OPB_NOALLOC_MAX_PARTICLES"] == _lib.NOALLOC_MAX_PARTICLES
    assert noalloc["OPB_NOALLOC_SCRATCH_BYTES"] == 12 * _lib.NOALLOC_MAX_PARTICLES + noalloc["OPB_NOALLOC_SORT_TEMP_BYTES"]
    assert _radix_temp(_lib.NOALLOC_MAX_PARTICLES, 2048) <= noalloc["OPB_NOALLOC_SORT_TEMP_BYTES"]


def _a256(b: int) -> int:
    return (b + 255) // 256 * 256


def _radix_temp(n: int, tile: int) -> int:
    """Scratch of the radix sort for n keys: 256 tile counts per tile of `tile` keys and 256 digit totals."""
    return _a256(256 * -(-n // tile) * 4) + _a256(256 * 4)


def test_sort_workspace_sizes_need_no_gpu():
    """The sort workspaces are sized on the host, with no device query: for opb_sort_particles three 4-byte
    arrays of n entries (keys in and out, the intermediate ids) and the radix scratch of 2048-key tiles; for
    opb_sort_segments the 64-bit keys, ids, slots, segment table, staged particle state and the radix scratch.
    Every piece starts on a 256-byte boundary."""
    lib = _lib.load()
    assert lib.opb_sort_workspace_bytes(0) == 0
    for n in (1, 2047, 2048, 2049, 1 << 20, 4_194_304, 45_728_029):
        assert lib.opb_sort_workspace_bytes(n) == 3 * _a256(4 * n) + _radix_temp(n, 2048), n
    assert lib.opb_sort_segments_workspace_bytes(0, 3) == 0
    for m, nseg in ((1, 1), (50_000, 3), (45_728_029, 256)):
        want = (2 * _a256(8 * m) + 3 * _a256(4 * m) + _a256(16 * nseg) + _a256(m) + _a256(8 * 13 * m) + _a256(8 * m)
                + _radix_temp(m, 2048))
        assert lib.opb_sort_segments_workspace_bytes(m, nseg) == want, (m, nseg)


def test_integration_stub_matches_the_binding():
    """The reference-side ctypes stub in INTEGRATION.md declares the structs with the header's layouts."""
    text = (ROOT / "INTEGRATION.md").read_text()
    block = re.search(r"```python\n(# offline_particles/kernels/roms/_b200\.py.*?)```", text, flags=re.S).group(1)
    real_cdll = ctypes.CDLL
    ns: dict = {}
    try:
        ctypes.CDLL = lambda name: real_cdll(str(_lib.LIB_PATH))  # the stub loads the library by name
        exec(compile(block, "INTEGRATION.md", "exec"), ns)
    finally:
        ctypes.CDLL = real_cdll
    for name in ("opb_field", "opb_roms_fields", "opb_time", "opb_particles", "opb_scalars", "opb_records"):
        stub, ours = ns[name], getattr(_lib, name)
        assert ctypes.sizeof(stub) == ctypes.sizeof(ours), name
        for fname, _ in ours._fields_:
            assert getattr(stub, fname.lstrip("_") if fname.lstrip("_") in dir(stub) else fname).offset == \
                getattr(ours, fname).offset, (name, fname)
