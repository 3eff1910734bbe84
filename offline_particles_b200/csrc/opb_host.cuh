// Host-side conversion of the C-ABI structs into kernel arguments, checks and
// dispatch, shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <map>
#include <mutex>
#include <utility>

#include "opb200.h"
#include "opb_device.cuh"
#include "opb_errors.h"

namespace opb {
namespace {

constexpr int kHostBlock = 256;

// -------------------------------------------------------------- dispatch
// Call f(T{}, I{}) for the storage type and the index width of a launch.
template <typename F>
void dispatch(int dtype, bool small_index, F &&f) {
    if (dtype == OPB_F32) {
        if (small_index) f(float{}, int{});
        else f(float{}, (long long){});
    } else {
        if (small_index) f(double{}, int{});
        else f(double{}, (long long){});
    }
}

// every field of the launch has fewer than 2^31 elements
bool fits_int(const DField &f) { return f.n0 * f.n1 * f.n2 < 0x7fffffffLL; }

// An offset of exactly +0.0 (a -0.0 offset changes idx + offset for idx = -0.0)
bool zero_offset(double o) { return o == 0.0 && !std::signbit(o); }

// Fill r.geo: whether the fields have the ROMS geometry (DGeom) and its sizes.
void set_geometry(DRoms &r) {
    DGeom &g = r.geo;
    g.nz = r.u.n0;
    g.ny = r.u.n1;
    g.nx = r.v.n2;
    g.roms = 0;
    g.w_centered = 0;
    const long long nz = g.nz, ny = g.ny, nx = g.nx;
    g.su0 = ny * (nx - 1);
    g.sv0 = (ny - 1) * nx;
    g.sw0 = ny * nx;
    auto is3 = [](const DField &f, long long a, long long b, long long c, double oa, double ob, double oc) {
        return f.n0 == a && f.n1 == b && f.n2 == c && f.o0 == oa && f.o1 == ob && f.o2 == oc &&
               (oa != 0.0 || zero_offset(f.o0)) && (ob != 0.0 || zero_offset(f.o1)) &&
               (oc != 0.0 || zero_offset(f.o2));
    };
    auto is2 = [&](const DField &f) {
        return f.n0 == ny && f.n1 == nx && f.n2 == 1 && zero_offset(f.o0) && zero_offset(f.o1);
    };
    if (!is3(r.u, nz, ny, nx - 1, 0.0, 0.0, -0.5) || !is3(r.v, nz, ny - 1, nx, 0.0, -0.5, 0.0)) return;
    if (!is2(r.zeta) || !is2(r.h) || !is2(r.dx) || !is2(r.dy)) return;
    if (!(r.C.n0 == nz && r.C.n1 == 1 && r.C.n2 == 1 && zero_offset(r.C.o0))) return;
    if (is3(r.w, nz + 1, ny, nx, 0.5, 0.0, 0.0)) {
        g.roms = 1;
    } else if (is3(r.w, nz, ny, nx, 0.0, 0.0, 0.0)) {
        g.roms = 1;
        g.w_centered = 1;
    }
}

// u, v, w, zeta time-dependent and h, dx, dy, C static, in the ROMS geometry
// (DGeom; `w_centered`: the w slot on rho points, as the isopycnal follower
// has it): the layout the ROMS presets use, compiled with the field kinds and
// the geometry fixed
bool roms_layout(const DRoms &r, bool w_centered = false) {
    return !r.u.is_static && !r.v.is_static && !r.w.is_static && !r.zeta.is_static && r.h.is_static &&
           r.dx.is_static && r.dy.is_static && r.C.is_static && r.geo.roms && (r.geo.w_centered != 0) == w_centered;
}

bool fits_int(const DRoms &r) {
    return fits_int(r.u) && fits_int(r.v) && fits_int(r.w) && fits_int(r.dx) && fits_int(r.dy) && fits_int(r.h) &&
           fits_int(r.zeta) && fits_int(r.C);
}

// ---------------------------------------------------------------- host side
int check_launch(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    clear_error();
    return OPB_OK;
}

unsigned grid_for(long long n) { return (unsigned)((n + kHostBlock - 1) / kHostBlock); }

// CTAs of `kernel` that stay resident on the whole device (SMs x blocks per SM),
// cached per (kernel, device)
int resident_ctas(const void *kernel, int block) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, int> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find({kernel, dev});
    if (it != cache.end()) return it->second;
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess) return 0;
    const int g = sms * (per_sm > 0 ? per_sm : 1);
    cache[{kernel, dev}] = g;
    return g;
}

int convert_particles(const opb_particles *in, DParticles &out, const char *what, bool need_positions) {
    if (!in) return fail(OPB_EINVAL, "%s: particles is NULL", what);
    if (in->n < 0) return fail(OPB_EINVAL, "%s: negative particle count", what);
    if (in->n > 0 && !in->status) return fail(OPB_EINVAL, "%s: status is NULL", what);
    if (in->n > 0 && need_positions && (!in->zidx || !in->yidx || !in->xidx))
        return fail(OPB_EINVAL, "%s: zidx/yidx/xidx is NULL", what);
    if ((long long)grid_for(in->n) > 0x7fffffffLL) return fail(OPB_EINVAL, "%s: too many particles", what);
    out.n = in->n;
    out.status = in->status;
    out.zidx = in->zidx;
    out.yidx = in->yidx;
    out.xidx = in->xidx;
    out.z = in->z;
    out.dxidx0 = in->dxidx0;
    out.dyidx0 = in->dyidx0;
    out.dz0 = in->dz0;
    out.dxidx1 = in->dxidx1;
    out.dyidx1 = in->dyidx1;
    out.dz1 = in->dz1;
    out.dxidx2 = in->dxidx2;
    out.dyidx2 = in->dyidx2;
    out.dz2 = in->dz2;
    out.err = in->err;
    out.rho_t = in->rho_t;
    return OPB_OK;
}

void convert_scalars(const opb_scalars *in, DScalars &out) {
    out.hc = in->hc;
    out.NZ = in->NZ;
    out.dt = in->dt;
    out.alpha = in->alpha;
    for (int k = 0; k < 6; ++k) out.bounds[k] = in->bounds[k];
    out.w_max = in->w_max;
    out.rho_scale = in->rho_scale;
}

int convert_field(const opb_field &in, DField &out, int ndim, const char *what, const char *name, int *dtype) {
    if (in.ndim != ndim)
        return fail(OPB_EINVAL, "%s: field '%s' has %d active dimensions, expected %d", what, name, in.ndim, ndim);
    long long n[3] = {1, 1, 1};
    for (int d = 0; d < ndim; ++d) {
        if (in.shape[d] < 2)
            return fail(OPB_EINVAL, "%s: field '%s' dimension %d has size %lld (< 2)", what, name, d,
                        (long long)in.shape[d]);
        n[d] = in.shape[d];
    }
    if (in.is_static) {
        if (!in.data[0]) return fail(OPB_EINVAL, "%s: field '%s' has no data", what, name);
        if (in.dtype != OPB_F64) return fail(OPB_EINVAL, "%s: static field '%s' must be float64", what, name);
    } else {
        if (in.nslots < 2 || in.nslots > OPB_MAX_SLOTS)
            return fail(OPB_EINVAL, "%s: field '%s' has %d snapshot slots", what, name, in.nslots);
        for (int k = 0; k < in.nslots; ++k)
            if (!in.data[k]) return fail(OPB_EINVAL, "%s: field '%s' slot %d is NULL", what, name, k);
        if (in.dtype != OPB_F64 && in.dtype != OPB_F32)
            return fail(OPB_EINVAL, "%s: field '%s' has unsupported dtype %d", what, name, in.dtype);
        if (*dtype < 0) *dtype = in.dtype;
        else if (*dtype != in.dtype)
            return fail(OPB_EINVAL, "%s: time-dependent fields must share one storage dtype", what);
    }
    for (int k = 0; k < OPB_MAX_SLOTS; ++k) out.data[k] = in.data[k];
    out.n0 = n[0];
    out.n1 = n[1];
    out.n2 = n[2];
    out.o0 = in.offset[0];
    out.o1 = ndim > 1 ? in.offset[1] : 0.0;
    out.o2 = ndim > 2 ? in.offset[2] : 0.0;
    out.is_static = in.is_static;
    return OPB_OK;
}

// `need_velocity`: u, v, w, dx, dy are read (not by update / post / compute_z)
int convert_fields(const opb_roms_fields *in, DRoms &out, const char *what, bool need_velocity, int *dtype) {
    if (!in) return fail(OPB_EINVAL, "%s: fields is NULL", what);
    *dtype = -1;
    int rc;
    if (need_velocity) {
        if ((rc = convert_field(in->u, out.u, 3, what, "u", dtype))) return rc;
        if ((rc = convert_field(in->v, out.v, 3, what, "v", dtype))) return rc;
        if ((rc = convert_field(in->w, out.w, 3, what, "w", dtype))) return rc;
        if ((rc = convert_field(in->dx, out.dx, 2, what, "dx", dtype))) return rc;
        if ((rc = convert_field(in->dy, out.dy, 2, what, "dy", dtype))) return rc;
    } else {
        memset(&out.u, 0, sizeof(DField));
        out.u.is_static = 1;
        out.v = out.w = out.dx = out.dy = out.u;
    }
    if ((rc = convert_field(in->h, out.h, 2, what, "h", dtype))) return rc;
    if ((rc = convert_field(in->zeta, out.zeta, 2, what, "zeta", dtype))) return rc;
    if ((rc = convert_field(in->C, out.C, 1, what, "C", dtype))) return rc;
    if (!in->C.is_static) return fail(OPB_EINVAL, "%s: field 'C' must be static", what);
    if (*dtype < 0) *dtype = OPB_F64;  // every field static
    memset(&out.geo, 0, sizeof(DGeom));
    if (need_velocity) set_geometry(out);
    return OPB_OK;
}

int check_time(const opb_time *t, const opb_roms_fields *f, const char *what) {
    if (!t) return fail(OPB_EINVAL, "%s: time is NULL", what);
    const opb_field *all[] = {&f->u, &f->v, &f->w, &f->zeta, &f->h, &f->dx, &f->dy};
    for (const opb_field *x : all) {
        if (x->is_static) continue;
        if (t->prev < 0 || t->prev >= x->nslots || t->next < 0 || t->next >= x->nslots)
            return fail(OPB_EINVAL, "%s: snapshot slot out of range", what);
    }
    return OPB_OK;
}

int stage_common(const char *what, const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                 const opb_time *t, bool need_velocity, DParticles &dp, DScalars &ds, DRoms &dr, int &dtype) {
    int rc;
    if ((rc = convert_particles(p, dp, what, true))) return rc;
    if (!s) return fail(OPB_EINVAL, "%s: scalars is NULL", what);
    convert_scalars(s, ds);
    if ((rc = convert_fields(f, dr, what, need_velocity, &dtype))) return rc;
    if ((rc = check_time(t, f, what))) return rc;
    return OPB_OK;
}

// Time-dependent fields may come as snapshot pairs (OPB_F32_PAIRS / OPB_F64_PAIRS), snapshot quads
// (OPB_F32_QUADS, with h, dx, dy as OPB_F64_XPAIRS) or snapshot octets (OPB_F32_OCTS, with h, dx, dy as
// OPB_F64_YXPAIRS), and the 2-D fields as bundles (zeta with h, dx with dy; float32 pairs or quads):
// `out` is `in` with the element dtypes, `layout` says which form it was (LAYOUT_PLAIN, LAYOUT_PAIRS,
// LAYOUT_QUADS, LAYOUT_OCTS) and `bundled` whether the 2-D fields are bundled.  All of u, v, w, zeta or
// none.
int unpair_fields(const opb_roms_fields *in, opb_roms_fields &out, int &layout, bool &bundled, const char *what) {
    if (!in) return fail(OPB_EINVAL, "%s: fields is NULL", what);
    // every vector load of a layout starts on its own size: the buffers must be aligned to it
    auto misaligned = [](const opb_field &x, uintptr_t align) {
        const int n = x.is_static ? 1 : (x.nslots < OPB_MAX_SLOTS ? x.nslots : OPB_MAX_SLOTS);
        for (int k = 0; k < n; ++k)
            if (((uintptr_t)x.data[k]) & (align - 1)) return true;
        return false;
    };
    for (const opb_field *x : {&in->u, &in->v, &in->w, &in->zeta, &in->h, &in->dx, &in->dy}) {
        const uintptr_t align = x->dtype == OPB_F32_PAIRS                                  ? 8
                                : x->dtype == OPB_F64_PAIRS || x->dtype == OPB_F32_QUADS ||
                                          x->dtype == OPB_F64_XPAIRS                       ? 16
                                : x->dtype == OPB_F32_OCTS || x->dtype == OPB_F64_YXPAIRS ||
                                          x->dtype == OPB_F32_ZETA_H || x->dtype == OPB_F64_DX_DY ? 32
                                                                                           : 1;
        if (align > 1 && misaligned(*x, align))
            return fail(OPB_EINVAL, "%s: a snapshot pair/quad/octet, x/yx-pair or bundle buffer is not %d-byte aligned",
                        what, (int)align);
    }
    out = *in;
    // 2-D bundles: all four codes or none
    const int nb = (in->zeta.dtype == OPB_F32_ZETA_H && !in->zeta.is_static) + (in->h.dtype == OPB_F64_IN_ZETA) +
                   (in->dx.dtype == OPB_F64_DX_DY && in->dx.is_static) + (in->dy.dtype == OPB_F64_IN_DX);
    if (nb != 0 && nb != 4)
        return fail(OPB_EINVAL, "%s: 2-D bundles need zeta as OPB_F32_ZETA_H, h as OPB_F64_IN_ZETA, dx as "
                    "OPB_F64_DX_DY and dy as OPB_F64_IN_DX together", what);
    bundled = nb == 4;
    if (bundled) {
        if (in->h.ndim != in->zeta.ndim || in->h.shape[0] != in->zeta.shape[0] || in->h.shape[1] != in->zeta.shape[1] ||
            in->h.offset[0] != in->zeta.offset[0] || in->h.offset[1] != in->zeta.offset[1] ||
            in->dy.ndim != in->dx.ndim || in->dy.shape[0] != in->dx.shape[0] || in->dy.shape[1] != in->dx.shape[1] ||
            in->dy.offset[0] != in->dx.offset[0] || in->dy.offset[1] != in->dx.offset[1])
            return fail(OPB_EINVAL, "%s: bundled fields must share their shape and offsets (h with zeta, dy with dx)",
                        what);
        out.zeta.dtype = OPB_F32;
        out.h.dtype = out.dx.dtype = out.dy.dtype = OPB_F64;
        // h and dy are read from the bundles: their own buffers are not needed
        if (!out.h.data[0]) out.h.data[0] = in->zeta.data[0];
        if (!out.dy.data[0]) out.dy.data[0] = in->dx.data[0];
    }
    int npairs = 0, nquads = 0, nocts = 0, ntd = 0, nx = 0, nyx = 0;
    for (opb_field *x : {&out.u, &out.v, &out.w, &out.zeta}) {
        if (x->is_static || (bundled && x == &out.zeta)) continue;
        ++ntd;
        if (x->dtype == OPB_F32_PAIRS || x->dtype == OPB_F64_PAIRS) {
            x->dtype = x->dtype == OPB_F32_PAIRS ? OPB_F32 : OPB_F64;
            ++npairs;
        } else if (x->dtype == OPB_F32_QUADS) {
            x->dtype = OPB_F32;
            ++nquads;
        } else if (x->dtype == OPB_F32_OCTS) {
            x->dtype = OPB_F32;
            ++nocts;
        }
    }
    for (opb_field *x : {&out.h, &out.dx, &out.dy}) {
        if (x->is_static && x->dtype == OPB_F64_XPAIRS) {
            x->dtype = OPB_F64;
            ++nx;
        } else if (x->is_static && x->dtype == OPB_F64_YXPAIRS) {
            x->dtype = OPB_F64;
            ++nyx;
        }
    }
    if ((npairs && npairs != ntd) || (nquads && nquads != ntd) || (nocts && nocts != ntd))
        return fail(OPB_EINVAL, "%s: either every time-dependent field is a snapshot pair (or quad, or octet) or none",
                    what);
    if (bundled && !(ntd > 0 && ((npairs == ntd && in->u.dtype == OPB_F32_PAIRS) || nquads == ntd)))
        return fail(OPB_EINVAL, "%s: 2-D bundles come with float32 snapshot pairs or quads of u, v, w", what);
    if (nquads && !bundled && nx != 3)
        return fail(OPB_EINVAL, "%s: snapshot quads need h, dx and dy as static x-pairs (OPB_F64_XPAIRS)", what);
    if (nocts && nyx != 3)
        return fail(OPB_EINVAL, "%s: snapshot octets need h, dx and dy as static yx-pairs (OPB_F64_YXPAIRS)", what);
    if (nx && !nquads)
        return fail(OPB_EINVAL, "%s: static x-pairs (OPB_F64_XPAIRS) come with snapshot quads only", what);
    if (nyx && !nocts)
        return fail(OPB_EINVAL, "%s: static yx-pairs (OPB_F64_YXPAIRS) come with snapshot octets only", what);
    layout = nocts ? LAYOUT_OCTS : nquads ? LAYOUT_QUADS : npairs ? LAYOUT_PAIRS : LAYOUT_PLAIN;
    return OPB_OK;
}

int need_fields(const opb_particles *p, const char *what, std::initializer_list<std::pair<const char *, const void *>> req) {
    if (!p || p->n == 0) return OPB_OK;
    for (auto &kv : req)
        if (!kv.second) return fail(OPB_EINVAL, "%s: particle field %s is NULL", what, kv.first);
    return OPB_OK;
}

}  // namespace
}  // namespace opb
