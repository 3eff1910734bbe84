// Per-particle stage functions shared by the ROMS kernels (opb_roms.cu) and
// the batched-release kernel (opb_batched.cu): the particle state, the fields
// of one stage, the level tables, and one function per reference kernel body.
// Every translation unit that includes this is compiled with -fmad=false
// (bit-identical float64 arithmetic; see opb_device.cuh).
#pragma once

#include <cuda_runtime.h>

#include "opb200.h"
#include "opb_device.cuh"

namespace opb {
namespace {

constexpr int kBlock = 256;

// ------------------------------------------------------------ per particle
struct PState {
    double zidx, yidx, xidx, z;
    double k0x, k0y, k0z;  // AB3 k(n)
    double k1x, k1y, k1z;  // RK2 k1 / AB3 k(n-1)
    double k2x, k2y, k2z;  // RK2 k2 / AB3 k(n-2)
    // h and zeta at (yidx, xidx) for the time selection `at`, left by the
    // previous step's last stage; the next step's first stage needs exactly
    // these values (same position, same time index) and reuses them
    double h_at, zeta_at;
    opb_time at;
    uint8_t status;
};

__device__ __forceinline__ bool same_time(const opb_time &a, const opb_time &b) {
    return a.prev == b.prev && a.next == b.next && a.ft == b.ft && a.gt == b.gt;
}

__device__ __forceinline__ void raise_zero_division(const DParticles &p) {
    if (p.err) atomicOr(p.err, (uint32_t)OPB_ERRF_ZERO_DIVISION);
}

// The fields of one stage.  FIXED: the ROMS layout (u, v, w, zeta
// time-dependent; h, dx, dy, C static), known at compile time; otherwise each
// field's kind is read at run time.  LAYOUT (FIXED only): how the
// time-dependent fields, and with LAYOUT_QUADS / LAYOUT_OCTS the static h, dx,
// dy, are read.
template <typename T, typename I, bool FIXED = false, int LAYOUT = LAYOUT_PLAIN, bool B2 = false>
struct Bound {
    static_assert(FIXED || LAYOUT == LAYOUT_PLAIN, "pair layouts need the ROMS field layout");
    static_assert(!B2 || (LAYOUT != LAYOUT_PLAIN && sizeof(T) == 4), "2-D bundles come with float32 pairs");
    static constexpr int KT = LAYOUT == LAYOUT_OCTS ? KIND_OCTS
                              : LAYOUT == LAYOUT_QUADS ? KIND_QUADS
                              : LAYOUT == LAYOUT_PAIRS ? KIND_PAIRS
                              : FIXED ? KIND_TD : KIND_ANY;
    static constexpr int KS = LAYOUT == LAYOUT_OCTS ? KIND_YXPAIRS
                              : LAYOUT == LAYOUT_QUADS ? KIND_XPAIRS
                              : FIXED ? KIND_STATIC : KIND_ANY;
    static constexpr int KC = FIXED ? KIND_STATIC : KIND_ANY;
    static constexpr bool BUNDLED = B2;
    View<T, I, KT> u, v, w, zeta;
    View<T, I, KS> dx, dy, h;
    View<T, I, KC> C;
    ZetaHView<I> zh;  // B2: zeta with h
    DxDyView<I> dd;   // B2: dx with dy
};

template <typename T, typename I, bool FIXED = false, int LAYOUT = LAYOUT_PLAIN, bool B2 = false>
__device__ __forceinline__ Bound<T, I, FIXED, LAYOUT, B2> bind_all(const DRoms &r, const opb_time &t) {
    using B = Bound<T, I, FIXED, LAYOUT, B2>;
    B b;
    b.u = bind<T, I, B::KT>(r.u, t);
    b.v = bind<T, I, B::KT>(r.v, t);
    b.w = bind<T, I, B::KT>(r.w, t);
    b.C = bind<T, I, B::KC>(r.C, t);  // static float64 (kernels/_core.pyx:5-9)
    if constexpr (B2) {
        b.zh.p = (const U4 *)r.zeta.data[t.prev];
        b.zh.ft = (float)t.ft;  // exact: the host rounded ft, gt to float32
        b.zh.gt = (float)t.gt;
        b.zh.n0 = (I)r.zeta.n0;
        b.zh.n1 = (I)r.zeta.n1;
        b.zh.o0 = r.zeta.o0;
        b.zh.o1 = r.zeta.o1;
        b.dd.p = (const D4 *)r.dx.data[0];
        b.dd.n0 = (I)r.dx.n0;
        b.dd.n1 = (I)r.dx.n1;
        b.dd.o0 = r.dx.o0;
        b.dd.o1 = r.dx.o1;
    } else {
        b.zeta = bind<T, I, B::KT>(r.zeta, t);
        b.dx = bind<T, I, B::KS>(r.dx, t);
        b.dy = bind<T, I, B::KS>(r.dy, t);
        b.h = bind<T, I, B::KS>(r.h, t);
    }
    return b;
}

// h and zeta at (y, x): one stencil for both when they are bundled
template <typename B>
__device__ __forceinline__ void hz_at(const B &f, double y, double x, double &h, double &zeta) {
    if constexpr (B::BUNDLED) {
        bilinear_pair(f.zh, y + f.zh.o0, x + f.zh.o1, h, zeta);
    } else {
        h = bilinear(f.h, y + f.h.o0, x + f.h.o1);
        zeta = bilinear(f.zeta, y + f.zeta.o0, x + f.zeta.o1);
    }
}

// dx and dy at (y, x)
template <typename B>
__device__ __forceinline__ void dxdy_at(const B &f, double y, double x, double &dx, double &dy) {
    if constexpr (B::BUNDLED) {
        bilinear_pair(f.dd, y + f.dd.o0, x + f.dd.o1, dx, dy);
    } else {
        dx = bilinear(f.dx, y + f.dx.o0, x + f.dx.o1);
        dy = bilinear(f.dy, y + f.dy.o0, x + f.dy.o1);
    }
}

// Every kernel starts here, before any thread can return: the block's shared
// tables of the sigma levels (used by compute_zidx).
#define OPB_LEVELS(r, sc)                                                                            \
    __shared__ double s_sigma[kMaxLevels];                                                           \
    __shared__ double s_C[kMaxLevels];                                                               \
    const Levels L = load_levels((const double *)(r).C.data[0], (r).C.n0, (r).C.o0, (sc).NZ, s_sigma, s_C); \
    __syncthreads()

// rk2_w_advection.pyx:97-153 (stage 1 for one particle).  Returns false on a
// zero grid spacing (the reference raises ZeroDivisionError).
template <typename B>
__device__ __forceinline__ bool rk2_stage1(PState &s, const B &f, const DScalars &sc, bool reuse_hz = false) {
    double h, zeta;
    if (reuse_hz) {
        h = s.h_at;
        zeta = s.zeta_at;
    } else {
        hz_at(f, s.yidx, s.xidx, h, zeta);
    }
    const double Cv = linear(f.C, s.zidx + f.C.o0);
    s.z = compute_z(s.zidx, sc.NZ, sc.hc, h, Cv, zeta);
    const double u = trilinear(f.u, s.zidx + f.u.o0, s.yidx + f.u.o1, s.xidx + f.u.o2);
    const double v = trilinear(f.v, s.zidx + f.v.o0, s.yidx + f.v.o1, s.xidx + f.v.o2);
    double dx, dy;
    dxdy_at(f, s.yidx, s.xidx, dx, dy);
    // gathered before the check (pure reads): every stencil's loads are in flight together
    const double w = trilinear(f.w, s.zidx + f.w.o0, s.yidx + f.w.o1, s.xidx + f.w.o2);
    if (dx == 0.0 || dy == 0.0) return false;
    s.k1x = u / dx;
    s.k1y = v / dy;
    s.k1z = w;
    return true;
}

// rk2_w_advection.pyx:225-275 (stage 2 for one particle)
template <typename B>
__device__ __forceinline__ bool rk2_stage2(PState &s, const B &f, const Levels &L, const DScalars &sc) {
    const double adt = sc.alpha * sc.dt;
    const double z_int = s.z + adt * s.k1z;
    const double y_int = s.yidx + adt * s.k1y;
    const double x_int = s.xidx + adt * s.k1x;
    double h, zeta;
    hz_at(f, y_int, x_int, h, zeta);
    const double z_idx = compute_zidx_hint(z_int, h, zeta, sc.hc, L, s.zidx);
    const double u = trilinear(f.u, z_idx + f.u.o0, y_int + f.u.o1, x_int + f.u.o2);
    const double v = trilinear(f.v, z_idx + f.v.o0, y_int + f.v.o1, x_int + f.v.o2);
    double dx, dy;
    dxdy_at(f, y_int, x_int, dx, dy);
    const double w = trilinear(f.w, z_idx + f.w.o0, y_int + f.w.o1, x_int + f.w.o2);
    if (dx == 0.0 || dy == 0.0) return false;
    s.k2x = u / dx;
    s.k2y = v / dy;
    s.k2z = w;
    return true;
}

// rk2_w_advection.pyx:316-354 (update for one particle); b1 = 1/(2 alpha)
// weights k1, the reference's own convention (rk2_w_advection.pyx:317-318).
template <typename B>
__device__ __forceinline__ void rk2_update(PState &s, const B &f, const Levels &L, const DScalars &sc) {
    const double b1 = 1.0 / (2.0 * sc.alpha);
    const double b2 = 1.0 - b1;
    const double b1dt = b1 * sc.dt;
    const double b2dt = b2 * sc.dt;
    s.z = s.z + b1dt * s.k1z + b2dt * s.k2z;
    s.yidx = s.yidx + b1dt * s.k1y + b2dt * s.k2y;
    s.xidx = s.xidx + b1dt * s.k1x + b2dt * s.k2x;
    double h, zeta;
    hz_at(f, s.yidx, s.xidx, h, zeta);
    s.zidx = compute_zidx_hint(s.z, h, zeta, sc.hc, L, s.zidx);
    s.h_at = h;
    s.zeta_at = zeta;
}

// ab3_w_advection.pyx:84-178 (AB3 step for one particle)
// The AB3 step's vertical velocity: the w field (ab3_w_advection.pyx:141-146),
// or the isopycnal follower's w_max * drho / (rho_scale + |drho|) with drho =
// rho(x) - rho_t from the density field in the w slot
// (ab3_isopycnal_following.pyx:124-132).  False on a zero divisor.
// finish(g, k): g is the trilinear value of the w-slot field at the particle.
struct WVel {
    __device__ __forceinline__ bool finish(double g, double &k) const {
        k = g;
        return true;
    }
};

struct IsoVel {
    double rho_t, w_max, rho_scale;
    __device__ __forceinline__ bool finish(double rho, double &k) const {
        const double drho = rho - rho_t;
        const double den = rho_scale + fabs(drho);
        if (den == 0.0) return false;
        k = w_max * drho / den;
        return true;
    }
};

template <typename B, typename VZ = WVel>
__device__ __forceinline__ bool ab3_step(PState &s, const B &f, const DScalars &sc, bool reuse_hz = false,
                                         const VZ &vz = VZ{}) {
    // every gather first (pure reads, so their loads are in flight together), then the divisions and
    // their zero checks in the reference's order: dx, dy, then the vertical velocity's
    const double u = trilinear(f.u, s.zidx + f.u.o0, s.yidx + f.u.o1, s.xidx + f.u.o2);
    double dx, dy;
    dxdy_at(f, s.yidx, s.xidx, dx, dy);
    const double v = trilinear(f.v, s.zidx + f.v.o0, s.yidx + f.v.o1, s.xidx + f.v.o2);
    const double wg = trilinear(f.w, s.zidx + f.w.o0, s.yidx + f.w.o1, s.xidx + f.w.o2);
    if (dx == 0.0) return false;
    s.k0x = u / dx;
    if (dy == 0.0) return false;
    s.k0y = v / dy;
    if (!vz.finish(wg, s.k0z)) return false;
    if (s.status == ST_MULTISTEP_1) {  // ab3_w_advection.pyx:122-131
        s.k1x = s.k0x;
        s.k1y = s.k0y;
        s.k1z = s.k0z;
        s.k2x = s.k0x;
        s.k2y = s.k0y;
        s.k2z = s.k0z;
        s.status = ST_MULTISTEP_2;
    } else if (s.status == ST_MULTISTEP_2) {  // ab3_w_advection.pyx:132-138
        s.k2x = -s.k0x + 2.0 * s.k1x;
        s.k2y = -s.k0y + 2.0 * s.k1y;
        s.k2z = -s.k0z + 2.0 * s.k1z;
        s.status = ST_NORMAL;
    }
    double h, zeta;
    if (reuse_hz) {
        h = s.h_at;
        zeta = s.zeta_at;
    } else {
        hz_at(f, s.yidx, s.xidx, h, zeta);
    }
    const double Cv = linear(f.C, s.zidx + f.C.o0);
    s.z = compute_z(s.zidx, sc.NZ, sc.hc, h, Cv, zeta);
    const double dt = sc.dt;
    s.z = s.z + dt * (23.0 * s.k0z - 16.0 * s.k1z + 5.0 * s.k2z) / 12.0;
    s.yidx = s.yidx + dt * (23.0 * s.k0y - 16.0 * s.k1y + 5.0 * s.k2y) / 12.0;
    s.xidx = s.xidx + dt * (23.0 * s.k0x - 16.0 * s.k1x + 5.0 * s.k2x) / 12.0;
    s.k2z = s.k1z;
    s.k2x = s.k1x;
    s.k2y = s.k1y;
    s.k1z = s.k0z;
    s.k1x = s.k0x;
    s.k1y = s.k0y;
    return true;
}

// ab3_w_advection.pyx:214-229 (post step for one particle)
template <typename B>
__device__ __forceinline__ void ab3_post(PState &s, const B &f, const Levels &L, const DScalars &sc) {
    double h, zeta;
    hz_at(f, s.yidx, s.xidx, h, zeta);
    s.zidx = compute_zidx_hint(s.z, h, zeta, sc.hc, L, s.zidx);
    s.h_at = h;
    s.zeta_at = zeta;
}

__device__ __forceinline__ long long gtid() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }

}  // namespace
}  // namespace opb
