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
// HS: the velocity history (RK2 k1, k2 / AB3 k(n-1), k(n-2)) lives in this
// thread's column of a [6][block] shared-memory table instead of registers.
// It is read and written once per step, after the stencil gathers, so that
// the registers stay free for the gathers in flight (more resident warps).
template <typename I = long long, bool HS = false>
struct PState {
    double zidx, yidx, xidx, z;
    double k0x, k0y, k0z;  // AB3 k(n)
    double k1x, k1y, k1z;  // RK2 k1 / AB3 k(n-1)  (HS: unused)
    double k2x, k2y, k2z;  // RK2 k2 / AB3 k(n-2)  (HS: unused)
    double *hs;            // HS: this thread's column (entry j at hs[j * hstride])
    int hstride;
    __device__ __forceinline__ void get_k1(double &x, double &y, double &z_) const {
        if constexpr (HS) {
            x = hs[0];
            y = hs[hstride];
            z_ = hs[2 * hstride];
        } else {
            x = k1x;
            y = k1y;
            z_ = k1z;
        }
    }
    __device__ __forceinline__ void get_k2(double &x, double &y, double &z_) const {
        if constexpr (HS) {
            x = hs[3 * hstride];
            y = hs[4 * hstride];
            z_ = hs[5 * hstride];
        } else {
            x = k2x;
            y = k2y;
            z_ = k2z;
        }
    }
    __device__ __forceinline__ void set_k1(double x, double y, double z_) {
        if constexpr (HS) {
            hs[0] = x;
            hs[hstride] = y;
            hs[2 * hstride] = z_;
        } else {
            k1x = x;
            k1y = y;
            k1z = z_;
        }
    }
    __device__ __forceinline__ void set_k2(double x, double y, double z_) {
        if constexpr (HS) {
            hs[3 * hstride] = x;
            hs[4 * hstride] = y;
            hs[5 * hstride] = z_;
        } else {
            k2x = x;
            k2y = y;
            k2z = z_;
        }
    }
    // h and zeta at (yidx, xidx) for the previous step's last time selection,
    // left by its last stage; the next step's first stage needs exactly these
    // values when it selects the same time (same position) and reuses them
    double h_at, zeta_at;
    // compiled ROMS layout: the rho-point stencil axes at (yidx, xidx), left by
    // the previous step's last stage (the position has not moved since)
    Axis<I> ya, xa;
    uint8_t status;
};

__device__ __forceinline__ bool same_time(const opb_time &a, const opb_time &b) {
    return a.prev == b.prev && a.next == b.next && a.ft == b.ft && a.gt == b.gt;
}

__device__ __forceinline__ void raise_zero_division(const DParticles &p) {
    if (p.err) atomicOr(p.err, (uint32_t)OPB_ERRF_ZERO_DIVISION);
}

// The fields of one stage.  FIXED: the ROMS layout (u, v, w, zeta
// time-dependent; h, dx, dy, C static) and the ROMS geometry (DGeom), known at
// compile time; otherwise each field's kind, shape and offsets are read at run
// time.  LAYOUT (FIXED only): how the time-dependent fields, and with
// LAYOUT_QUADS / LAYOUT_OCTS the static h, dx, dy, are read.
template <typename T, typename I, bool FIXED = false, int LAYOUT = LAYOUT_PLAIN, bool B2 = false>
struct Bound {
    static_assert(FIXED || LAYOUT == LAYOUT_PLAIN, "pair layouts need the ROMS field layout");
    static_assert(!B2 || (LAYOUT != LAYOUT_PLAIN && sizeof(T) == 4), "2-D bundles come with float32 pairs");
    using index_type = I;
    static constexpr bool kFixed = FIXED;
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
    I nz, ny, nx;     // FIXED: rho-point sizes (DGeom)
    I su0, sv0, sw0;  // FIXED: level strides of u, v and w (DGeom)
};

template <typename T, typename I, bool FIXED = false, int LAYOUT = LAYOUT_PLAIN, bool B2 = false>
__device__ __forceinline__ Bound<T, I, FIXED, LAYOUT, B2> bind_all(const DRoms &r, const opb_time &t) {
    using B = Bound<T, I, FIXED, LAYOUT, B2>;
    B b;
    b.u = bind<T, I, B::KT>(r.u, t);
    b.v = bind<T, I, B::KT>(r.v, t);
    b.w = bind<T, I, B::KT>(r.w, t);
    b.C = bind<T, I, B::KC>(r.C, t);  // static float64 (kernels/_core.pyx:5-9)
    b.nz = (I)r.geo.nz;
    b.ny = (I)r.geo.ny;
    b.nx = (I)r.geo.nx;
    b.su0 = (I)r.geo.su0;
    b.sv0 = (I)r.geo.sv0;
    b.sw0 = (I)r.geo.sw0;
    if constexpr (B2) {
        b.zh.p = (const U4 *)r.zeta.data[t.prev];
        b.zh.ft = (float)t.ft;  // exact: the host rounded ft, gt to float32
        b.zh.gt = (float)t.gt;
        b.zh.w = blend_weights(b.zh.ft, b.zh.gt);
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

// ---------------------------------------------- compiled ROMS layout: axes
// The stencil axes at one position.  In the ROMS geometry each dimension has
// two kinds of points: rho points (offset 0: u and v in z, u and w in y, v and
// w in x, the 2-D fields, C) and half a cell off (w in z at +0.5, v in y and u
// in x at -0.5).  Each axis is make_axis(idx + offset, n - 2) of the fields on
// those points, exactly what trilinear()/bilinear()/linear() compute for each
// of them, so one evaluation serves them all.
template <typename I>
struct Axes {
    Axis<I> zc, zs, yc, ys, xc, xs;
};

template <typename B, typename I = typename B::index_type>
__device__ __forceinline__ void rho_axes_h(const B &f, double y, double x, Axis<I> &yc, Axis<I> &xc) {
    yc = make_axis(y + 0.0, (I)(f.ny - 2));
    xc = make_axis(x + 0.0, (I)(f.nx - 2));
}

// the remaining axes at (z, y, x) once the rho-point ones in y and x are known;
// W_CENTERED: the w slot sits on rho points and needs no zs
template <bool W_CENTERED, typename B, typename I = typename B::index_type>
__device__ __forceinline__ void other_axes(const B &f, double z, double y, double x, Axes<I> &a) {
    a.zc = make_axis(z + 0.0, (I)(f.nz - 2));
    if constexpr (!W_CENTERED) a.zs = make_axis(z + 0.5, (I)(f.nz - 1));
    a.ys = make_axis(y + -0.5, (I)(f.ny - 3));
    a.xs = make_axis(x + -0.5, (I)(f.nx - 3));
}

// u, v and the w-slot field at the axes' position, and dx, dy
template <bool W_CENTERED, typename B, typename I = typename B::index_type>
__device__ __forceinline__ void velocity_ax(const B &f, const Axes<I> &a, double &u, double &v, double &w, double &dx,
                                            double &dy) {
    const I nx = f.nx;
    u = trilinear_ax(f.u, a.zc, a.yc, a.xs, f.su0, nx - 1);
    if constexpr (B::BUNDLED) {
        bilinear_pair_ax(f.dd, a.yc, a.xc, nx, dx, dy);
    } else {
        dx = bilinear_ax(f.dx, a.yc, a.xc, nx);
        dy = bilinear_ax(f.dy, a.yc, a.xc, nx);
    }
    v = trilinear_ax(f.v, a.zc, a.ys, a.xc, f.sv0, nx);
    if constexpr (W_CENTERED) w = trilinear_ax(f.w, a.zc, a.yc, a.xc, f.sw0, nx);
    else w = trilinear_ax(f.w, a.zs, a.yc, a.xc, f.sw0, nx);
}

// h and zeta on the rho-point axes
template <typename B, typename I = typename B::index_type>
__device__ __forceinline__ void hz_ax(const B &f, const Axis<I> &yc, const Axis<I> &xc, double &h, double &zeta) {
    if constexpr (B::BUNDLED) {
        bilinear_pair_ax(f.zh, yc, xc, f.nx, h, zeta);
    } else {
        h = bilinear_ax(f.h, yc, xc, f.nx);
        zeta = bilinear_ax(f.zeta, yc, xc, f.nx);
    }
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

// h and zeta at the particle's (yidx, xidx), leaving the rho-point axes there
// in the state (compiled layout) for the next stage at this position
template <typename B, typename S>
__device__ __forceinline__ void hz_here(S &s, const B &f, double &h, double &zeta) {
    if constexpr (B::kFixed) {
        rho_axes_h(f, s.yidx, s.xidx, s.ya, s.xa);
        hz_ax(f, s.ya, s.xa, h, zeta);
    } else {
        hz_at(f, s.yidx, s.xidx, h, zeta);
    }
}

// Every kernel starts here, before any thread can return: the block's shared
// tables of the sigma levels (used by compute_zidx and, in the compiled
// layout, by the interpolation of C).
#define OPB_LEVELS(r, sc)                                                                            \
    __shared__ double s_sigma[kMaxLevels];                                                           \
    __shared__ double s_C[kMaxLevels];                                                               \
    const Levels L = load_levels((const double *)(r).C.data[0], (r).C.n0, (r).C.o0, (sc).NZ, s_sigma, s_C); \
    __syncthreads()

// C at z on the rho-point axis (compiled layout: C has nz levels at offset 0)
template <typename B, typename I = typename B::index_type>
__device__ __forceinline__ double C_ax(const B &f, const Levels &L, const Axis<I> &zc) {
    return linear_ax(L.C, zc);
}

// rk2_w_advection.pyx:97-153 (stage 1 for one particle).  Returns false on a
// zero grid spacing (the reference raises ZeroDivisionError).  `carried`: the
// state's rho-point axes describe the current position (compiled layout);
// `reuse_hz`: so do h_at and zeta_at, for this stage's time selection.
template <typename B, typename S>
__device__ __forceinline__ bool rk2_stage1(S &s, const B &f, const DScalars &sc, const Levels &L,
                                           bool reuse_hz = false, bool carried = false) {
    double h, zeta, u, v, w, dx, dy;
    if constexpr (B::kFixed) {
        using I = typename B::index_type;
        Axes<I> a;
        if (!carried) rho_axes_h(f, s.yidx, s.xidx, s.ya, s.xa);
        a.yc = s.ya;
        a.xc = s.xa;
        other_axes<false>(f, s.zidx, s.yidx, s.xidx, a);
        if (reuse_hz) {
            h = s.h_at;
            zeta = s.zeta_at;
        } else {
            hz_ax(f, a.yc, a.xc, h, zeta);
        }
        const double Cv = C_ax(f, L, a.zc);
        s.z = compute_z(s.zidx, sc.NZ, sc.hc, h, Cv, zeta);
        velocity_ax<false>(f, a, u, v, w, dx, dy);
    } else {
        if (reuse_hz) {
            h = s.h_at;
            zeta = s.zeta_at;
        } else {
            hz_at(f, s.yidx, s.xidx, h, zeta);
        }
        const double Cv = linear(f.C, s.zidx + f.C.o0);
        s.z = compute_z(s.zidx, sc.NZ, sc.hc, h, Cv, zeta);
        u = trilinear(f.u, s.zidx + f.u.o0, s.yidx + f.u.o1, s.xidx + f.u.o2);
        v = trilinear(f.v, s.zidx + f.v.o0, s.yidx + f.v.o1, s.xidx + f.v.o2);
        dxdy_at(f, s.yidx, s.xidx, dx, dy);
        // gathered before the check (pure reads): every stencil's loads are in flight together
        w = trilinear(f.w, s.zidx + f.w.o0, s.yidx + f.w.o1, s.xidx + f.w.o2);
    }
    if (dx == 0.0 || dy == 0.0) return false;
    s.set_k1(u / dx, v / dy, w);
    return true;
}

// rk2_w_advection.pyx:225-275 (stage 2 for one particle)
template <typename B, typename S>
__device__ __forceinline__ bool rk2_stage2(S &s, const B &f, const Levels &L, const DScalars &sc) {
    const double adt = sc.alpha * sc.dt;
    double k1x, k1y, k1z;
    s.get_k1(k1x, k1y, k1z);
    const double z_int = s.z + adt * k1z;
    const double y_int = s.yidx + adt * k1y;
    const double x_int = s.xidx + adt * k1x;
    double h, zeta, u, v, w, dx, dy;
    if constexpr (B::kFixed) {
        using I = typename B::index_type;
        Axes<I> a;
        rho_axes_h(f, y_int, x_int, a.yc, a.xc);
        hz_ax(f, a.yc, a.xc, h, zeta);
        const double z_idx = compute_zidx_hint(z_int, h, zeta, sc.hc, L, s.zidx);
        other_axes<false>(f, z_idx, y_int, x_int, a);
        velocity_ax<false>(f, a, u, v, w, dx, dy);
    } else {
        hz_at(f, y_int, x_int, h, zeta);
        const double z_idx = compute_zidx_hint(z_int, h, zeta, sc.hc, L, s.zidx);
        u = trilinear(f.u, z_idx + f.u.o0, y_int + f.u.o1, x_int + f.u.o2);
        v = trilinear(f.v, z_idx + f.v.o0, y_int + f.v.o1, x_int + f.v.o2);
        dxdy_at(f, y_int, x_int, dx, dy);
        w = trilinear(f.w, z_idx + f.w.o0, y_int + f.w.o1, x_int + f.w.o2);
    }
    if (dx == 0.0 || dy == 0.0) return false;
    s.set_k2(u / dx, v / dy, w);
    return true;
}

// rk2_w_advection.pyx:316-354 (update for one particle); b1 = 1/(2 alpha)
// weights k1, the reference's own convention (rk2_w_advection.pyx:317-318).
template <typename B, typename S>
__device__ __forceinline__ void rk2_update(S &s, const B &f, const Levels &L, const DScalars &sc) {
    const double b1 = 1.0 / (2.0 * sc.alpha);
    const double b2 = 1.0 - b1;
    const double b1dt = b1 * sc.dt;
    const double b2dt = b2 * sc.dt;
    double k1x, k1y, k1z, k2x, k2y, k2z;
    s.get_k1(k1x, k1y, k1z);
    s.get_k2(k2x, k2y, k2z);
    s.z = s.z + b1dt * k1z + b2dt * k2z;
    s.yidx = s.yidx + b1dt * k1y + b2dt * k2y;
    s.xidx = s.xidx + b1dt * k1x + b2dt * k2x;
    double h, zeta;
    hz_here(s, f, h, zeta);
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
// kCentered: the w-slot field sits on rho points (density) rather than on w
// levels.
struct WVel {
    static constexpr bool kCentered = false;
    __device__ __forceinline__ bool finish(double g, double &k) const {
        k = g;
        return true;
    }
};

struct IsoVel {
    static constexpr bool kCentered = true;
    double rho_t, w_max, rho_scale;
    __device__ __forceinline__ bool finish(double rho, double &k) const {
        const double drho = rho - rho_t;
        const double den = rho_scale + fabs(drho);
        if (den == 0.0) return false;
        k = w_max * drho / den;
        return true;
    }
};

template <typename B, typename S, typename VZ = WVel>
__device__ __forceinline__ bool ab3_step(S &s, const B &f, const DScalars &sc, const Levels &L, bool reuse_hz = false,
                                         bool carried = false, const VZ &vz = VZ{}) {
    // every gather first (pure reads, so their loads are in flight together), then the divisions and
    // their zero checks in the reference's order: dx, dy, then the vertical velocity's
    double u, v, wg, dx, dy, h, zeta, Cv;
    if constexpr (B::kFixed) {
        using I = typename B::index_type;
        Axes<I> a;
        if (!carried) rho_axes_h(f, s.yidx, s.xidx, s.ya, s.xa);
        a.yc = s.ya;
        a.xc = s.xa;
        other_axes<VZ::kCentered>(f, s.zidx, s.yidx, s.xidx, a);
        velocity_ax<VZ::kCentered>(f, a, u, v, wg, dx, dy);
        if (reuse_hz) {
            h = s.h_at;
            zeta = s.zeta_at;
        } else {
            hz_ax(f, a.yc, a.xc, h, zeta);
        }
        Cv = C_ax(f, L, a.zc);
    } else {
        u = trilinear(f.u, s.zidx + f.u.o0, s.yidx + f.u.o1, s.xidx + f.u.o2);
        dxdy_at(f, s.yidx, s.xidx, dx, dy);
        v = trilinear(f.v, s.zidx + f.v.o0, s.yidx + f.v.o1, s.xidx + f.v.o2);
        wg = trilinear(f.w, s.zidx + f.w.o0, s.yidx + f.w.o1, s.xidx + f.w.o2);
    }
    if (dx == 0.0) return false;
    s.k0x = u / dx;
    if (dy == 0.0) return false;
    s.k0y = v / dy;
    if (!vz.finish(wg, s.k0z)) return false;
    double k1x, k1y, k1z, k2x, k2y, k2z;
    s.get_k1(k1x, k1y, k1z);
    s.get_k2(k2x, k2y, k2z);
    if (s.status == ST_MULTISTEP_1) {  // ab3_w_advection.pyx:122-131
        k1x = s.k0x;
        k1y = s.k0y;
        k1z = s.k0z;
        k2x = s.k0x;
        k2y = s.k0y;
        k2z = s.k0z;
        s.status = ST_MULTISTEP_2;
    } else if (s.status == ST_MULTISTEP_2) {  // ab3_w_advection.pyx:132-138
        k2x = -s.k0x + 2.0 * k1x;
        k2y = -s.k0y + 2.0 * k1y;
        k2z = -s.k0z + 2.0 * k1z;
        s.status = ST_NORMAL;
    }
    if constexpr (!B::kFixed) {
        if (reuse_hz) {
            h = s.h_at;
            zeta = s.zeta_at;
        } else {
            hz_at(f, s.yidx, s.xidx, h, zeta);
        }
        Cv = linear(f.C, s.zidx + f.C.o0);
    }
    s.z = compute_z(s.zidx, sc.NZ, sc.hc, h, Cv, zeta);
    const double dt = sc.dt;
    // ab3_w_advection.pyx:168-170: (dt * (...)) / 12.0, the quotient through div12 (the same bits)
    s.z = s.z + div12(dt * (23.0 * s.k0z - 16.0 * k1z + 5.0 * k2z));
    s.yidx = s.yidx + div12(dt * (23.0 * s.k0y - 16.0 * k1y + 5.0 * k2y));
    s.xidx = s.xidx + div12(dt * (23.0 * s.k0x - 16.0 * k1x + 5.0 * k2x));
    s.set_k2(k1x, k1y, k1z);
    s.set_k1(s.k0x, s.k0y, s.k0z);
    return true;
}

// ab3_w_advection.pyx:214-229 (post step for one particle)
template <typename B, typename S>
__device__ __forceinline__ void ab3_post(S &s, const B &f, const Levels &L, const DScalars &sc) {
    double h, zeta;
    hz_here(s, f, h, zeta);
    s.zidx = compute_zidx_hint(s.z, h, zeta, sc.hc, L, s.zidx);
    s.h_at = h;
    s.zeta_at = zeta;
}

__device__ __forceinline__ long long gtid() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }

}  // namespace
}  // namespace opb
