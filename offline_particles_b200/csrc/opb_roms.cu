// ROMS particle-advection kernels for B200 (sm_100a) and their C ABI.
//
// One thread per particle.  Stage kernels map 1:1 onto the reference's
// kernel functions; the fused kernels run whole RK2 / AB3 steps -- and
// several of them per launch -- with the particle state held in registers,
// reading the state once and writing it once per launch.  Compiled with
// -fmad=false: see opb_device.cuh.
#include <cuda_runtime.h>

#include <map>
#include <mutex>

#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <string>
#include <utility>

#include "opb200.h"
#include "opb_device.cuh"
#include "opb_errors.h"

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
// field's kind is read at run time.
template <typename T, typename I, bool FIXED = false>
struct Bound {
    static constexpr int KT = FIXED ? KIND_TD : KIND_ANY;
    static constexpr int KS = FIXED ? KIND_STATIC : KIND_ANY;
    View<T, I, KT> u, v, w, zeta;
    View<T, I, KS> dx, dy, h, C;
};

template <typename T, typename I, bool FIXED = false>
__device__ __forceinline__ Bound<T, I, FIXED> bind_all(const DRoms &r, const opb_time &t) {
    using B = Bound<T, I, FIXED>;
    B b;
    b.u = bind<T, I, B::KT>(r.u, t);
    b.v = bind<T, I, B::KT>(r.v, t);
    b.w = bind<T, I, B::KT>(r.w, t);
    b.zeta = bind<T, I, B::KT>(r.zeta, t);
    b.dx = bind<T, I, B::KS>(r.dx, t);
    b.dy = bind<T, I, B::KS>(r.dy, t);
    b.h = bind<T, I, B::KS>(r.h, t);
    b.C = bind<T, I, B::KS>(r.C, t);  // static float64 (kernels/_core.pyx:5-9)
    return b;
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
    const double h = reuse_hz ? s.h_at : bilinear(f.h, s.yidx + f.h.o0, s.xidx + f.h.o1);
    const double zeta = reuse_hz ? s.zeta_at : bilinear(f.zeta, s.yidx + f.zeta.o0, s.xidx + f.zeta.o1);
    const double Cv = linear(f.C, s.zidx + f.C.o0);
    s.z = compute_z(s.zidx, sc.NZ, sc.hc, h, Cv, zeta);
    const double u = trilinear(f.u, s.zidx + f.u.o0, s.yidx + f.u.o1, s.xidx + f.u.o2);
    const double v = trilinear(f.v, s.zidx + f.v.o0, s.yidx + f.v.o1, s.xidx + f.v.o2);
    const double dx = bilinear(f.dx, s.yidx + f.dx.o0, s.xidx + f.dx.o1);
    const double dy = bilinear(f.dy, s.yidx + f.dy.o0, s.xidx + f.dy.o1);
    if (dx == 0.0 || dy == 0.0) return false;
    s.k1x = u / dx;
    s.k1y = v / dy;
    s.k1z = trilinear(f.w, s.zidx + f.w.o0, s.yidx + f.w.o1, s.xidx + f.w.o2);
    return true;
}

// rk2_w_advection.pyx:225-275 (stage 2 for one particle)
template <typename B>
__device__ __forceinline__ bool rk2_stage2(PState &s, const B &f, const Levels &L, const DScalars &sc) {
    const double adt = sc.alpha * sc.dt;
    const double z_int = s.z + adt * s.k1z;
    const double y_int = s.yidx + adt * s.k1y;
    const double x_int = s.xidx + adt * s.k1x;
    const double h = bilinear(f.h, y_int + f.h.o0, x_int + f.h.o1);
    const double zeta = bilinear(f.zeta, y_int + f.zeta.o0, x_int + f.zeta.o1);
    const double z_idx = compute_zidx_hint(z_int, h, zeta, sc.hc, L, s.zidx);
    const double u = trilinear(f.u, z_idx + f.u.o0, y_int + f.u.o1, x_int + f.u.o2);
    const double v = trilinear(f.v, z_idx + f.v.o0, y_int + f.v.o1, x_int + f.v.o2);
    const double dx = bilinear(f.dx, y_int + f.dx.o0, x_int + f.dx.o1);
    const double dy = bilinear(f.dy, y_int + f.dy.o0, x_int + f.dy.o1);
    if (dx == 0.0 || dy == 0.0) return false;
    s.k2x = u / dx;
    s.k2y = v / dy;
    s.k2z = trilinear(f.w, z_idx + f.w.o0, y_int + f.w.o1, x_int + f.w.o2);
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
    const double h = bilinear(f.h, s.yidx + f.h.o0, s.xidx + f.h.o1);
    const double zeta = bilinear(f.zeta, s.yidx + f.zeta.o0, s.xidx + f.zeta.o1);
    s.zidx = compute_zidx_hint(s.z, h, zeta, sc.hc, L, s.zidx);
    s.h_at = h;
    s.zeta_at = zeta;
}

// ab3_w_advection.pyx:84-178 (AB3 step for one particle)
template <typename B>
__device__ __forceinline__ bool ab3_step(PState &s, const B &f, const DScalars &sc, bool reuse_hz = false) {
    const double u = trilinear(f.u, s.zidx + f.u.o0, s.yidx + f.u.o1, s.xidx + f.u.o2);
    const double dx = bilinear(f.dx, s.yidx + f.dx.o0, s.xidx + f.dx.o1);
    if (dx == 0.0) return false;
    s.k0x = u / dx;
    const double v = trilinear(f.v, s.zidx + f.v.o0, s.yidx + f.v.o1, s.xidx + f.v.o2);
    const double dy = bilinear(f.dy, s.yidx + f.dy.o0, s.xidx + f.dy.o1);
    if (dy == 0.0) return false;
    s.k0y = v / dy;
    s.k0z = trilinear(f.w, s.zidx + f.w.o0, s.yidx + f.w.o1, s.xidx + f.w.o2);
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
    const double h = reuse_hz ? s.h_at : bilinear(f.h, s.yidx + f.h.o0, s.xidx + f.h.o1);
    const double zeta = reuse_hz ? s.zeta_at : bilinear(f.zeta, s.yidx + f.zeta.o0, s.xidx + f.zeta.o1);
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
    const double h = bilinear(f.h, s.yidx + f.h.o0, s.xidx + f.h.o1);
    const double zeta = bilinear(f.zeta, s.yidx + f.zeta.o0, s.xidx + f.zeta.o1);
    s.zidx = compute_zidx_hint(s.z, h, zeta, sc.hc, L, s.zidx);
    s.h_at = h;
    s.zeta_at = zeta;
}

__device__ __forceinline__ long long gtid() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }

// ------------------------------------------------------------ stage kernels
__global__ void __launch_bounds__(kBlock) k_validation(const __grid_constant__ DParticles p,
                                                       const __grid_constant__ DScalars sc, int finite, int bounds) {
    const long long i = gtid();
    if (i >= p.n) return;
    const uint8_t st = p.status[i];
    if (st & ST_INACTIVE) return;
    const double zi = p.zidx[i], yi = p.yidx[i], xi = p.xidx[i];
    uint8_t out = st;
    if (finite && (!is_finite(zi) || !is_finite(yi) || !is_finite(xi))) out = ST_NONFINITE;
    if (bounds && !(out & ST_INACTIVE)) out = validate(out, zi, yi, xi, sc.bounds);
    if (out != st) p.status[i] = out;
}

template <typename T, typename I>
__global__ void __launch_bounds__(kBlock) k_compute_z(const __grid_constant__ DParticles p, double *out,
                                                      const __grid_constant__ DScalars sc,
                                                      const __grid_constant__ DRoms r, opb_time t) {
    const long long i = gtid();
    if (i >= p.n || (p.status[i] & ST_INACTIVE)) return;
    const Bound<T, I> f = bind_all<T, I>(r, t);
    const double yi = p.yidx[i], xi = p.xidx[i], zi = p.zidx[i];
    const double h = bilinear(f.h, yi + f.h.o0, xi + f.h.o1);
    const double zeta = bilinear(f.zeta, yi + f.zeta.o0, xi + f.zeta.o1);
    const double Cv = linear(f.C, zi + f.C.o0);
    out[i] = compute_z(zi, sc.NZ, sc.hc, h, Cv, zeta);
}

template <typename T, typename I>
__global__ void __launch_bounds__(kBlock) k_rk2_step_1(const __grid_constant__ DParticles p,
                                                       const __grid_constant__ DScalars sc,
                                                       const __grid_constant__ DRoms r, opb_time t) {
    const long long i = gtid();
    if (i >= p.n || (p.status[i] & ST_INACTIVE)) return;
    PState s;
    s.zidx = p.zidx[i];
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    const bool ok = rk2_stage1(s, bind_all<T, I>(r, t), sc);
    p.z[i] = s.z;
    if (!ok) {
        raise_zero_division(p);
        return;
    }
    p.dxidx1[i] = s.k1x;
    p.dyidx1[i] = s.k1y;
    p.dz1[i] = s.k1z;
}

template <typename T, typename I>
__global__ void __launch_bounds__(kBlock) k_rk2_step_2(const __grid_constant__ DParticles p,
                                                       const __grid_constant__ DScalars sc,
                                                       const __grid_constant__ DRoms r, opb_time t) {
    OPB_LEVELS(r, sc);
    const long long i = gtid();
    if (i >= p.n || (p.status[i] & ST_INACTIVE)) return;
    PState s;
    s.zidx = p.zidx[i];  // hint for the vertical search
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    s.z = p.z[i];
    s.k1x = p.dxidx1[i];
    s.k1y = p.dyidx1[i];
    s.k1z = p.dz1[i];
    if (!rk2_stage2(s, bind_all<T, I>(r, t), L, sc)) {
        raise_zero_division(p);
        return;
    }
    p.dxidx2[i] = s.k2x;
    p.dyidx2[i] = s.k2y;
    p.dz2[i] = s.k2z;
}

template <typename T, typename I>
__global__ void __launch_bounds__(kBlock) k_rk2_update(const __grid_constant__ DParticles p,
                                                       const __grid_constant__ DScalars sc,
                                                       const __grid_constant__ DRoms r, opb_time t) {
    OPB_LEVELS(r, sc);
    const long long i = gtid();
    if (i >= p.n || (p.status[i] & ST_INACTIVE)) return;
    PState s;
    s.zidx = p.zidx[i];
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    s.z = p.z[i];
    s.k1x = p.dxidx1[i];
    s.k1y = p.dyidx1[i];
    s.k1z = p.dz1[i];
    s.k2x = p.dxidx2[i];
    s.k2y = p.dyidx2[i];
    s.k2z = p.dz2[i];
    rk2_update(s, bind_all<T, I>(r, t), L, sc);
    p.z[i] = s.z;
    p.yidx[i] = s.yidx;
    p.xidx[i] = s.xidx;
    p.zidx[i] = s.zidx;
}

template <typename T, typename I>
__global__ void __launch_bounds__(kBlock) k_ab3(const __grid_constant__ DParticles p,
                                                const __grid_constant__ DScalars sc,
                                                const __grid_constant__ DRoms r, opb_time t) {
    const long long i = gtid();
    if (i >= p.n) return;
    PState s;
    s.status = p.status[i];
    if (s.status & ST_INACTIVE) return;
    s.zidx = p.zidx[i];
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    s.k1x = p.dxidx1[i];
    s.k1y = p.dyidx1[i];
    s.k1z = p.dz1[i];
    s.k2x = p.dxidx2[i];
    s.k2y = p.dyidx2[i];
    s.k2z = p.dz2[i];
    if (!ab3_step(s, bind_all<T, I>(r, t), sc)) {
        raise_zero_division(p);
        return;
    }
    p.status[i] = s.status;
    p.z[i] = s.z;
    p.yidx[i] = s.yidx;
    p.xidx[i] = s.xidx;
    p.dxidx0[i] = s.k1x;  // after the history shift k1 == k0
    p.dyidx0[i] = s.k1y;
    p.dz0[i] = s.k1z;
    p.dxidx1[i] = s.k1x;
    p.dyidx1[i] = s.k1y;
    p.dz1[i] = s.k1z;
    p.dxidx2[i] = s.k2x;
    p.dyidx2[i] = s.k2y;
    p.dz2[i] = s.k2z;
}

template <typename T, typename I>
__global__ void __launch_bounds__(kBlock) k_ab3_post(const __grid_constant__ DParticles p,
                                                     const __grid_constant__ DScalars sc,
                                                     const __grid_constant__ DRoms r, opb_time t) {
    OPB_LEVELS(r, sc);
    const long long i = gtid();
    if (i >= p.n || (p.status[i] & ST_INACTIVE)) return;
    PState s;
    s.zidx = p.zidx[i];  // hint for the vertical search
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    s.z = p.z[i];
    ab3_post(s, bind_all<T, I>(r, t), L, sc);
    p.zidx[i] = s.zidx;
}

// ------------------------------------------------------------ fused kernels
// `nsteps` RK2 steps (timesteppers.py:241-257) per launch.  table[3*k + j]
// selects the fields of step k, stage j (t, t + alpha dt, t + dt).
template <typename T, typename I, bool FIXED>
__global__ void __launch_bounds__(kBlock, 2) k_rk2_steps(const __grid_constant__ DParticles p,
                                                      const __grid_constant__ DScalars sc,
                                                      const __grid_constant__ DRoms r,
                                                      const opb_time *__restrict__ table, int nsteps, int validate_pre) {
    OPB_LEVELS(r, sc);
    const long long i = gtid();
    if (i >= p.n) return;
    PState s;
    s.status = p.status[i];
    if (s.status & ST_INACTIVE) return;
    s.zidx = p.zidx[i];
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    const uint8_t st0 = s.status;
    bool moved = false;
    for (int k = 0; k < nsteps; ++k) {
        if (validate_pre) s.status = validate(s.status, s.zidx, s.yidx, s.xidx, sc.bounds);
        if (s.status & ST_INACTIVE) break;
        const opb_time t1 = table[3 * k], t2 = table[3 * k + 1], t3 = table[3 * k + 2];
        const bool reuse = k > 0 && same_time(t1, s.at);
        if (!rk2_stage1(s, bind_all<T, I, FIXED>(r, t1), sc, reuse)) {
            raise_zero_division(p);
            break;
        }
        moved = true;
        if (!rk2_stage2(s, bind_all<T, I, FIXED>(r, t2), L, sc)) {
            raise_zero_division(p);
            break;
        }
        rk2_update(s, bind_all<T, I, FIXED>(r, t3), L, sc);
        s.at = t3;
    }
    if (s.status != st0) p.status[i] = s.status;
    if (!moved) return;
    p.zidx[i] = s.zidx;
    p.yidx[i] = s.yidx;
    p.xidx[i] = s.xidx;
    p.z[i] = s.z;
    p.dxidx1[i] = s.k1x;
    p.dyidx1[i] = s.k1y;
    p.dz1[i] = s.k1z;
    p.dxidx2[i] = s.k2x;
    p.dyidx2[i] = s.k2y;
    p.dz2[i] = s.k2z;
}

// `nsteps` AB3 steps (timesteppers.py:296-305) per launch.  table[2*k + j]
// selects the fields of step k at t (j = 0) and t + dt (j = 1).
template <typename T, typename I, bool FIXED>
__global__ void __launch_bounds__(kBlock, 2) k_ab3_steps(const __grid_constant__ DParticles p,
                                                      const __grid_constant__ DScalars sc,
                                                      const __grid_constant__ DRoms r,
                                                      const opb_time *__restrict__ table, int nsteps, int validate_pre) {
    OPB_LEVELS(r, sc);
    const long long i = gtid();
    if (i >= p.n) return;
    PState s;
    s.status = p.status[i];
    if (s.status & ST_INACTIVE) return;
    s.zidx = p.zidx[i];
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    s.k1x = p.dxidx1[i];
    s.k1y = p.dyidx1[i];
    s.k1z = p.dz1[i];
    s.k2x = p.dxidx2[i];
    s.k2y = p.dyidx2[i];
    s.k2z = p.dz2[i];
    const uint8_t st0 = s.status;
    bool moved = false;
    for (int k = 0; k < nsteps; ++k) {
        if (validate_pre) s.status = validate(s.status, s.zidx, s.yidx, s.xidx, sc.bounds);
        if (s.status & ST_INACTIVE) break;
        const opb_time t1 = table[2 * k], t2 = table[2 * k + 1];
        const bool reuse = k > 0 && same_time(t1, s.at);
        if (!ab3_step(s, bind_all<T, I, FIXED>(r, t1), sc, reuse)) {
            raise_zero_division(p);
            break;
        }
        moved = true;
        ab3_post(s, bind_all<T, I, FIXED>(r, t2), L, sc);
        s.at = t2;
    }
    if (s.status != st0) p.status[i] = s.status;
    if (!moved) return;
    p.zidx[i] = s.zidx;
    p.yidx[i] = s.yidx;
    p.xidx[i] = s.xidx;
    p.z[i] = s.z;
    p.dxidx0[i] = s.k1x;
    p.dyidx0[i] = s.k1y;
    p.dz0[i] = s.k1z;
    p.dxidx1[i] = s.k1x;
    p.dyidx1[i] = s.k1y;
    p.dz1[i] = s.k1z;
    p.dxidx2[i] = s.k2x;
    p.dyidx2[i] = s.k2y;
    p.dz2[i] = s.k2z;
}

// ------------------------------------------------------- batched experiments
// Many release experiments in one persistent launch.  Every warp claims
// chunks of OPB_BATCH_CHUNK consecutive particles from a counter in the
// header; a chunk lies inside one experiment's segment, so the 32 lanes of a
// warp share a scheme, a step count and a time table and never diverge on
// them.  Each lane runs its particle through the same stage functions as
// k_rk2_steps / k_ab3_steps with its experiment's dt and alpha.
template <typename T, typename I>
__device__ __forceinline__ void batched_particle(const DParticles &p, long long i, const opb_experiment &E,
                                                 const DScalars &sc0, const DRoms &r, const opb_time *table,
                                                 const Levels &L) {
    PState s;
    s.status = p.status[i];
    if (s.status & ST_INACTIVE) return;
    DScalars sc = sc0;
    sc.dt = E.dt;
    sc.alpha = E.alpha;
    s.zidx = p.zidx[i];
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    const bool ab3 = E.scheme == OPB_SCHEME_AB3;
    if (ab3) {
        s.k1x = p.dxidx1[i];
        s.k1y = p.dyidx1[i];
        s.k1z = p.dz1[i];
        s.k2x = p.dxidx2[i];
        s.k2y = p.dyidx2[i];
        s.k2z = p.dz2[i];
    }
    const uint8_t st0 = s.status;
    bool moved = false;
    const opb_time *tab = table + E.table_offset;
    for (int k = 0; k < E.nsteps; ++k) {
        if (E.validate) s.status = validate(s.status, s.zidx, s.yidx, s.xidx, sc.bounds);
        if (s.status & ST_INACTIVE) break;
        if (ab3) {
            const opb_time t1 = tab[2 * k], t2 = tab[2 * k + 1];
            const bool reuse = k > 0 && same_time(t1, s.at);
            if (!ab3_step(s, bind_all<T, I, true>(r, t1), sc, reuse)) {
                raise_zero_division(p);
                break;
            }
            moved = true;
            ab3_post(s, bind_all<T, I, true>(r, t2), L, sc);
            s.at = t2;
        } else {
            const opb_time t1 = tab[3 * k], t2 = tab[3 * k + 1], t3 = tab[3 * k + 2];
            const bool reuse = k > 0 && same_time(t1, s.at);
            if (!rk2_stage1(s, bind_all<T, I, true>(r, t1), sc, reuse)) {
                raise_zero_division(p);
                break;
            }
            moved = true;
            if (!rk2_stage2(s, bind_all<T, I, true>(r, t2), L, sc)) {
                raise_zero_division(p);
                break;
            }
            rk2_update(s, bind_all<T, I, true>(r, t3), L, sc);
            s.at = t3;
        }
    }
    if (s.status != st0) p.status[i] = s.status;
    if (!moved) return;
    p.zidx[i] = s.zidx;
    p.yidx[i] = s.yidx;
    p.xidx[i] = s.xidx;
    p.z[i] = s.z;
    if (ab3) {
        p.dxidx0[i] = s.k1x;
        p.dyidx0[i] = s.k1y;
        p.dz0[i] = s.k1z;
    }
    p.dxidx1[i] = s.k1x;
    p.dyidx1[i] = s.k1y;
    p.dz1[i] = s.k1z;
    p.dxidx2[i] = s.k2x;
    p.dyidx2[i] = s.k2y;
    p.dz2[i] = s.k2z;
}

// 128 registers per thread at any block size: 16 warps per SM
template <typename T, typename I, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 512 / BLOCK) k_batched_steps(const __grid_constant__ DParticles p,
                                                                   opb_batch_header *__restrict__ hdr,
                                                                   const opb_experiment *__restrict__ exps,
                                                                   const __grid_constant__ DScalars sc,
                                                                   const __grid_constant__ DRoms r,
                                                                   const opb_time *__restrict__ table) {
    OPB_LEVELS(r, sc);
    const int nexp = hdr->nexp;
    const long long nchunks = hdr->nchunks;
    const int lane = threadIdx.x & 31;
    unsigned long long *counter = (unsigned long long *)&hdr->next_chunk;
    for (;;) {
        unsigned long long c = 0;
        if (lane == 0) c = atomicAdd(counter, 1ULL);
        c = __shfl_sync(0xffffffffu, c, 0);
        if ((long long)c >= nchunks) break;
        // the experiment owning chunk c: the last one whose first_chunk <= c
        int lo = 0, hi = nexp - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (exps[mid].first_chunk <= (long long)c) lo = mid;
            else hi = mid - 1;
        }
        const opb_experiment E = exps[lo];
        const long long j = ((long long)c - E.first_chunk) * OPB_BATCH_CHUNK + lane;
        if (j < 0 || j >= E.count || E.nsteps <= 0) continue;
        const long long i = E.start + j;
        if (i < 0 || i >= p.n) continue;
        batched_particle<T, I>(p, i, E, sc, r, table, L);
    }
}

// ---------------------------------------------------------- output kernels
// kernels/output/linear_interpolation.pyx:34-136: sample one field (static,
// or blended in time like every other field) at the active particles.
template <typename T, typename I, int ND>
__global__ void __launch_bounds__(kBlock) k_interpolate(const __grid_constant__ DParticles p,
                                                        const double *__restrict__ i0,
                                                        const double *__restrict__ i1,
                                                        const double *__restrict__ i2,
                                                        const __grid_constant__ DField f, opb_time t, double *out) {
    const long long i = gtid();
    if (i >= p.n || (p.status[i] & ST_INACTIVE)) return;
    const View<T, I> v = bind<T, I>(f, t);
    if (ND == 1) out[i] = linear(v, i0[i] + v.o0);
    else if (ND == 2) out[i] = bilinear(v, i0[i] + v.o0, i1[i] + v.o1);
    else out[i] = trilinear(v, i0[i] + v.o0, i1[i] + v.o1, i2[i] + v.o2);
}

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

// u, v, w, zeta time-dependent and h, dx, dy, C static: the layout the ROMS
// presets use, compiled with the field kinds fixed
bool roms_layout(const DRoms &r) {
    return !r.u.is_static && !r.v.is_static && !r.w.is_static && !r.zeta.is_static && r.h.is_static &&
           r.dx.is_static && r.dy.is_static && r.C.is_static;
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

unsigned grid_for(long long n) { return (unsigned)((n + kBlock - 1) / kBlock); }

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
    return OPB_OK;
}

void convert_scalars(const opb_scalars *in, DScalars &out) {
    out.hc = in->hc;
    out.NZ = in->NZ;
    out.dt = in->dt;
    out.alpha = in->alpha;
    for (int k = 0; k < 6; ++k) out.bounds[k] = in->bounds[k];
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

}  // namespace
}  // namespace opb

using namespace opb;

// ====================================================================== C ABI
extern "C" {

int opb_abi_version(void) { return OPB_ABI_VERSION; }

static int validation_impl(const opb_particles *p, const opb_scalars *s, void *stream, int finite, int bounds,
                           const char *what) {
    DParticles dp;
    int rc;
    if ((rc = convert_particles(p, dp, what, true))) return rc;
    DScalars ds{};
    if (bounds) {
        if (!s) return fail(OPB_EINVAL, "%s: scalars is NULL", what);
        convert_scalars(s, ds);
    }
    if (dp.n == 0) return OPB_OK;
    k_validation<<<grid_for(dp.n), kBlock, 0, (cudaStream_t)stream>>>(dp, ds, finite, bounds);
    return check_launch(what);
}

int opb_finite_indices(const opb_particles *p, void *stream) {
    return validation_impl(p, nullptr, stream, 1, 0, "opb_finite_indices");
}

int opb_domain_bounds(const opb_particles *p, const opb_scalars *s, void *stream) {
    return validation_impl(p, s, stream, 0, 1, "opb_domain_bounds");
}

int opb_validation(const opb_particles *p, const opb_scalars *s, void *stream) {
    return validation_impl(p, s, stream, 1, 1, "opb_validation");
}

int opb_compute_z(const opb_particles *p, double *out, const opb_scalars *s, const opb_roms_fields *f,
                  const opb_time *t, void *stream) {
    const char *what = "opb_compute_z";
    DParticles dp;
    DScalars ds;
    DRoms dr;
    int dtype, rc;
    if ((rc = stage_common(what, p, s, f, t, false, dp, ds, dr, dtype))) return rc;
    if (dp.n > 0 && !out) return fail(OPB_EINVAL, "%s: out is NULL", what);
    if (dp.n == 0) return OPB_OK;
    dispatch(dtype, fits_int(dr), [&](auto tv, auto iv) {
        k_compute_z<decltype(tv), decltype(iv)><<<grid_for(dp.n), kBlock, 0, (cudaStream_t)stream>>>(dp, out, ds,
                                                                                                   dr, *t);
    });
    return check_launch(what);
}

static int need_fields(const opb_particles *p, const char *what, std::initializer_list<std::pair<const char *, const void *>> req) {
    if (!p || p->n == 0) return OPB_OK;
    for (auto &kv : req)
        if (!kv.second) return fail(OPB_EINVAL, "%s: particle field %s is NULL", what, kv.first);
    return OPB_OK;
}

static int stage_launch(const char *what, int which, const opb_particles *p, const opb_scalars *s,
                        const opb_roms_fields *f, const opb_time *t, void *stream) {
    DParticles dp;
    DScalars ds;
    DRoms dr;
    int dtype, rc;
    const bool need_vel = (which == 0 || which == 1 || which == 3);
    if ((rc = stage_common(what, p, s, f, t, need_vel, dp, ds, dr, dtype))) return rc;
    switch (which) {
        case 0: rc = need_fields(p, what, {{"z", p->z}, {"_dxidx1", p->dxidx1}, {"_dyidx1", p->dyidx1}, {"_dz1", p->dz1}}); break;
        case 1:
        case 2:
            rc = need_fields(p, what, {{"z", p->z}, {"_dxidx1", p->dxidx1}, {"_dyidx1", p->dyidx1}, {"_dz1", p->dz1},
                                       {"_dxidx2", p->dxidx2}, {"_dyidx2", p->dyidx2}, {"_dz2", p->dz2}});
            break;
        case 3:
            rc = need_fields(p, what, {{"z", p->z}, {"_dxidx0", p->dxidx0}, {"_dyidx0", p->dyidx0}, {"_dz0", p->dz0},
                                       {"_dxidx1", p->dxidx1}, {"_dyidx1", p->dyidx1}, {"_dz1", p->dz1},
                                       {"_dxidx2", p->dxidx2}, {"_dyidx2", p->dyidx2}, {"_dz2", p->dz2}});
            break;
        default: rc = need_fields(p, what, {{"z", p->z}}); break;
    }
    if (rc) return rc;
    if (dp.n == 0) return OPB_OK;
    const unsigned g = grid_for(dp.n);
    cudaStream_t st = (cudaStream_t)stream;
    dispatch(dtype, fits_int(dr), [&](auto tv, auto iv) {
        using T = decltype(tv);
        using I = decltype(iv);
        switch (which) {
            case 0: k_rk2_step_1<T, I><<<g, kBlock, 0, st>>>(dp, ds, dr, *t); break;
            case 1: k_rk2_step_2<T, I><<<g, kBlock, 0, st>>>(dp, ds, dr, *t); break;
            case 2: k_rk2_update<T, I><<<g, kBlock, 0, st>>>(dp, ds, dr, *t); break;
            case 3: k_ab3<T, I><<<g, kBlock, 0, st>>>(dp, ds, dr, *t); break;
            default: k_ab3_post<T, I><<<g, kBlock, 0, st>>>(dp, ds, dr, *t); break;
        }
    });
    return check_launch(what);
}

int opb_rk2_w_advection_step_1(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                               const opb_time *t, void *stream) {
    return stage_launch("opb_rk2_w_advection_step_1", 0, p, s, f, t, stream);
}

int opb_rk2_w_advection_step_2(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                               const opb_time *t, void *stream) {
    return stage_launch("opb_rk2_w_advection_step_2", 1, p, s, f, t, stream);
}

int opb_rk2_w_advection_update(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                               const opb_time *t, void *stream) {
    return stage_launch("opb_rk2_w_advection_update", 2, p, s, f, t, stream);
}

int opb_ab3_w_advection(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f, const opb_time *t,
                        void *stream) {
    return stage_launch("opb_ab3_w_advection", 3, p, s, f, t, stream);
}

int opb_ab3_post_w_advection(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                             const opb_time *t, void *stream) {
    return stage_launch("opb_ab3_post_w_advection", 4, p, s, f, t, stream);
}

static int steps_launch(const char *what, bool rk2, const opb_particles *p, const opb_scalars *s,
                        const opb_roms_fields *f, const opb_time *table, int32_t nsteps, int32_t validate_pre,
                        void *stream) {
    DParticles dp;
    DScalars ds;
    DRoms dr;
    int dtype, rc;
    if ((rc = convert_particles(p, dp, what, true))) return rc;
    if (!s) return fail(OPB_EINVAL, "%s: scalars is NULL", what);
    convert_scalars(s, ds);
    if ((rc = convert_fields(f, dr, what, true, &dtype))) return rc;
    if (nsteps < 0) return fail(OPB_EINVAL, "%s: negative step count", what);
    if (nsteps > 0 && !table) return fail(OPB_EINVAL, "%s: step table is NULL", what);
    if (rk2)
        rc = need_fields(p, what, {{"z", p->z}, {"_dxidx1", p->dxidx1}, {"_dyidx1", p->dyidx1}, {"_dz1", p->dz1},
                                   {"_dxidx2", p->dxidx2}, {"_dyidx2", p->dyidx2}, {"_dz2", p->dz2}});
    else
        rc = need_fields(p, what, {{"z", p->z}, {"_dxidx0", p->dxidx0}, {"_dyidx0", p->dyidx0}, {"_dz0", p->dz0},
                                   {"_dxidx1", p->dxidx1}, {"_dyidx1", p->dyidx1}, {"_dz1", p->dz1},
                                   {"_dxidx2", p->dxidx2}, {"_dyidx2", p->dyidx2}, {"_dz2", p->dz2}});
    if (rc) return rc;
    if (dp.n == 0 || nsteps == 0) return OPB_OK;
    const unsigned g = grid_for(dp.n);
    cudaStream_t st = (cudaStream_t)stream;
    const bool fixed = roms_layout(dr);
    dispatch(dtype, fits_int(dr), [&](auto tv, auto iv) {
        using T = decltype(tv);
        using I = decltype(iv);
        if (rk2) {
            if (fixed) k_rk2_steps<T, I, true><<<g, kBlock, 0, st>>>(dp, ds, dr, table, nsteps, validate_pre);
            else k_rk2_steps<T, I, false><<<g, kBlock, 0, st>>>(dp, ds, dr, table, nsteps, validate_pre);
        } else {
            if (fixed) k_ab3_steps<T, I, true><<<g, kBlock, 0, st>>>(dp, ds, dr, table, nsteps, validate_pre);
            else k_ab3_steps<T, I, false><<<g, kBlock, 0, st>>>(dp, ds, dr, table, nsteps, validate_pre);
        }
    });
    return check_launch(what);
}

int opb_rk2_w_advection_steps(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                              const opb_time *table, int32_t nsteps, int32_t validate, void *stream) {
    return steps_launch("opb_rk2_w_advection_steps", true, p, s, f, table, nsteps, validate, stream);
}

int opb_ab3_w_advection_steps(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                              const opb_time *table, int32_t nsteps, int32_t validate, void *stream) {
    return steps_launch("opb_ab3_w_advection_steps", false, p, s, f, table, nsteps, validate, stream);
}

static int interpolate_impl(const char *what, int nd, const opb_particles *p, const double *i0, const double *i1,
                            const double *i2, const opb_field *f, const opb_time *t, double *out, void *stream) {
    DParticles dp;
    int rc;
    if ((rc = convert_particles(p, dp, what, false))) return rc;
    if (!f) return fail(OPB_EINVAL, "%s: field is NULL", what);
    DField df;
    int dtype = -1;
    if ((rc = convert_field(*f, df, nd, what, "field", &dtype))) return rc;
    opb_time tt = {0, 1, 0.0, 1.0};
    if (!f->is_static) {
        if (!t) return fail(OPB_EINVAL, "%s: time is NULL", what);
        if (t->prev < 0 || t->prev >= f->nslots || t->next < 0 || t->next >= f->nslots)
            return fail(OPB_EINVAL, "%s: snapshot slot out of range", what);
        tt = *t;
    }
    if (dp.n == 0) return OPB_OK;
    const double *idx[3] = {i0, i1, i2};
    for (int d = 0; d < nd; ++d)
        if (!idx[d]) return fail(OPB_EINVAL, "%s: index array %d is NULL", what, d);
    if (!out) return fail(OPB_EINVAL, "%s: out is NULL", what);
    const unsigned g = grid_for(dp.n);
    cudaStream_t st = (cudaStream_t)stream;
    dispatch(f->is_static ? OPB_F64 : dtype, fits_int(df), [&](auto tv, auto iv) {
        using T = decltype(tv);
        using I = decltype(iv);
        if (nd == 1) k_interpolate<T, I, 1><<<g, kBlock, 0, st>>>(dp, i0, i1, i2, df, tt, out);
        else if (nd == 2) k_interpolate<T, I, 2><<<g, kBlock, 0, st>>>(dp, i0, i1, i2, df, tt, out);
        else k_interpolate<T, I, 3><<<g, kBlock, 0, st>>>(dp, i0, i1, i2, df, tt, out);
    });
    return check_launch(what);
}

int opb_linear_interpolation(const opb_particles *p, const double *idx, const opb_field *f, const opb_time *t,
                             double *out, void *stream) {
    return interpolate_impl("opb_linear_interpolation", 1, p, idx, nullptr, nullptr, f, t, out, stream);
}

int opb_bilinear_interpolation(const opb_particles *p, const double *idx0, const double *idx1, const opb_field *f,
                               const opb_time *t, double *out, void *stream) {
    return interpolate_impl("opb_bilinear_interpolation", 2, p, idx0, idx1, nullptr, f, t, out, stream);
}

int opb_trilinear_interpolation(const opb_particles *p, const opb_field *f, const opb_time *t, double *out,
                                void *stream) {
    if (!p) return fail(OPB_EINVAL, "opb_trilinear_interpolation: particles is NULL");
    return interpolate_impl("opb_trilinear_interpolation", 3, p, p->zidx, p->yidx, p->xidx, f, t, out, stream);
}

int opb_batched_steps(const opb_particles *p, opb_batch_header *header, const opb_experiment *experiments,
                      const opb_scalars *s, const opb_roms_fields *f, const opb_time *table, int32_t block,
                      int32_t ctas, void *stream) {
    const char *what = "opb_batched_steps";
    DParticles dp;
    DScalars ds;
    DRoms dr;
    int dtype, rc;
    if ((rc = convert_particles(p, dp, what, true))) return rc;
    if (!s) return fail(OPB_EINVAL, "%s: scalars is NULL", what);
    convert_scalars(s, ds);
    if ((rc = convert_fields(f, dr, what, true, &dtype))) return rc;
    if (!header || !experiments || !table) return fail(OPB_EINVAL, "%s: NULL device array", what);
    if (block != 128 && block != 256 && block != 512) return fail(OPB_EINVAL, "%s: block must be 128, 256 or 512", what);
    if (ctas < 0) return fail(OPB_EINVAL, "%s: negative CTA count", what);
    if (!roms_layout(dr)) return fail(OPB_EINVAL, "%s: fields must have the ROMS layout (u, v, w, zeta "
                                      "time-dependent; h, dx, dy, C static)", what);
    rc = need_fields(p, what, {{"z", p->z}, {"_dxidx1", p->dxidx1}, {"_dyidx1", p->dyidx1}, {"_dz1", p->dz1},
                               {"_dxidx2", p->dxidx2}, {"_dyidx2", p->dyidx2}, {"_dz2", p->dz2},
                               {"_dxidx0", p->dxidx0}, {"_dyidx0", p->dyidx0}, {"_dz0", p->dz0}});
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(&header->next_chunk, 0, sizeof(header->next_chunk), st);
    if (e != cudaSuccess) return fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    if (dp.n == 0) return OPB_OK;
    int launched = 0;
    dispatch(dtype, fits_int(dr), [&](auto tv, auto iv) {
        using T = decltype(tv);
        using I = decltype(iv);
        auto go = [&](auto kernel, int B) {
            const int g = ctas > 0 ? ctas : resident_ctas((const void *)kernel, B);
            if (g <= 0) return;
            kernel<<<g, B, 0, st>>>(dp, header, experiments, ds, dr, table);
            launched = 1;
        };
        if (block == 128) go(k_batched_steps<T, I, 128>, 128);
        else if (block == 256) go(k_batched_steps<T, I, 256>, 256);
        else go(k_batched_steps<T, I, 512>, 512);
    });
    if (!launched) return fail(OPB_ECUDA, "%s: occupancy query failed", what);
    return check_launch(what);
}

}  // extern "C"
