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
#include <algorithm>
#include <initializer_list>
#include <string>
#include <type_traits>
#include <utility>

#include "opb200.h"
#include "opb_device.cuh"
#include "opb_errors.h"
#include "opb_host.cuh"
#include "opb_stages.cuh"

// Threads per CTA of the fused steppers, and the resident CTAs per SM they are
// compiled for (their register budget: 65536 / (OPB_FUSED_BLOCK *
// OPB_FUSED_MINB) per thread).
#ifndef OPB_FUSED_BLOCK
#define OPB_FUSED_BLOCK 256
#endif
#ifndef OPB_FUSED_MINB
#define OPB_FUSED_MINB 2
#endif
// 1: the fused steppers keep the velocity history in shared memory (PState HS)
#ifndef OPB_FUSED_HIST_SMEM
#define OPB_FUSED_HIST_SMEM 0
#endif

namespace opb {
namespace {

constexpr int kFusedBlock = OPB_FUSED_BLOCK;
unsigned fused_grid(long long n) { return (unsigned)((n + kFusedBlock - 1) / kFusedBlock); }

// opb_records: the particle state after chosen steps of a fused launch
struct DRecords {
    unsigned long long mask[4];
    long long stride;
    double *zidx, *yidx, *xidx, *z;
    uint8_t *status;
    bool any;

    __device__ __forceinline__ bool at(int k) const { return any && ((mask[k >> 6] >> (k & 63)) & 1ull); }
    // records before step k: the slot of step k's record
    __device__ __forceinline__ long long slot(int k) const {
        int c = 0;
        for (int w = 0; w < (k >> 6); ++w) c += __popcll(mask[w]);
        const int b = k & 63;
        return c + (b ? __popcll(mask[k >> 6] & ((1ull << b) - 1ull)) : 0);
    }
    __device__ __forceinline__ void put(int k, long long i, uint8_t st, double zi, double yi, double xi,
                                        double zz) const {
        const long long o = slot(k) * stride + i;
        status[o] = st;
        zidx[o] = zi;
        yidx[o] = yi;
        xidx[o] = xi;
        z[o] = zz;
    }
    // steps [from, to) of a particle whose state no longer changes
    __device__ __forceinline__ void hold(int from, int to, long long i, uint8_t st, double zi, double yi, double xi,
                                         double zz) const {
        if (!any) return;
        for (int k = from; k < to; ++k)
            if (at(k)) put(k, i, st, zi, yi, xi, zz);
    }
};

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
    PState<I> s;
    s.zidx = p.zidx[i];
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    const bool ok = rk2_stage1(s, bind_all<T, I>(r, t), sc, Levels{});
    p.z[i] = s.z;
    if (!ok) {
        raise_zero_division(p);
        return;
    }
    s.get_k1(p.dxidx1[i], p.dyidx1[i], p.dz1[i]);
}

template <typename T, typename I>
__global__ void __launch_bounds__(kBlock) k_rk2_step_2(const __grid_constant__ DParticles p,
                                                       const __grid_constant__ DScalars sc,
                                                       const __grid_constant__ DRoms r, opb_time t) {
    OPB_LEVELS(r, sc);
    const long long i = gtid();
    if (i >= p.n || (p.status[i] & ST_INACTIVE)) return;
    PState<I> s;
    s.zidx = p.zidx[i];  // hint for the vertical search
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    s.z = p.z[i];
    s.set_k1(p.dxidx1[i], p.dyidx1[i], p.dz1[i]);
    if (!rk2_stage2(s, bind_all<T, I>(r, t), L, sc)) {
        raise_zero_division(p);
        return;
    }
    s.get_k2(p.dxidx2[i], p.dyidx2[i], p.dz2[i]);
}

template <typename T, typename I>
__global__ void __launch_bounds__(kBlock) k_rk2_update(const __grid_constant__ DParticles p,
                                                       const __grid_constant__ DScalars sc,
                                                       const __grid_constant__ DRoms r, opb_time t) {
    OPB_LEVELS(r, sc);
    const long long i = gtid();
    if (i >= p.n || (p.status[i] & ST_INACTIVE)) return;
    PState<I> s;
    s.zidx = p.zidx[i];
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    s.z = p.z[i];
    s.set_k1(p.dxidx1[i], p.dyidx1[i], p.dz1[i]);
    s.set_k2(p.dxidx2[i], p.dyidx2[i], p.dz2[i]);
    rk2_update(s, bind_all<T, I>(r, t), L, sc);
    p.z[i] = s.z;
    p.yidx[i] = s.yidx;
    p.xidx[i] = s.xidx;
    p.zidx[i] = s.zidx;
}

template <typename T, typename I, bool ISO>
__device__ __forceinline__ bool ab3_any(PState<I> &s, const Bound<T, I> &f, const DScalars &sc, const DParticles &p,
                                        long long i) {
    if constexpr (ISO) return ab3_step(s, f, sc, Levels{}, false, false, IsoVel{p.rho_t[i], sc.w_max, sc.rho_scale});
    else return ab3_step(s, f, sc, Levels{});
}

template <typename T, typename I, bool ISO = false>
__global__ void __launch_bounds__(kBlock) k_ab3(const __grid_constant__ DParticles p,
                                                const __grid_constant__ DScalars sc,
                                                const __grid_constant__ DRoms r, opb_time t) {
    const long long i = gtid();
    if (i >= p.n) return;
    PState<I> s;
    s.status = p.status[i];
    if (s.status & ST_INACTIVE) return;
    s.zidx = p.zidx[i];
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    s.set_k1(p.dxidx1[i], p.dyidx1[i], p.dz1[i]);
    s.set_k2(p.dxidx2[i], p.dyidx2[i], p.dz2[i]);
    if (!ab3_any<T, I, ISO>(s, bind_all<T, I>(r, t), sc, p, i)) {
        raise_zero_division(p);
        return;
    }
    p.status[i] = s.status;
    p.z[i] = s.z;
    p.yidx[i] = s.yidx;
    p.xidx[i] = s.xidx;
    s.get_k1(p.dxidx0[i], p.dyidx0[i], p.dz0[i]);  // after the history shift k1 == k0
    s.get_k1(p.dxidx1[i], p.dyidx1[i], p.dz1[i]);
    s.get_k2(p.dxidx2[i], p.dyidx2[i], p.dz2[i]);
}

template <typename T, typename I>
__global__ void __launch_bounds__(kBlock) k_ab3_post(const __grid_constant__ DParticles p,
                                                     const __grid_constant__ DScalars sc,
                                                     const __grid_constant__ DRoms r, opb_time t) {
    OPB_LEVELS(r, sc);
    const long long i = gtid();
    if (i >= p.n || (p.status[i] & ST_INACTIVE)) return;
    PState<I> s;
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
template <typename T, typename I, bool FIXED, int LAYOUT = LAYOUT_PLAIN, bool B2 = false>
__global__ void __launch_bounds__(kFusedBlock, OPB_FUSED_MINB) k_rk2_steps(const __grid_constant__ DParticles p,
                                                      const __grid_constant__ DScalars sc,
                                                      const __grid_constant__ DRoms r,
                                                      const __grid_constant__ StepTable table, int nsteps,
                                                      int validate_pre, const __grid_constant__ DRecords rec) {
    OPB_LEVELS(r, sc);
    const long long i = gtid();
    if (i >= p.n) return;
    constexpr bool HS = OPB_FUSED_HIST_SMEM != 0;
    PState<I, HS> s;
    if constexpr (HS) {
        __shared__ double s_hist[6 * kFusedBlock];
        s.hs = s_hist + threadIdx.x;
        s.hstride = kFusedBlock;
    }
    s.status = p.status[i];
    if (s.status & ST_INACTIVE) {
        rec.hold(0, nsteps, i, s.status, p.zidx[i], p.yidx[i], p.xidx[i], p.z[i]);
        return;
    }
    s.zidx = p.zidx[i];
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    const uint8_t st0 = s.status;
    bool moved = false;
    int k = 0;
    for (; k < nsteps; ++k) {
        if (validate_pre) s.status = validate(s.status, s.zidx, s.yidx, s.xidx, sc.bounds);
        if (s.status & ST_INACTIVE) break;
        const opb_time t1 = table.at(3 * k), t2 = table.at(3 * k + 1), t3 = table.at(3 * k + 2);
        // h and zeta of the last update (at the previous step's t + dt, the entry before t1) carry over
        // when t1 selects the same snapshots and weights
        const bool reuse = k > 0 && same_time(t1, table.at(3 * k - 1));
        if (!rk2_stage1(s, bind_all<T, I, FIXED, LAYOUT, B2>(r, t1), sc, L, reuse, k > 0)) {
            raise_zero_division(p);
            break;
        }
        moved = true;
        if (!rk2_stage2(s, bind_all<T, I, FIXED, LAYOUT, B2>(r, t2), L, sc)) {
            raise_zero_division(p);
            break;
        }
        rk2_update(s, bind_all<T, I, FIXED, LAYOUT, B2>(r, t3), L, sc);
        if (rec.at(k)) rec.put(k, i, s.status, s.zidx, s.yidx, s.xidx, s.z);
    }
    rec.hold(k, nsteps, i, s.status, s.zidx, s.yidx, s.xidx, moved ? s.z : p.z[i]);
    if (s.status != st0) p.status[i] = s.status;
    if (!moved) return;
    p.zidx[i] = s.zidx;
    p.yidx[i] = s.yidx;
    p.xidx[i] = s.xidx;
    p.z[i] = s.z;
    s.get_k1(p.dxidx1[i], p.dyidx1[i], p.dz1[i]);
    s.get_k2(p.dxidx2[i], p.dyidx2[i], p.dz2[i]);
}

// `nsteps` AB3 steps (timesteppers.py:296-305) per launch.  table[2*k + j]
// selects the fields of step k at t (j = 0) and t + dt (j = 1).
template <typename T, typename I, bool FIXED, int LAYOUT = LAYOUT_PLAIN, bool ISO = false, bool B2 = false>
__global__ void __launch_bounds__(kFusedBlock, OPB_FUSED_MINB) k_ab3_steps(const __grid_constant__ DParticles p,
                                                      const __grid_constant__ DScalars sc,
                                                      const __grid_constant__ DRoms r,
                                                      const __grid_constant__ StepTable table, int nsteps,
                                                      int validate_pre, const __grid_constant__ DRecords rec) {
    OPB_LEVELS(r, sc);
    const long long i = gtid();
    if (i >= p.n) return;
    constexpr bool HS = OPB_FUSED_HIST_SMEM != 0;
    PState<I, HS> s;
    if constexpr (HS) {
        __shared__ double s_hist[6 * kFusedBlock];
        s.hs = s_hist + threadIdx.x;
        s.hstride = kFusedBlock;
    }
    s.status = p.status[i];
    if (s.status & ST_INACTIVE) {
        rec.hold(0, nsteps, i, s.status, p.zidx[i], p.yidx[i], p.xidx[i], p.z[i]);
        return;
    }
    s.zidx = p.zidx[i];
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    s.set_k1(p.dxidx1[i], p.dyidx1[i], p.dz1[i]);
    s.set_k2(p.dxidx2[i], p.dyidx2[i], p.dz2[i]);
    const double rho_t = ISO ? p.rho_t[i] : 0.0;
    const uint8_t st0 = s.status;
    bool moved = false;
    int k = 0;
    for (; k < nsteps; ++k) {
        if (validate_pre) s.status = validate(s.status, s.zidx, s.yidx, s.xidx, sc.bounds);
        if (s.status & ST_INACTIVE) break;
        const opb_time t1 = table.at(2 * k), t2 = table.at(2 * k + 1);
        // h and zeta of the last post step (at the previous step's t + dt, the entry before t1) carry over
        // when t1 selects the same snapshots and weights
        const bool reuse = k > 0 && same_time(t1, table.at(2 * k - 1));
        bool ok;
        if constexpr (ISO)
            ok = ab3_step(s, bind_all<T, I, FIXED, LAYOUT, B2>(r, t1), sc, L, reuse, k > 0,
                          IsoVel{rho_t, sc.w_max, sc.rho_scale});
        else ok = ab3_step(s, bind_all<T, I, FIXED, LAYOUT, B2>(r, t1), sc, L, reuse, k > 0);
        if (!ok) {
            raise_zero_division(p);
            break;
        }
        moved = true;
        ab3_post(s, bind_all<T, I, FIXED, LAYOUT, B2>(r, t2), L, sc);
        if (rec.at(k)) rec.put(k, i, s.status, s.zidx, s.yidx, s.xidx, s.z);
    }
    rec.hold(k, nsteps, i, s.status, s.zidx, s.yidx, s.xidx, moved ? s.z : p.z[i]);
    if (s.status != st0) p.status[i] = s.status;
    if (!moved) return;
    p.zidx[i] = s.zidx;
    p.yidx[i] = s.yidx;
    p.xidx[i] = s.xidx;
    p.z[i] = s.z;
    s.get_k1(p.dxidx0[i], p.dyidx0[i], p.dz0[i]);
    s.get_k1(p.dxidx1[i], p.dyidx1[i], p.dz1[i]);
    s.get_k2(p.dxidx2[i], p.dyidx2[i], p.dz2[i]);
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

// div12 against the IEEE division of the same build: counts the x[i] whose two
// quotients differ in any bit (two NaNs agree)
__global__ void __launch_bounds__(kBlock) k_check_div12(const double *__restrict__ x, long long n,
                                                        unsigned long long *bad) {
    unsigned long long mine = 0;
    for (long long i = gtid(); i < n; i += (long long)gridDim.x * blockDim.x) {
        const double a = div12(x[i]);
        const double b = x[i] / 12.0;
        if (__double_as_longlong(a) != __double_as_longlong(b) && !(isnan(a) && isnan(b))) ++mine;
    }
    if (mine) atomicAdd(bad, mine);
}

}  // namespace
}  // namespace opb

using namespace opb;

// ====================================================================== C ABI
extern "C" {

int opb_abi_version(void) { return OPB_ABI_VERSION; }

int opb_check_div12(const double *x, int64_t n, uint64_t *mismatches, void *stream) {
    if (n < 0 || (n > 0 && (!x || !mismatches))) return fail(OPB_EINVAL, "opb_check_div12: bad arguments");
    if (n == 0) return OPB_OK;
    const long long blocks = std::min<long long>((n + kBlock - 1) / kBlock, 148LL * 8);
    k_check_div12<<<(unsigned)blocks, kBlock, 0, (cudaStream_t)stream>>>(x, n, (unsigned long long *)mismatches);
    return check_launch("opb_check_div12");
}

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


static int stage_launch(const char *what, int which, const opb_particles *p, const opb_scalars *s,
                        const opb_roms_fields *f, const opb_time *t, void *stream) {
    DParticles dp;
    DScalars ds;
    DRoms dr;
    int dtype, rc;
    const bool need_vel = (which == 0 || which == 1 || which == 3 || which == 5);
    if ((rc = stage_common(what, p, s, f, t, need_vel, dp, ds, dr, dtype))) return rc;
    switch (which) {
        case 0: rc = need_fields(p, what, {{"z", p->z}, {"_dxidx1", p->dxidx1}, {"_dyidx1", p->dyidx1}, {"_dz1", p->dz1}}); break;
        case 1:
        case 2:
            rc = need_fields(p, what, {{"z", p->z}, {"_dxidx1", p->dxidx1}, {"_dyidx1", p->dyidx1}, {"_dz1", p->dz1},
                                       {"_dxidx2", p->dxidx2}, {"_dyidx2", p->dyidx2}, {"_dz2", p->dz2}});
            break;
        case 3:
        case 5:
            rc = need_fields(p, what, {{"z", p->z}, {"_dxidx0", p->dxidx0}, {"_dyidx0", p->dyidx0}, {"_dz0", p->dz0},
                                       {"_dxidx1", p->dxidx1}, {"_dyidx1", p->dyidx1}, {"_dz1", p->dz1},
                                       {"_dxidx2", p->dxidx2}, {"_dyidx2", p->dyidx2}, {"_dz2", p->dz2}});
            if (!rc && which == 5) rc = need_fields(p, what, {{"rho_t", p->rho_t}});
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
            case 5: k_ab3<T, I, true><<<g, kBlock, 0, st>>>(dp, ds, dr, *t); break;
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

// opb_records -> DRecords, checked against the launch
static int convert_records(const opb_records *rec, long long n, int32_t nsteps, DRecords &d, const char *what) {
    d = DRecords{};
    if (!rec) return OPB_OK;
    int count = 0;
    for (int w = 0; w < 4; ++w) {
        d.mask[w] = rec->mask[w];
        for (int b = 0; b < 64; ++b)
            if ((rec->mask[w] >> b) & 1ull) {
                if (w * 64 + b >= nsteps) return fail(OPB_EINVAL, "%s: a record after step %d of %d", what, w * 64 + b, nsteps);
                ++count;
            }
    }
    if (count == 0) return OPB_OK;
    if (rec->stride < n) return fail(OPB_EINVAL, "%s: record stride %lld below the particle count", what,
                                     (long long)rec->stride);
    if (!rec->zidx || !rec->yidx || !rec->xidx || !rec->z || !rec->status)
        return fail(OPB_EINVAL, "%s: a record array is NULL", what);
    d.stride = rec->stride;
    d.zidx = rec->zidx;
    d.yidx = rec->yidx;
    d.xidx = rec->xidx;
    d.z = rec->z;
    d.status = rec->status;
    d.any = true;
    return OPB_OK;
}

static int steps_launch(const char *what, bool rk2, const opb_particles *p, const opb_scalars *s,
                        const opb_roms_fields *f, const opb_time *table, int32_t nsteps, int32_t validate_pre,
                        void *stream, bool iso = false, const opb_records *records = nullptr) {
    DParticles dp;
    DScalars ds;
    DRoms dr;
    int dtype, rc;
    if ((rc = convert_particles(p, dp, what, true))) return rc;
    if (!s) return fail(OPB_EINVAL, "%s: scalars is NULL", what);
    convert_scalars(s, ds);
    opb_roms_fields g;
    int layout = LAYOUT_PLAIN;
    bool bundled = false;
    if ((rc = unpair_fields(f, g, layout, bundled, what))) return rc;
    if ((rc = convert_fields(&g, dr, what, true, &dtype))) return rc;
    if (layout != LAYOUT_PLAIN && !roms_layout(dr, iso))
        return fail(OPB_EINVAL, "%s: snapshot pairs need the ROMS field layout and geometry", what);
    if (nsteps < 0) return fail(OPB_EINVAL, "%s: negative step count", what);
    DRecords rec;
    if ((rc = convert_records(records, dp.n, nsteps, rec, what))) return rc;
    if (nsteps > 0 && !table) return fail(OPB_EINVAL, "%s: step table is NULL", what);
    if (rk2)
        rc = need_fields(p, what, {{"z", p->z}, {"_dxidx1", p->dxidx1}, {"_dyidx1", p->dyidx1}, {"_dz1", p->dz1},
                                   {"_dxidx2", p->dxidx2}, {"_dyidx2", p->dyidx2}, {"_dz2", p->dz2}});
    else
        rc = need_fields(p, what, {{"z", p->z}, {"_dxidx0", p->dxidx0}, {"_dyidx0", p->dyidx0}, {"_dz0", p->dz0},
                                   {"_dxidx1", p->dxidx1}, {"_dyidx1", p->dyidx1}, {"_dz1", p->dz1},
                                   {"_dxidx2", p->dxidx2}, {"_dyidx2", p->dyidx2}, {"_dz2", p->dz2}});
    if (!rc && iso) rc = need_fields(p, what, {{"rho_t", p->rho_t}});
    if (rc) return rc;
    if (dp.n == 0 || nsteps == 0) return OPB_OK;
    static thread_local StepTable tab;  // up to 17 KB: kept off the stack
    int nslots = 0;
    for (const opb_field *x : {&g.u, &g.v, &g.w, &g.zeta})
        if (!x->is_static && (nslots == 0 || x->nslots < nslots)) nslots = x->nslots;
    if ((rc = make_step_table(table, (long long)nsteps * (rk2 ? 3 : 2), tab, what, nslots))) return rc;
    const unsigned grid = fused_grid(dp.n);
    cudaStream_t st = (cudaStream_t)stream;
    const bool fixed = roms_layout(dr, iso);
    auto go = [&](auto tv, auto iv, auto lv, auto bv) {
        using T = decltype(tv);
        using I = decltype(iv);
        constexpr int LAYOUT = decltype(lv)::value;
        constexpr bool B2 = decltype(bv)::value;
        if (rk2) k_rk2_steps<T, I, true, LAYOUT, B2><<<grid, kFusedBlock, 0, st>>>(dp, ds, dr, tab, nsteps, validate_pre, rec);
        else if (iso)
            k_ab3_steps<T, I, true, LAYOUT, true, B2><<<grid, kFusedBlock, 0, st>>>(dp, ds, dr, tab, nsteps, validate_pre, rec);
        else k_ab3_steps<T, I, true, LAYOUT, false, B2><<<grid, kFusedBlock, 0, st>>>(dp, ds, dr, tab, nsteps, validate_pre, rec);
    };
    using NoB = std::false_type;
    using Bun = std::true_type;
    const bool small = fits_int(dr);
    if (layout == LAYOUT_QUADS || layout == LAYOUT_OCTS || bundled) {
        if (dtype != OPB_F32)
            return fail(OPB_EINVAL, "%s: snapshot quads, octets and 2-D bundles hold float32 storage", what);
        using Q = std::integral_constant<int, LAYOUT_QUADS>;
        using O = std::integral_constant<int, LAYOUT_OCTS>;
        using P = std::integral_constant<int, LAYOUT_PAIRS>;
        if (layout == LAYOUT_OCTS) {
            if (small) go(float{}, int{}, O{}, NoB{});
            else go(float{}, (long long){}, O{}, NoB{});
        } else if (layout == LAYOUT_QUADS) {
            if (small) bundled ? go(float{}, int{}, Q{}, Bun{}) : go(float{}, int{}, Q{}, NoB{});
            else bundled ? go(float{}, (long long){}, Q{}, Bun{}) : go(float{}, (long long){}, Q{}, NoB{});
        } else {
            if (small) go(float{}, int{}, P{}, Bun{});
            else go(float{}, (long long){}, P{}, Bun{});
        }
        return check_launch(what);
    }
    dispatch(dtype, small, [&](auto tv, auto iv) {
        using T = decltype(tv);
        using I = decltype(iv);
        if (layout == LAYOUT_PAIRS) go(tv, iv, std::integral_constant<int, LAYOUT_PAIRS>{}, NoB{});
        else if (fixed) go(tv, iv, std::integral_constant<int, LAYOUT_PLAIN>{}, NoB{});
        else if (rk2) k_rk2_steps<T, I, false><<<grid, kFusedBlock, 0, st>>>(dp, ds, dr, tab, nsteps, validate_pre, rec);
        else if (iso)
            k_ab3_steps<T, I, false, LAYOUT_PLAIN, true><<<grid, kFusedBlock, 0, st>>>(dp, ds, dr, tab, nsteps,
                                                                                 validate_pre, rec);
        else k_ab3_steps<T, I, false><<<grid, kFusedBlock, 0, st>>>(dp, ds, dr, tab, nsteps, validate_pre, rec);
    });
    return check_launch(what);
}

int opb_ab3_isopycnal_following(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                                const opb_time *t, void *stream) {
    return stage_launch("opb_ab3_isopycnal_following", 5, p, s, f, t, stream);
}

int opb_ab3_isopycnal_following_steps(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                                      const opb_time *table, int32_t nsteps, int32_t validate, void *stream) {
    return steps_launch("opb_ab3_isopycnal_following_steps", false, p, s, f, table, nsteps, validate, stream, true);
}

int opb_rk2_w_advection_steps(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                              const opb_time *table, int32_t nsteps, int32_t validate, void *stream) {
    return steps_launch("opb_rk2_w_advection_steps", true, p, s, f, table, nsteps, validate, stream);
}

int opb_ab3_w_advection_steps(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                              const opb_time *table, int32_t nsteps, int32_t validate, void *stream) {
    return steps_launch("opb_ab3_w_advection_steps", false, p, s, f, table, nsteps, validate, stream);
}

int opb_rk2_w_advection_steps_rec(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                                  const opb_time *table, int32_t nsteps, int32_t validate, const opb_records *rec,
                                  void *stream) {
    return steps_launch("opb_rk2_w_advection_steps_rec", true, p, s, f, table, nsteps, validate, stream, false, rec);
}

int opb_ab3_w_advection_steps_rec(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                                  const opb_time *table, int32_t nsteps, int32_t validate, const opb_records *rec,
                                  void *stream) {
    return steps_launch("opb_ab3_w_advection_steps_rec", false, p, s, f, table, nsteps, validate, stream, false,
                        rec);
}

int opb_ab3_isopycnal_following_steps_rec(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                                          const opb_time *table, int32_t nsteps, int32_t validate,
                                          const opb_records *rec, void *stream) {
    return steps_launch("opb_ab3_isopycnal_following_steps_rec", false, p, s, f, table, nsteps, validate, stream,
                        true, rec);
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

}  // extern "C"
