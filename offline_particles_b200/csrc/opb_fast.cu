// Reduced-precision fused steppers (float32 arithmetic) and level quantisation.
//
// Same algorithm as opb_roms.cu -- rk2_w_advection.pyx:31-354 and
// ab3_w_advection.pyx:20-229 of the reference, the validation pre-step of the
// ROMS presets -- evaluated in float32:
//   * interpolation weights and sums, the time blend and the velocity
//     divisions in float32 (multiply-adds may contract in this file);
//   * the fractional y/x indices kept as compensated float32 pairs (hi + lo,
//     updated with an error-free 2Sum), because a bare float32 index near
//     1000 would lose ~1e-4 cells every step;
//   * z = zeta + (zeta + h) S and its inverse in float64 when the column is
//     shallower than kShallow metres (there the sigma layers are thin and
//     float32 would move particles between layers), float32 elsewhere;
//   * time-dependent fields stored as float32, or as bfloat16 / float16 with
//     one scale per (snapshot, level).
// Results are not bit-identical to the reference; the error is reported as
// trajectory separation against the float64 path.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <initializer_list>

#include "opb200.h"
#include "opb_errors.h"
#include "opb_steptable.cuh"

namespace opb_fast {
namespace {

using opb::fail;
using opb::make_step_table;
using opb::StepTable;

constexpr int kBlock = 256;
constexpr int kMaxLevels = 128;
constexpr float kShallow = 100.0f;
constexpr uint8_t ST_INACTIVE = OPB_STATUS_INACTIVE;

struct FField {
    const void *data[OPB_MAX_SLOTS];
    const float *scale[OPB_MAX_SLOTS];
    int n0, n1, n2;
    float o0, o1, o2;
};

struct FRoms {
    FField u, v, w, zeta;  // time-dependent, storage S
    FField dx, dy, h, C;   // static float64
};

struct FParticles {
    long long n;
    uint8_t *status;
    double *zidx, *yidx, *xidx, *z;
    double *dxidx0, *dyidx0, *dz0;
    double *dxidx1, *dyidx1, *dz1;
    double *dxidx2, *dyidx2, *dz2;
    uint32_t *err;
};

struct FScalars {
    double hc;
    int NZ;
    double dt, alpha;
    double bounds[6];
};

template <typename S>
__device__ __forceinline__ float to_f(S v);
template <>
__device__ __forceinline__ float to_f<float>(float v) {
    return v;
}
template <>
__device__ __forceinline__ float to_f<__half>(__half v) {
    return __half2float(v);
}
template <>
__device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) {
    return __bfloat162float(v);
}

// ------------------------------------------------------ compensated indices
struct CPos {
    float hi, lo;
};

__device__ __forceinline__ CPos cpos(double x) {
    const float h = (float)x;
    return {h, (float)(x - (double)h)};
}

__device__ __forceinline__ double cval(const CPos &p) { return (double)p.hi + (double)p.lo; }

// p += d without losing d's low bits: 2Sum of hi and d, error folded into lo
__device__ __forceinline__ void cadd(CPos &p, float d) {
    const float s = p.hi + d;
    const float bb = s - p.hi;
    const float err = (p.hi - (s - bb)) + (d - bb);
    const float lo = p.lo + err;
    const float h2 = s + lo;
    p.lo = lo - (h2 - s);
    p.hi = h2;
}

// cell index (clamped to [0, max_idx], the clamp then extrapolating through
// the fraction, as linear.pxd:3-17 does) and fraction of a compensated index
__device__ __forceinline__ void split(const CPos &p, float off, int max_idx, int &I, float &f) {
    const float ph = p.hi + off;  // exact: off is 0 or +-0.5 and |hi| < 2^22
    if (!(fabsf(ph) < 1.0e9f)) {  // non-finite or absurd: cell 0, fraction carries the NaN/inf
        I = 0;
        f = ph;
        return;
    }
    const float fl = floorf(ph);
    float fr = (ph - fl) + p.lo;
    int i = (int)fl;
    if (fr < 0.0f) {
        i -= 1;
        fr += 1.0f;
    } else if (fr >= 1.0f) {
        i += 1;
        fr -= 1.0f;
    }
    if (i < 0) {
        fr += (float)i;
        i = 0;
    } else if (i > max_idx) {
        fr += (float)(i - max_idx);
        i = max_idx;
    }
    I = i;
    f = fr;
}

// ------------------------------------------------------------------ fields
// A time-dependent field at one time selection: value = stored * scale(level)
// blended as prev * gt + next * ft.  Per level l the coefficients are
// cp[l] = sp[l] * gt and cn[l] = sn[l] * ft (sp = sn = 1 when unscaled).
template <typename S, bool SCALED>
struct TDView {
    const S *prev;
    const S *next;
    const float *sp;
    const float *sn;
    float ft, gt;
    int n0, n1, n2;
    float o0, o1, o2;

    __device__ __forceinline__ void coef(int level, float &cp, float &cn) const {
        if (SCALED) {
            cp = __ldg(sp + level) * gt;
            cn = __ldg(sn + level) * ft;
        } else {
            cp = gt;
            cn = ft;
        }
    }
    __device__ __forceinline__ float at(int i, float cp, float cn) const {
        return to_f(prev[i]) * cp + to_f(next[i]) * cn;
    }
};

struct StaticView {
    const double *a;
    int n0, n1;
    float o0, o1;
    __device__ __forceinline__ float at(int i) const { return (float)__ldg(a + i); }
};

template <typename S, bool SCALED>
__device__ __forceinline__ TDView<S, SCALED> bind_td(const FField &f, const opb_time &t) {
    TDView<S, SCALED> v;
    v.prev = (const S *)f.data[t.prev];
    v.next = (const S *)f.data[t.next];
    v.sp = f.scale[t.prev];
    v.sn = f.scale[t.next];
    v.ft = (float)t.ft;
    v.gt = (float)t.gt;
    v.n0 = f.n0;
    v.n1 = f.n1;
    v.n2 = f.n2;
    v.o0 = f.o0;
    v.o1 = f.o1;
    v.o2 = f.o2;
    return v;
}

__device__ __forceinline__ StaticView bind_static(const FField &f) {
    StaticView v;
    v.a = (const double *)f.data[0];
    v.n0 = f.n0;
    v.n1 = f.n1;
    v.o0 = f.o0;
    v.o1 = f.o1;
    return v;
}

template <typename S, bool SCALED>
__device__ __forceinline__ float trilinear(const TDView<S, SCALED> &f, const CPos &z, const CPos &y, const CPos &x) {
    int I0, I1, I2;
    float f0, f1, f2;
    split(z, f.o0, f.n0 - 2, I0, f0);
    split(y, f.o1, f.n1 - 2, I1, f1);
    split(x, f.o2, f.n2 - 2, I2, f2);
    const float g0 = 1.0f - f0, g1 = 1.0f - f1, g2 = 1.0f - f2;
    const int s1 = f.n2, s0 = f.n1 * f.n2;
    const int b = I0 * s0 + I1 * s1 + I2;
    float cp0, cn0, cp1, cn1;
    f.coef(I0, cp0, cn0);
    f.coef(I0 + 1, cp1, cn1);
    const float v000 = f.at(b, cp0, cn0), v001 = f.at(b + 1, cp0, cn0);
    const float v010 = f.at(b + s1, cp0, cn0), v011 = f.at(b + s1 + 1, cp0, cn0);
    const float v100 = f.at(b + s0, cp1, cn1), v101 = f.at(b + s0 + 1, cp1, cn1);
    const float v110 = f.at(b + s0 + s1, cp1, cn1), v111 = f.at(b + s0 + s1 + 1, cp1, cn1);
    const float a0 = g1 * (g2 * v000 + f2 * v001) + f1 * (g2 * v010 + f2 * v011);
    const float a1 = g1 * (g2 * v100 + f2 * v101) + f1 * (g2 * v110 + f2 * v111);
    return g0 * a0 + f0 * a1;
}

// 2-D time-dependent field (zeta): one level, scale index 0
template <typename S, bool SCALED>
__device__ __forceinline__ float bilinear_td(const TDView<S, SCALED> &f, const CPos &y, const CPos &x) {
    int I0, I1;
    float f0, f1;
    split(y, f.o0, f.n0 - 2, I0, f0);
    split(x, f.o1, f.n1 - 2, I1, f1);
    float cp, cn;
    f.coef(0, cp, cn);
    const int b = I0 * f.n1 + I1;
    const float v00 = f.at(b, cp, cn), v01 = f.at(b + 1, cp, cn);
    const float v10 = f.at(b + f.n1, cp, cn), v11 = f.at(b + f.n1 + 1, cp, cn);
    return (1.0f - f0) * ((1.0f - f1) * v00 + f1 * v01) + f0 * ((1.0f - f1) * v10 + f1 * v11);
}

__device__ __forceinline__ float bilinear_static(const StaticView &f, const CPos &y, const CPos &x) {
    int I0, I1;
    float f0, f1;
    split(y, f.o0, f.n0 - 2, I0, f0);
    split(x, f.o1, f.n1 - 2, I1, f1);
    const int b = I0 * f.n1 + I1;
    const float v00 = f.at(b), v01 = f.at(b + 1), v10 = f.at(b + f.n1), v11 = f.at(b + f.n1 + 1);
    return (1.0f - f0) * ((1.0f - f1) * v00 + f1 * v01) + f0 * ((1.0f - f1) * v10 + f1 * v11);
}

__device__ __forceinline__ double linear_static_d(const StaticView &f, double idx) {
    // the C table: a 1-D static field, interpolated in the vertical coordinate's precision
    const double p = idx + (double)f.o0;
    long long i = (p >= 1.0 && p < 1.0e9) ? (long long)p : 0;
    if (i > f.n0 - 2) i = f.n0 - 2;
    const double fr = p - (double)i;
    return (1.0 - fr) * __ldg(f.a + i) + fr * __ldg(f.a + i + 1);
}

// ----------------------------------------------------- vertical coordinate
// _vertical_coordinate.pxd:19-103 in precision R (float or double); zero
// divisors return 0 as in the reference.
struct Levels {
    const double *sigma;
    const double *C;
    int size;
    double C_offset;
    int Nz;
    bool monotone;
};

template <typename R>
__device__ __forceinline__ R S_coord(R hc, R sigma, R h, R C) {
    const R den = hc + h;
    if (den == R(0)) return R(0);
    return (hc * sigma + h * C) / den;
}

template <typename R>
__device__ __forceinline__ R compute_z_r(R zidx, int Nz, R hc, R h, R C, R zeta) {
    const R sigma = Nz == 0 ? R(0) : (zidx + R(0.5)) / R(Nz) - R(1);
    return zeta + (zeta + h) * S_coord(hc, sigma, h, C);
}

template <typename R>
__device__ __forceinline__ R S_lev(const Levels &L, int k, R hc, R h) {
    return S_coord<R>(hc, (R)L.sigma[k], h, (R)L.C[k]);
}

template <typename R>
__device__ __forceinline__ R zidx_search(R S, R h, R hc, const Levels &L, double hint) {
    const int top = L.size - 2;
    int Cidx;
    R S_low, S_high;
    bool done = false;
    if (L.monotone && top >= 1 && !(S != S)) {
        // walk from the hint (the particle's previous level)
        const double hk = hint + L.C_offset;
        int k = (hk >= 1.0 && hk < (double)top) ? (int)hk : (hk >= (double)top ? top : 0);
        R lo_v = S_lev<R>(L, k, hc, h);
        for (int walk = 0; walk < 4 && !done; ++walk) {
            if (lo_v > S && k > 0) {
                --k;
                lo_v = S_lev<R>(L, k, hc, h);
                continue;
            }
            if (lo_v > S) {  // below the bottom level
                Cidx = 0;
                S_low = lo_v;
                S_high = S_lev<R>(L, 1, hc, h);
                done = true;
                break;
            }
            if (k == top) {
                Cidx = top;
                S_low = lo_v;
                S_high = S_lev<R>(L, top + 1, hc, h);
                done = true;
                break;
            }
            const R hi_v = S_lev<R>(L, k + 1, hc, h);
            if (hi_v > S) {
                Cidx = k;
                S_low = lo_v;
                S_high = hi_v;
                done = true;
                break;
            }
            ++k;
            lo_v = hi_v;
        }
    }
    if (!done) {  // binary search
        int lo = 0, hi = top;
        const R S0 = S_lev<R>(L, 0, hc, h);
        if (S <= S0) {
            Cidx = 0;
            S_low = S0;
            S_high = S_lev<R>(L, 1, hc, h);
        } else {
            const R Sn = S_lev<R>(L, top, hc, h);
            if (S >= Sn) {
                Cidx = top;
                S_low = Sn;
                S_high = S_lev<R>(L, top + 1, hc, h);
            } else {
                R s_lo = S0, s_hi = Sn;
                while (lo < hi - 1) {
                    const int mid = (lo + hi) / 2;
                    const R s_mid = S_lev<R>(L, mid, hc, h);
                    if (s_mid <= S) {
                        lo = mid;
                        s_lo = s_mid;
                    } else {
                        hi = mid;
                        s_hi = s_mid;
                    }
                }
                Cidx = lo;
                S_low = s_lo;
                S_high = (hi == lo + 1) ? s_hi : S_lev<R>(L, lo + 1, hc, h);
            }
        }
    }
    const R den = S_high - S_low;
    if (den == R(0)) return R(0);
    return (R)((R)Cidx - (R)L.C_offset) + (S - S_low) / den;
}

template <typename R>
__device__ __forceinline__ R compute_zidx_r(R z, R h, R zeta, R hc, const Levels &L, double hint) {
    const R den = zeta + h;
    const R S = den == R(0) ? R(0) : (z - zeta) / den;
    return zidx_search<R>(S, h, hc, L, hint);
}

// double z and zidx, evaluated in float64 for shallow columns, float32 elsewhere
__device__ __forceinline__ double compute_z_mixed(double zidx, int Nz, double hc, float h, float C, float zeta) {
    if (h < kShallow)
        return compute_z_r<double>(zidx, Nz, hc, (double)h, (double)C, (double)zeta);
    return (double)compute_z_r<float>((float)zidx, Nz, (float)hc, h, C, zeta);
}

__device__ __forceinline__ double compute_zidx_mixed(double z, float h, float zeta, double hc, const Levels &L,
                                                     double hint) {
    if (h < kShallow) return compute_zidx_r<double>(z, (double)h, (double)zeta, hc, L, hint);
    return (double)compute_zidx_r<float>((float)z, h, zeta, (float)hc, L, hint);
}

// ------------------------------------------------------------- per particle
struct FState {
    double zidx, z;
    CPos y, x;
    float k0x, k0y, k0z, k1x, k1y, k1z, k2x, k2y, k2z;
    float h_at, zeta_at;
    opb_time at;
    uint8_t status;
};

__device__ __forceinline__ bool same_time(const opb_time &a, const opb_time &b) {
    return a.prev == b.prev && a.next == b.next && a.ft == b.ft && a.gt == b.gt;
}

__device__ __forceinline__ uint8_t validate(uint8_t st, double zi, double yi, double xi, const double *b) {
    if (st & ST_INACTIVE) return st;
    if (!isfinite(zi) || !isfinite(yi) || !isfinite(xi)) return OPB_STATUS_NONFINITE;
    if (!(b[0] <= zi && zi <= b[1] && b[2] <= yi && yi <= b[3] && b[4] <= xi && xi <= b[5]))
        return OPB_STATUS_OUT_OF_DOMAIN;
    return st;
}

template <typename S, bool SCALED>
struct FBound {
    TDView<S, SCALED> u, v, w, zeta;
    StaticView dx, dy, h, C;
};

template <typename S, bool SCALED>
__device__ __forceinline__ FBound<S, SCALED> bind_all(const FRoms &r, const opb_time &t) {
    FBound<S, SCALED> b;
    b.u = bind_td<S, SCALED>(r.u, t);
    b.v = bind_td<S, SCALED>(r.v, t);
    b.w = bind_td<S, SCALED>(r.w, t);
    b.zeta = bind_td<S, SCALED>(r.zeta, t);
    b.dx = bind_static(r.dx);
    b.dy = bind_static(r.dy);
    b.h = bind_static(r.h);
    b.C = bind_static(r.C);
    return b;
}

// velocities in index space at (z, y, x): u/dx, v/dy, w.  false: zero spacing
template <typename B>
__device__ __forceinline__ bool velocity(const B &f, const CPos &z, const CPos &y, const CPos &x, float &kx, float &ky,
                                         float &kz) {
    const float u = trilinear(f.u, z, y, x);
    const float dx = bilinear_static(f.dx, y, x);
    const float v = trilinear(f.v, z, y, x);
    const float dy = bilinear_static(f.dy, y, x);
    if (dx == 0.0f || dy == 0.0f) return false;
    kx = u / dx;
    ky = v / dy;
    kz = trilinear(f.w, z, y, x);
    return true;
}

// ab3_w_advection.pyx:84-178 in float32
template <typename B>
__device__ __forceinline__ bool ab3_step(FState &s, const B &f, const FScalars &sc, bool reuse_hz) {
    const CPos zc = cpos(s.zidx);
    if (!velocity(f, zc, s.y, s.x, s.k0x, s.k0y, s.k0z)) return false;
    if (s.status == OPB_STATUS_MULTISTEP_1) {
        s.k1x = s.k2x = s.k0x;
        s.k1y = s.k2y = s.k0y;
        s.k1z = s.k2z = s.k0z;
        s.status = OPB_STATUS_MULTISTEP_2;
    } else if (s.status == OPB_STATUS_MULTISTEP_2) {
        s.k2x = -s.k0x + 2.0f * s.k1x;
        s.k2y = -s.k0y + 2.0f * s.k1y;
        s.k2z = -s.k0z + 2.0f * s.k1z;
        s.status = OPB_STATUS_NORMAL;
    }
    const float h = reuse_hz ? s.h_at : bilinear_static(f.h, s.y, s.x);
    const float zeta = reuse_hz ? s.zeta_at : bilinear_td(f.zeta, s.y, s.x);
    const float C = (float)linear_static_d(f.C, s.zidx);
    s.z = compute_z_mixed(s.zidx, sc.NZ, sc.hc, h, C, zeta);
    const float dt = (float)sc.dt;
    const float c = dt / 12.0f;
    s.z += (double)(c * (23.0f * s.k0z - 16.0f * s.k1z + 5.0f * s.k2z));
    cadd(s.y, c * (23.0f * s.k0y - 16.0f * s.k1y + 5.0f * s.k2y));
    cadd(s.x, c * (23.0f * s.k0x - 16.0f * s.k1x + 5.0f * s.k2x));
    s.k2x = s.k1x;
    s.k2y = s.k1y;
    s.k2z = s.k1z;
    s.k1x = s.k0x;
    s.k1y = s.k0y;
    s.k1z = s.k0z;
    return true;
}

// ab3_w_advection.pyx:214-229 in mixed precision
template <typename B>
__device__ __forceinline__ void ab3_post(FState &s, const B &f, const Levels &L, const FScalars &sc) {
    const float h = bilinear_static(f.h, s.y, s.x);
    const float zeta = bilinear_td(f.zeta, s.y, s.x);
    s.zidx = compute_zidx_mixed(s.z, h, zeta, sc.hc, L, s.zidx);
    s.h_at = h;
    s.zeta_at = zeta;
}

// rk2_w_advection.pyx:97-354 in float32: stage 1, stage 2, update
template <typename B>
__device__ __forceinline__ bool rk2_stage1(FState &s, const B &f, const FScalars &sc, bool reuse_hz) {
    const float h = reuse_hz ? s.h_at : bilinear_static(f.h, s.y, s.x);
    const float zeta = reuse_hz ? s.zeta_at : bilinear_td(f.zeta, s.y, s.x);
    const float C = (float)linear_static_d(f.C, s.zidx);
    s.z = compute_z_mixed(s.zidx, sc.NZ, sc.hc, h, C, zeta);
    return velocity(f, cpos(s.zidx), s.y, s.x, s.k1x, s.k1y, s.k1z);
}

template <typename B>
__device__ __forceinline__ bool rk2_stage2(FState &s, const B &f, const Levels &L, const FScalars &sc) {
    const float adt = (float)(sc.alpha * sc.dt);
    const double z_int = s.z + (double)(adt * s.k1z);
    CPos y_int = s.y, x_int = s.x;
    cadd(y_int, adt * s.k1y);
    cadd(x_int, adt * s.k1x);
    const float h = bilinear_static(f.h, y_int, x_int);
    const float zeta = bilinear_td(f.zeta, y_int, x_int);
    const double zi = compute_zidx_mixed(z_int, h, zeta, sc.hc, L, s.zidx);
    return velocity(f, cpos(zi), y_int, x_int, s.k2x, s.k2y, s.k2z);
}

template <typename B>
__device__ __forceinline__ void rk2_update(FState &s, const B &f, const Levels &L, const FScalars &sc) {
    const double b1 = 1.0 / (2.0 * sc.alpha);
    const float b1dt = (float)(b1 * sc.dt), b2dt = (float)((1.0 - b1) * sc.dt);
    s.z += (double)(b1dt * s.k1z + b2dt * s.k2z);
    cadd(s.y, b1dt * s.k1y + b2dt * s.k2y);
    cadd(s.x, b1dt * s.k1x + b2dt * s.k2x);
    const float h = bilinear_static(f.h, s.y, s.x);
    const float zeta = bilinear_td(f.zeta, s.y, s.x);
    s.zidx = compute_zidx_mixed(s.z, h, zeta, sc.hc, L, s.zidx);
    s.h_at = h;
    s.zeta_at = zeta;
}

// shared tables of the sigma levels and C (monotonicity decides the search)
#define FAST_LEVELS(r, sc)                                                                            \
    __shared__ double s_sigma[kMaxLevels];                                                            \
    __shared__ double s_C[kMaxLevels];                                                                \
    Levels L;                                                                                         \
    {                                                                                                 \
        const int C_size = (r).C.n0;                                                                  \
        const double *Cg = (const double *)(r).C.data[0];                                             \
        for (int k = threadIdx.x; k < C_size; k += blockDim.x) {                                      \
            s_sigma[k] = (sc).NZ == 0 ? 0.0 : (((double)k - (double)(r).C.o0) + 0.5) / (sc).NZ - 1.0; \
            s_C[k] = __ldg(Cg + k);                                                                   \
        }                                                                                             \
        __syncthreads();                                                                              \
        bool ok = (sc).NZ > 0;                                                                        \
        for (int k = threadIdx.x; k + 1 < C_size; k += blockDim.x)                                    \
            ok = ok && s_sigma[k] <= s_sigma[k + 1] && s_C[k] <= s_C[k + 1];                          \
        L.monotone = __syncthreads_and(ok) != 0;                                                      \
        L.sigma = s_sigma;                                                                            \
        L.C = s_C;                                                                                    \
        L.size = C_size;                                                                              \
        L.C_offset = (double)(r).C.o0;                                                                \
        L.Nz = (sc).NZ;                                                                               \
    }

__device__ __forceinline__ void raise_zero_division(const FParticles &p) {
    if (p.err) atomicOr(p.err, (uint32_t)OPB_ERRF_ZERO_DIVISION);
}

__device__ __forceinline__ void load_state(FState &s, const FParticles &p, long long i, bool history) {
    s.zidx = p.zidx[i];
    s.y = cpos(p.yidx[i]);
    s.x = cpos(p.xidx[i]);
    if (history) {
        s.k1x = (float)p.dxidx1[i];
        s.k1y = (float)p.dyidx1[i];
        s.k1z = (float)p.dz1[i];
        s.k2x = (float)p.dxidx2[i];
        s.k2y = (float)p.dyidx2[i];
        s.k2z = (float)p.dz2[i];
    }
}

template <typename S, bool SCALED>
__global__ void __launch_bounds__(kBlock, 2) k_ab3_steps_fp32(const __grid_constant__ FParticles p,
                                                              const __grid_constant__ FScalars sc,
                                                              const __grid_constant__ FRoms r,
                                                              const __grid_constant__ StepTable table, int nsteps,
                                                              int validate_pre) {
    FAST_LEVELS(r, sc);
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    FState s;
    s.status = p.status[i];
    if (s.status & ST_INACTIVE) return;
    load_state(s, p, i, true);
    const uint8_t st0 = s.status;
    bool moved = false;
    for (int k = 0; k < nsteps; ++k) {
        if (validate_pre) s.status = validate(s.status, s.zidx, cval(s.y), cval(s.x), sc.bounds);
        if (s.status & ST_INACTIVE) break;
        const opb_time t1 = table.at(2 * k), t2 = table.at(2 * k + 1);
        const bool reuse = k > 0 && same_time(t1, s.at);
        if (!ab3_step(s, bind_all<S, SCALED>(r, t1), sc, reuse)) {
            raise_zero_division(p);
            break;
        }
        moved = true;
        ab3_post(s, bind_all<S, SCALED>(r, t2), L, sc);
        s.at = t2;
    }
    if (s.status != st0) p.status[i] = s.status;
    if (!moved) return;
    p.zidx[i] = s.zidx;
    p.yidx[i] = cval(s.y);
    p.xidx[i] = cval(s.x);
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

template <typename S, bool SCALED>
__global__ void __launch_bounds__(kBlock, 2) k_rk2_steps_fp32(const __grid_constant__ FParticles p,
                                                              const __grid_constant__ FScalars sc,
                                                              const __grid_constant__ FRoms r,
                                                              const __grid_constant__ StepTable table, int nsteps,
                                                              int validate_pre) {
    FAST_LEVELS(r, sc);
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    FState s;
    s.status = p.status[i];
    if (s.status & ST_INACTIVE) return;
    load_state(s, p, i, false);
    const uint8_t st0 = s.status;
    bool moved = false;
    for (int k = 0; k < nsteps; ++k) {
        if (validate_pre) s.status = validate(s.status, s.zidx, cval(s.y), cval(s.x), sc.bounds);
        if (s.status & ST_INACTIVE) break;
        const opb_time t1 = table.at(3 * k), t2 = table.at(3 * k + 1), t3 = table.at(3 * k + 2);
        const bool reuse = k > 0 && same_time(t1, s.at);
        if (!rk2_stage1(s, bind_all<S, SCALED>(r, t1), sc, reuse)) {
            raise_zero_division(p);
            break;
        }
        moved = true;
        if (!rk2_stage2(s, bind_all<S, SCALED>(r, t2), L, sc)) {
            raise_zero_division(p);
            break;
        }
        rk2_update(s, bind_all<S, SCALED>(r, t3), L, sc);
        s.at = t3;
    }
    if (s.status != st0) p.status[i] = s.status;
    if (!moved) return;
    p.zidx[i] = s.zidx;
    p.yidx[i] = cval(s.y);
    p.xidx[i] = cval(s.x);
    p.z[i] = s.z;
    p.dxidx1[i] = s.k1x;
    p.dyidx1[i] = s.k1y;
    p.dz1[i] = s.k1z;
    p.dxidx2[i] = s.k2x;
    p.dyidx2[i] = s.k2y;
    p.dz2[i] = s.k2z;
}

// ------------------------------------------------------------ quantisation
// one block per (snapshot, level): max |value|
__global__ void __launch_bounds__(kBlock) k_level_absmax(const float *__restrict__ src, long long per_level,
                                                        float *__restrict__ scales) {
    const float *a = src + (long long)blockIdx.x * per_level;
    float m = 0.0f;
    for (long long j = threadIdx.x; j < per_level; j += blockDim.x) m = fmaxf(m, fabsf(a[j]));
    __shared__ float red[kBlock / 32];
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < kBlock / 32 ? red[threadIdx.x] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) scales[blockIdx.x] = (m > 0.0f && isfinite(m)) ? m / 32768.0f : 1.0f;
    }
}

template <typename S>
__device__ __forceinline__ S from_f(float v);
template <>
__device__ __forceinline__ __half from_f<__half>(float v) {
    return __float2half_rn(v);
}
template <>
__device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) {
    return __float2bfloat16_rn(v);
}

template <typename S>
__global__ void __launch_bounds__(kBlock) k_quantize(const float *__restrict__ src, long long per_level, long long total,
                                                    const float *__restrict__ scales, S *__restrict__ dst) {
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < total;
         j += (long long)gridDim.x * blockDim.x)
        dst[j] = from_f<S>(__fdiv_rn(src[j], scales[j / per_level]));  // IEEE division in this file too
}

// ------------------------------------------------------------------ host
int convert_particles(const opb_particles *in, FParticles &out, const char *what, bool ab3) {
    if (!in) return fail(OPB_EINVAL, "%s: particles is NULL", what);
    if (in->n < 0) return fail(OPB_EINVAL, "%s: negative particle count", what);
    if (in->n > 0) {
        const void *need[] = {in->status, in->zidx, in->yidx, in->xidx, in->z, in->dxidx1, in->dyidx1, in->dz1,
                              in->dxidx2, in->dyidx2, in->dz2};
        for (const void *q : need)
            if (!q) return fail(OPB_EINVAL, "%s: a required particle field is NULL", what);
        if (ab3 && (!in->dxidx0 || !in->dyidx0 || !in->dz0))
            return fail(OPB_EINVAL, "%s: a required particle field is NULL", what);
    }
    if ((in->n + kBlock - 1) / kBlock > 0x7fffffffLL) return fail(OPB_EINVAL, "%s: too many particles", what);
    out = FParticles{in->n, in->status, in->zidx, in->yidx, in->xidx, in->z, in->dxidx0, in->dyidx0, in->dz0,
                     in->dxidx1, in->dyidx1, in->dz1, in->dxidx2, in->dyidx2, in->dz2, in->err};
    return OPB_OK;
}

int convert_field(const opb_field &in, FField &out, int ndim, bool td, int *dtype, bool *scaled, const char *what,
                  const char *name) {
    if (in.ndim != ndim) return fail(OPB_EINVAL, "%s: field '%s' must have %d active dimensions", what, name, ndim);
    long long total = 1;
    int n[3] = {1, 1, 1};
    for (int d = 0; d < ndim; ++d) {
        if (in.shape[d] < 2) return fail(OPB_EINVAL, "%s: field '%s' dimension %d has size < 2", what, name, d);
        total *= in.shape[d];
        n[d] = (int)in.shape[d];
    }
    if (total >= 0x7fffffffLL) return fail(OPB_EINVAL, "%s: field '%s' has 2^31 elements or more", what, name);
    if (ndim == 3 && in.shape[0] > kMaxLevels && td && in.scale[0])
        return fail(OPB_EINVAL, "%s: field '%s' has too many levels", what, name);
    if (td) {
        if (in.is_static)
            return fail(OPB_EINVAL, "%s: the float32 steppers need '%s' time-dependent (the ROMS layout)", what, name);
        if (in.nslots < 2 || in.nslots > OPB_MAX_SLOTS)
            return fail(OPB_EINVAL, "%s: field '%s' has %d snapshot slots", what, name, in.nslots);
        if (in.dtype != OPB_F32 && in.dtype != OPB_BF16 && in.dtype != OPB_F16)
            return fail(OPB_EINVAL, "%s: field '%s': storage must be float32, bfloat16 or float16", what, name);
        const bool sc = in.scale[0] != nullptr;
        if (in.dtype != OPB_F32 && !sc)
            return fail(OPB_EINVAL, "%s: field '%s': bfloat16/float16 storage needs level scales", what, name);
        for (int k = 0; k < in.nslots; ++k) {
            if (!in.data[k]) return fail(OPB_EINVAL, "%s: field '%s' slot %d is NULL", what, name, k);
            if (sc != (in.scale[k] != nullptr))
                return fail(OPB_EINVAL, "%s: field '%s': scales must be given for every slot or none", what, name);
        }
        if (*dtype < 0) {
            *dtype = in.dtype;
            *scaled = sc;
        } else if (*dtype != in.dtype || *scaled != sc) {
            return fail(OPB_EINVAL, "%s: time-dependent fields must share one storage dtype and scaling", what);
        }
    } else {
        if (!in.is_static || in.dtype != OPB_F64 || !in.data[0])
            return fail(OPB_EINVAL, "%s: '%s' must be a static float64 field (the ROMS layout)", what, name);
    }
    for (int k = 0; k < OPB_MAX_SLOTS; ++k) {
        out.data[k] = in.data[k];
        out.scale[k] = td ? in.scale[k] : nullptr;
    }
    out.n0 = n[0];
    out.n1 = n[1];
    out.n2 = n[2];
    out.o0 = (float)in.offset[0];
    out.o1 = ndim > 1 ? (float)in.offset[1] : 0.0f;
    out.o2 = ndim > 2 ? (float)in.offset[2] : 0.0f;
    return OPB_OK;
}

int steps_fp32(const char *what, bool rk2, const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
               const opb_time *table, int32_t nsteps, int32_t validate_pre, void *stream) {
    FParticles fp;
    int rc;
    if ((rc = convert_particles(p, fp, what, !rk2))) return rc;
    if (!s) return fail(OPB_EINVAL, "%s: scalars is NULL", what);
    if (!f) return fail(OPB_EINVAL, "%s: fields is NULL", what);
    FScalars fs{s->hc, s->NZ, s->dt, s->alpha, {s->bounds[0], s->bounds[1], s->bounds[2], s->bounds[3],
                                                s->bounds[4], s->bounds[5]}};
    FRoms fr;
    int dtype = -1;
    bool scaled = false;
    if ((rc = convert_field(f->u, fr.u, 3, true, &dtype, &scaled, what, "u")) ||
        (rc = convert_field(f->v, fr.v, 3, true, &dtype, &scaled, what, "v")) ||
        (rc = convert_field(f->w, fr.w, 3, true, &dtype, &scaled, what, "w")) ||
        (rc = convert_field(f->zeta, fr.zeta, 2, true, &dtype, &scaled, what, "zeta")) ||
        (rc = convert_field(f->dx, fr.dx, 2, false, &dtype, &scaled, what, "dx")) ||
        (rc = convert_field(f->dy, fr.dy, 2, false, &dtype, &scaled, what, "dy")) ||
        (rc = convert_field(f->h, fr.h, 2, false, &dtype, &scaled, what, "h")) ||
        (rc = convert_field(f->C, fr.C, 1, false, &dtype, &scaled, what, "C")))
        return rc;
    if (fr.C.n0 > kMaxLevels) return fail(OPB_EINVAL, "%s: more than %d levels in C", what, kMaxLevels);
    if (nsteps < 0) return fail(OPB_EINVAL, "%s: negative step count", what);
    if (nsteps > 0 && !table) return fail(OPB_EINVAL, "%s: step table is NULL", what);
    if (fp.n == 0 || nsteps == 0) return OPB_OK;
    static thread_local StepTable tab;  // up to 17 KB: kept off the stack
    int nslots = 0;
    for (const opb_field *x : {&f->u, &f->v, &f->w, &f->zeta})
        if (!x->is_static && (nslots == 0 || x->nslots < nslots)) nslots = x->nslots;
    if ((rc = make_step_table(table, (long long)nsteps * (rk2 ? 3 : 2), tab, what, nslots))) return rc;
    const unsigned g = (unsigned)((fp.n + kBlock - 1) / kBlock);
    cudaStream_t st = (cudaStream_t)stream;
#define OPB_FAST_LAUNCH(S, SC)                                                                  \
    do {                                                                                        \
        if (rk2) k_rk2_steps_fp32<S, SC><<<g, kBlock, 0, st>>>(fp, fs, fr, tab, nsteps, validate_pre); \
        else k_ab3_steps_fp32<S, SC><<<g, kBlock, 0, st>>>(fp, fs, fr, tab, nsteps, validate_pre);     \
    } while (0)
    if (dtype == OPB_F32) {
        if (scaled) OPB_FAST_LAUNCH(float, true);
        else OPB_FAST_LAUNCH(float, false);
    } else if (dtype == OPB_BF16) {
        OPB_FAST_LAUNCH(__nv_bfloat16, true);
    } else {
        OPB_FAST_LAUNCH(__half, true);
    }
#undef OPB_FAST_LAUNCH
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    opb::clear_error();
    return OPB_OK;
}

}  // namespace
}  // namespace opb_fast

using namespace opb_fast;

extern "C" {

int opb_rk2_w_advection_steps_fp32(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                                   const opb_time *table, int32_t nsteps, int32_t validate, void *stream) {
    return steps_fp32("opb_rk2_w_advection_steps_fp32", true, p, s, f, table, nsteps, validate, stream);
}

int opb_ab3_w_advection_steps_fp32(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                                   const opb_time *table, int32_t nsteps, int32_t validate, void *stream) {
    return steps_fp32("opb_ab3_w_advection_steps_fp32", false, p, s, f, table, nsteps, validate, stream);
}

int opb_quantize_levels(const float *src, int64_t nsnap, int64_t nlev, int64_t per_level, int32_t dtype, void *dst,
                        float *scales, void *stream) {
    const char *what = "opb_quantize_levels";
    if (nsnap < 0 || nlev < 0 || per_level < 0) return fail(OPB_EINVAL, "%s: negative size", what);
    if (dtype != OPB_BF16 && dtype != OPB_F16) return fail(OPB_EINVAL, "%s: dtype must be bfloat16 or float16", what);
    const long long groups = nsnap * nlev;
    if (groups == 0 || per_level == 0) return OPB_OK;
    if (!src || !dst || !scales) return fail(OPB_EINVAL, "%s: NULL argument", what);
    if (groups > 0x7fffffffLL) return fail(OPB_EINVAL, "%s: too many levels", what);
    cudaStream_t st = (cudaStream_t)stream;
    k_level_absmax<<<(unsigned)groups, kBlock, 0, st>>>(src, per_level, scales);
    const long long total = groups * per_level;
    const unsigned g = (unsigned)((total + kBlock - 1) / kBlock < 148LL * 64 ? (total + kBlock - 1) / kBlock : 148 * 64);
    if (dtype == OPB_BF16) k_quantize<__nv_bfloat16><<<g, kBlock, 0, st>>>(src, per_level, total, scales, (__nv_bfloat16 *)dst);
    else k_quantize<__half><<<g, kBlock, 0, st>>>(src, per_level, total, scales, (__half *)dst);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    opb::clear_error();
    return OPB_OK;
}

}  // extern "C"
