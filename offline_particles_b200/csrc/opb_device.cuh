// Device building blocks of the ROMS advection step, shared by every kernel.
//
// Arithmetic follows the reference's Cython in operation order; the
// translation units that include this header are compiled with -fmad=false so
// that no multiply-add is contracted, which makes every result bit-identical
// to the reference's x86-64 build (gcc -O3, SSE2, no FMA).
#pragma once

#include <cstdint>

#include "opb200.h"
#include "opb_steptable.cuh"

namespace opb {

constexpr uint8_t ST_INACTIVE = OPB_STATUS_INACTIVE;
constexpr uint8_t ST_NORMAL = OPB_STATUS_NORMAL;
constexpr uint8_t ST_NONFINITE = OPB_STATUS_NONFINITE;
constexpr uint8_t ST_OUT_OF_DOMAIN = OPB_STATUS_OUT_OF_DOMAIN;
constexpr uint8_t ST_MULTISTEP_1 = OPB_STATUS_MULTISTEP_1;
constexpr uint8_t ST_MULTISTEP_2 = OPB_STATUS_MULTISTEP_2;

// ---------------------------------------------------------------- host-side
// structs passed by value as __grid_constant__ kernel parameters.
struct DField {
    const void *data[OPB_MAX_SLOTS];
    long long n0, n1, n2;  // active shape, slowest first (unused = 1)
    double o0, o1, o2;     // offsets of the active dimensions
    int is_static;         // 1: data[0] is float64 and time-invariant
};

// The ROMS field geometry (Arakawa C grid) on nz x ny x nx rho points: u on
// (nz, ny, nx - 1) at x offset -0.5, v on (nz, ny - 1, nx) at y offset -0.5,
// w on (nz + 1, ny, nx) at z offset +0.5 (w_centered: the field in the w slot
// sits on rho points, (nz, ny, nx), as the isopycnal follower's density does),
// zeta, h, dx, dy on (ny, nx) and C on nz levels, all other offsets 0.  The
// host sets `roms` when every field of a launch has exactly this geometry;
// the compiled-layout kernels then share one set of stencil axes per position
// across all fields.
struct DGeom {
    long long nz, ny, nx;
    long long su0, sv0, sw0;  // level strides of u (ny (nx - 1)), v ((ny - 1) nx) and w (ny nx)
    int roms;        // 1: the geometry above holds
    int w_centered;  // 1: the w slot is on rho points (nz, ny, nx), offsets 0
};

struct DRoms {
    DField u, v, w, dx, dy, h, zeta, C;
    DGeom geo;
};

struct DParticles {
    long long n;
    uint8_t *status;
    double *zidx, *yidx, *xidx, *z;
    double *dxidx0, *dyidx0, *dz0;
    double *dxidx1, *dyidx1, *dz1;
    double *dxidx2, *dyidx2, *dz2;
    uint32_t *err;
    const double *rho_t;
};

struct DScalars {
    double hc;
    int NZ;
    double dt, alpha;
    double bounds[6];
    double w_max, rho_scale;
};

// ------------------------------------------------------------------ fields
// A field bound to one time selection: FieldData(array, offsets) of
// fields.py:12 whose array is the blend prev*gt + next*ft (fields.py:426-428),
// evaluated per gathered element instead of over the whole grid.  `I` is the
// index type: int when every field has fewer than 2^31 elements (cheaper
// address arithmetic, fewer registers), else long long.
// Field kinds: KIND_ANY decides per access (static or time-dependent, known
// only at run time); KIND_STATIC / KIND_TD fix it at compile time, which lets
// the compiler drop the per-corner test (the ROMS layout: u, v, w, zeta
// time-dependent; h, dx, dy, C static).
// KIND_PAIRS: time-dependent, both snapshots of the blend interleaved in one
// buffer (element 2i earlier, 2i+1 later): one 8- or 16-byte load per corner.
// KIND_QUADS (float32 storage): time-dependent, element i holds {earlier[i],
// later[i], earlier[i+1], later[i+1]}: a stencil's two x-neighbouring corners
// with both snapshots of their blends in one 16-byte load.
// KIND_XPAIRS: static float64, element i holds {s[i], s[i+1]}: the two
// x-neighbouring corners in one 16-byte load.
// KIND_OCTS (float32 storage): time-dependent, element i holds the snapshot
// pairs of i, i+1, i+R, i+R+1 (R: the field's row length, its x size), so one
// 32-byte load fetches the four corners of a stencil face at one level.
// KIND_YXPAIRS: static float64, element i holds {s[i], s[i+1], s[i+R],
// s[i+R+1]}: a bilinear stencil in one 32-byte load.
constexpr int KIND_ANY = 0, KIND_STATIC = 1, KIND_TD = 2, KIND_PAIRS = 3, KIND_QUADS = 4, KIND_XPAIRS = 5,
              KIND_OCTS = 6, KIND_YXPAIRS = 7;

// How a launch reads its fields: plain snapshots, snapshot pairs, snapshot
// quads with x-pairs of the static fields h, dx, dy, or snapshot octets with
// yx-pairs of h, dx, dy.
constexpr int LAYOUT_PLAIN = 0, LAYOUT_PAIRS = 1, LAYOUT_QUADS = 2, LAYOUT_OCTS = 3;

// 32-byte read-only loads (sm_100: ld.global.nc.v4.f64 / .v4.u64); the
// address must be 32-byte aligned
struct alignas(32) D4 {
    double v[4];
};
__device__ __forceinline__ D4 ldg256(const D4 *p) {
    D4 r;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(r.v[0]), "=d"(r.v[1]), "=d"(r.v[2]), "=d"(r.v[3]) : "l"(p));
    return r;
}

// four 64-bit words: four float32 snapshot pairs, or h and zeta-pair words (2-D bundles)
struct alignas(32) U4 {
    unsigned long long v[4];
};
__device__ __forceinline__ U4 ldg256(const U4 *p) {
    U4 r;
    asm("ld.global.nc.v4.u64 {%0, %1, %2, %3}, [%4];" : "=l"(r.v[0]), "=l"(r.v[1]), "=l"(r.v[2]), "=l"(r.v[3]) : "l"(p));
    return r;
}

template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
    using type = float2;
};
template <>
struct Vec2<double> {
    using type = double2;
};

// The float32 time blend of one snapshot pair held as one 64-bit word
// {earlier (low half), later (high half)}, with w = {gt, ft}: both products in
// one packed multiply (mul.rn.f32x2 rounds each lane to nearest, exactly as
// two float32 multiplies do), then their float32 sum, widened to float64.
__device__ __forceinline__ double blend_word(unsigned long long pn, unsigned long long w) {
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pn), "l"(w));
    return (double)(__uint_as_float((unsigned)(r & 0xffffffffull)) + __uint_as_float((unsigned)(r >> 32)));
}

// {gt, ft} as one 64-bit word for blend_word
__device__ __forceinline__ unsigned long long blend_weights(float ft, float gt) {
    return (unsigned long long)__float_as_uint(gt) | ((unsigned long long)__float_as_uint(ft) << 32);
}

template <typename T, typename I, int KIND = KIND_ANY>
struct View {
    using index_type = I;
    static_assert((KIND != KIND_QUADS && KIND != KIND_OCTS) || sizeof(T) == 4,
                  "snapshot quads and octets hold float32 storage");
    const T *prev;
    const T *next;
    const double *stat;  // non-null: static float64 field
    T ft, gt;
    unsigned long long w;  // float32 storage: {gt, ft} for blend_word
    I n0, n1, n2;
    double o0, o1, o2;

    // fields.py:423-428: both products and their sum in the storage dtype,
    // then widened to float64 (np.add(..., out=float64, casting="unsafe")
    // adds in the inputs' dtype).
    __device__ __forceinline__ double blend(T a, T b) const {
        const T x = a * gt;
        const T y = b * ft;
        return (double)(x + y);
    }

    __device__ __forceinline__ double at(I i) const {
        if constexpr (KIND == KIND_YXPAIRS) {
            return __ldg(stat + 4 * (long long)i);
        } else if constexpr (KIND == KIND_OCTS) {
            return blend_word(__ldg((const unsigned long long *)prev + 4 * (long long)i), w);
        } else if constexpr (KIND == KIND_XPAIRS) {
            return __ldg(stat + 2 * (long long)i);
        } else if constexpr (KIND == KIND_QUADS) {
            return blend_word(__ldg((const unsigned long long *)prev + 2 * (long long)i), w);
        } else if constexpr (KIND == KIND_PAIRS && sizeof(T) == 4) {
            return blend_word(__ldg((const unsigned long long *)prev + i), w);
        } else if constexpr (KIND == KIND_PAIRS) {
            const typename Vec2<T>::type v = __ldg((const typename Vec2<T>::type *)prev + i);
            return blend(v.x, v.y);
        } else {
            if (KIND == KIND_STATIC || (KIND == KIND_ANY && stat)) return __ldg(stat + i);
            return blend(__ldg(prev + i), __ldg(next + i));
        }
    }

    // the values at i and i + 1 (x-neighbours: i + 1 stays in i's row for every
    // stencil, whose lowest corner index is clamped to n - 2)
    __device__ __forceinline__ void at2(I i, double &lo, double &hi) const {
        if constexpr (KIND == KIND_YXPAIRS) {
            const double2 v = __ldg((const double2 *)stat + 2 * (long long)i);
            lo = v.x;
            hi = v.y;
        } else if constexpr (KIND == KIND_OCTS) {
            const ulonglong2 v = __ldg((const ulonglong2 *)prev + 2 * (long long)i);
            lo = blend_word(v.x, w);
            hi = blend_word(v.y, w);
        } else if constexpr (KIND == KIND_XPAIRS) {
            const double2 v = __ldg((const double2 *)stat + i);
            lo = v.x;
            hi = v.y;
        } else if constexpr (KIND == KIND_QUADS) {
            const ulonglong2 v = __ldg((const ulonglong2 *)prev + i);
            lo = blend_word(v.x, w);
            hi = blend_word(v.y, w);
        } else {
            lo = at(i);
            hi = at(i + 1);
        }
    }

    // the values at i, i + 1, i + row, i + row + 1 (row: the field's x size; the
    // lowest corner's indices are clamped so that all four lie in the field)
    __device__ __forceinline__ void at4(I i, I row, double &v00, double &v01, double &v10, double &v11) const {
        if constexpr (KIND == KIND_YXPAIRS) {
            const D4 v = ldg256((const D4 *)stat + i);
            v00 = v.v[0];
            v01 = v.v[1];
            v10 = v.v[2];
            v11 = v.v[3];
        } else if constexpr (KIND == KIND_OCTS) {
            const U4 v = ldg256((const U4 *)prev + i);
            v00 = blend_word(v.v[0], w);
            v01 = blend_word(v.v[1], w);
            v10 = blend_word(v.v[2], w);
            v11 = blend_word(v.v[3], w);
        } else {
            at2(i, v00, v01);
            at2(i + row, v10, v11);
        }
    }
};

// ------------------------------------------------------ 2-D field bundles
// h, zeta, dx and dy share one stagger in the ROMS layout, so one bilinear
// stencil serves them all.  A bundle holds two of them element by element with
// the x-neighbour, 32 bytes per element, so one load fetches both fields' values
// at two corners:
//   zeta with h (zeta float32, time-dependent): {h[i], zeta pair[i], h[i+1],
//     zeta pair[i+1]} as four 64-bit words (a zeta pair: the earlier snapshot's
//     value in the low half, the later's in the high half);
//   dx with dy (static): {dx[i], dy[i], dx[i+1], dy[i+1]}.

template <typename I>
struct ZetaHView {
    using index_type = I;
    const U4 *p;
    float ft, gt;
    unsigned long long w;  // {gt, ft} for blend_word
    I n0, n1;
    double o0, o1;
    // the blend of one zeta pair word, as View::blend in float32
    __device__ __forceinline__ double zeta(unsigned long long pn) const { return blend_word(pn, w); }
    // h and zeta at i and i + 1
    __device__ __forceinline__ void at2(I i, double &h0, double &z0, double &h1, double &z1) const {
        const U4 w = ldg256(p + i);
        h0 = __longlong_as_double((long long)w.v[0]);
        z0 = zeta(w.v[1]);
        h1 = __longlong_as_double((long long)w.v[2]);
        z1 = zeta(w.v[3]);
    }
};

template <typename I>
struct DxDyView {
    using index_type = I;
    const D4 *p;
    I n0, n1;
    double o0, o1;
    // dx and dy at i and i + 1
    __device__ __forceinline__ void at2(I i, double &a0, double &b0, double &a1, double &b1) const {
        const D4 w = ldg256(p + i);
        a0 = w.v[0];
        b0 = w.v[1];
        a1 = w.v[2];
        b1 = w.v[3];
    }
};

template <typename T, typename I, int KIND = KIND_ANY>
__device__ __forceinline__ View<T, I, KIND> bind(const DField &f, const opb_time &t) {
    View<T, I, KIND> v;
    if (f.is_static) {
        v.stat = (const double *)f.data[0];
        v.prev = v.next = nullptr;
        v.ft = v.gt = T(0);
    } else {
        v.stat = nullptr;
        v.prev = (const T *)f.data[t.prev];
        v.next = (const T *)f.data[t.next];
        v.ft = (T)t.ft;  // exact: the host rounded ft, gt to the storage dtype
        v.gt = (T)t.gt;
    }
    if constexpr (sizeof(T) == 4) v.w = blend_weights((float)v.ft, (float)v.gt);
    v.n0 = (I)f.n0;
    v.n1 = (I)f.n1;
    v.n2 = (I)f.n2;
    v.o0 = f.o0;
    v.o1 = f.o1;
    v.o2 = f.o2;
    return v;
}

// ----------------------------------------------------------- interpolation
// kernels/_interpolation/linear.pxd:3-9.  The reference's `(Py_ssize_t)idx`
// is x86-64 cvttsd2si, which yields INT64_MIN for NaN and for values outside
// the int64 range; the clamp then maps those to 0.  CUDA's conversion
// saturates instead, so the out-of-range cases are mapped explicitly.
__device__ __forceinline__ long long trunc_index(double idx, long long max_idx) {
    long long i = (idx < 9.223372036854775808e18) ? (long long)idx : 0LL;  // NaN, +big -> 0
    if (i < 0) i = 0;
    else if (i > max_idx) i = max_idx;
    return i;
}

// The same map in 32-bit arithmetic, for max_idx < 2^31: anything that is not
// in [1, 2^63) (NaN, negatives, -inf, +huge) gives 0, [max_idx, 2^63) gives
// max_idx, and the rest truncates exactly as the 64-bit conversion does.
//
// Without branches: the saturating conversion (cvt.rzi.s32: toward zero,
// values past INT_MAX give INT_MAX) then min with max_idx gives (int)idx below
// max_idx and max_idx from there on (idx >= max_idx implies trunc(idx) >=
// max_idx, an integer); the range test selects 0 outside [1, 2^63).
__device__ __forceinline__ int trunc_index(double idx, int max_idx) {
    const bool in = idx >= 1.0 && idx < 9.223372036854775808e18;
    const int t = min(__double2int_rz(idx), max_idx);
    return in ? t : 0;
}

// linear.pxd:11-17
template <typename F>
__device__ __forceinline__ double linear(const F &f, double idx) {
    using I = typename F::index_type;
    const I I0 = trunc_index(idx, (I)(f.n0 - 2));
    const double f0 = idx - (double)I0;
    const double g0 = 1.0 - f0;
    double v0, v1;
    f.at2(I0, v0, v1);
    return g0 * v0 + f0 * v1;
}

// linear.pxd:19-33
template <typename F>
__device__ __forceinline__ double bilinear(const F &f, double idx0, double idx1) {
    using I = typename F::index_type;
    const I I0 = trunc_index(idx0, (I)(f.n0 - 2));
    const I I1 = trunc_index(idx1, (I)(f.n1 - 2));
    const double f0 = idx0 - (double)I0;
    const double f1 = idx1 - (double)I1;
    const double g0 = 1.0 - f0;
    const double g1 = 1.0 - f1;
    const I b = I0 * f.n1 + I1;
    double v00, v01, v10, v11;
    f.at4(b, f.n1, v00, v01, v10, v11);
    return g0 * g1 * v00 + g0 * f1 * v01 + f0 * g1 * v10 + f0 * f1 * v11;
}

// Two fields of one bundle on one stencil: each is bilinear() of its own values
// (the same weights, the same expression, so the same bits).
template <typename F>
__device__ __forceinline__ void bilinear_pair(const F &f, double idx0, double idx1, double &a, double &b) {
    using I = typename F::index_type;
    const I I0 = trunc_index(idx0, (I)(f.n0 - 2));
    const I I1 = trunc_index(idx1, (I)(f.n1 - 2));
    const double f0 = idx0 - (double)I0;
    const double f1 = idx1 - (double)I1;
    const double g0 = 1.0 - f0;
    const double g1 = 1.0 - f1;
    const I base = I0 * f.n1 + I1;
    double a00, b00, a01, b01, a10, b10, a11, b11;
    f.at2(base, a00, b00, a01, b01);
    f.at2(base + f.n1, a10, b10, a11, b11);
    a = g0 * g1 * a00 + g0 * f1 * a01 + f0 * g1 * a10 + f0 * f1 * a11;
    b = g0 * g1 * b00 + g0 * f1 * b01 + f0 * g1 * b10 + f0 * f1 * b11;
}

// linear.pxd:35-65
template <typename F>
__device__ __forceinline__ double trilinear(const F &f, double idx0, double idx1, double idx2) {
    using I = typename F::index_type;
    const I I0 = trunc_index(idx0, (I)(f.n0 - 2));
    const I I1 = trunc_index(idx1, (I)(f.n1 - 2));
    const I I2 = trunc_index(idx2, (I)(f.n2 - 2));
    const double f0 = idx0 - (double)I0;
    const double f1 = idx1 - (double)I1;
    const double f2 = idx2 - (double)I2;
    const double g0 = 1.0 - f0;
    const double g1 = 1.0 - f1;
    const double g2 = 1.0 - f2;
    const I s1 = f.n2;
    const I s0 = f.n1 * f.n2;
    const I b = I0 * s0 + I1 * s1 + I2;
    double v000, v001, v010, v011, v100, v101, v110, v111;
    f.at4(b, s1, v000, v001, v010, v011);
    f.at4(b + s0, s1, v100, v101, v110, v111);
    return (g0 * g1 * g2 * v000 +
            g0 * g1 * f2 * v001 +
            g0 * f1 * g2 * v010 +
            g0 * f1 * f2 * v011 +
            f0 * g1 * g2 * v100 +
            f0 * g1 * f2 * v101 +
            f0 * f1 * g2 * v110 +
            f0 * f1 * f2 * v111);
}

// ------------------------------------------------------ shared stencil axes
// One axis of a linear stencil (linear.pxd:3-9 for one dimension): the lower
// corner I = truncate_index(idx, max_idx), its weight f = idx - I and
// g = 1 - f.  Every stencil of a field is a product of such axes, so fields
// that sit on the same points in a dimension share that dimension's axis: the
// value is the same expression of the same inputs, hence the same bits.
template <typename I>
struct Axis {
    I i;
    double f, g;
};

template <typename I>
__device__ __forceinline__ Axis<I> make_axis(double idx, I max_idx) {
    Axis<I> a;
    a.i = trunc_index(idx, max_idx);
    a.f = idx - (double)a.i;
    a.g = 1.0 - a.f;
    return a;
}

// linear() over an axis of values read from `v` (any readable pointer, e.g. a
// shared-memory table): g0 * v[I0] + f0 * v[I0 + 1] (linear.pxd:11-17)
template <typename I>
__device__ __forceinline__ double linear_ax(const double *v, const Axis<I> &a) {
    return a.g * v[a.i] + a.f * v[a.i + 1];
}

// bilinear() over two axes; `row`: the field's x size (linear.pxd:19-33)
template <typename F, typename I>
__device__ __forceinline__ double bilinear_ax(const F &f, const Axis<I> &a0, const Axis<I> &a1, I row) {
    const double g0 = a0.g, f0 = a0.f, g1 = a1.g, f1 = a1.f;
    double v00, v01, v10, v11;
    f.at4(a0.i * row + a1.i, row, v00, v01, v10, v11);
    return g0 * g1 * v00 + g0 * f1 * v01 + f0 * g1 * v10 + f0 * f1 * v11;
}

// bilinear_pair() over two axes: both fields of a bundle on one stencil
template <typename F, typename I>
__device__ __forceinline__ void bilinear_pair_ax(const F &f, const Axis<I> &a0, const Axis<I> &a1, I row, double &a,
                                                 double &b) {
    const double g0 = a0.g, f0 = a0.f, g1 = a1.g, f1 = a1.f;
    const I base = a0.i * row + a1.i;
    double a00, b00, a01, b01, a10, b10, a11, b11;
    f.at2(base, a00, b00, a01, b01);
    f.at2(base + row, a10, b10, a11, b11);
    a = g0 * g1 * a00 + g0 * f1 * a01 + f0 * g1 * a10 + f0 * f1 * a11;
    b = g0 * g1 * b00 + g0 * f1 * b01 + f0 * g1 * b10 + f0 * f1 * b11;
}

// trilinear() over three axes; s0, s1: the field's level and row strides
// (linear.pxd:35-65)
template <typename F, typename I>
__device__ __forceinline__ double trilinear_ax(const F &f, const Axis<I> &a0, const Axis<I> &a1, const Axis<I> &a2,
                                               I s0, I s1) {
    const double g0 = a0.g, f0 = a0.f, g1 = a1.g, f1 = a1.f, g2 = a2.g, f2 = a2.f;
    const I b = a0.i * s0 + a1.i * s1 + a2.i;
    double v000, v001, v010, v011, v100, v101, v110, v111;
    f.at4(b, s1, v000, v001, v010, v011);
    f.at4(b + s0, s1, v100, v101, v110, v111);
    return (g0 * g1 * g2 * v000 +
            g0 * g1 * f2 * v001 +
            g0 * f1 * g2 * v010 +
            g0 * f1 * f2 * v011 +
            f0 * g1 * g2 * v100 +
            f0 * g1 * f2 * v101 +
            f0 * f1 * g2 * v110 +
            f0 * f1 * f2 * v111);
}

// ----------------------------------------------------- vertical coordinate
// kernels/roms/_vertical_coordinate.pxd.  A zero divisor makes the helper
// that divides return 0.0: that is what the reference's `noexcept nogil`
// helpers do under Cython's cdivision=False (the exception is printed as
// unraisable and the function returns 0).

// _vertical_coordinate.pxd:19-21
__device__ __forceinline__ double sigma_coordinate(double zidx, int Nz) {
    const double num = zidx + 0.5;
    if (Nz == 0) return 0.0;
    return num / (double)Nz - 1.0;
}

// _vertical_coordinate.pxd:23-25
__device__ __forceinline__ double S_coordinate(double hc, double sigma, double h, double C) {
    const double num = hc * sigma + h * C;
    const double den = hc + h;
    if (den == 0.0) return 0.0;
    return num / den;
}

// _vertical_coordinate.pxd:31-35
__device__ __forceinline__ double compute_z(double zidx, int Nz, double hc, double h, double C, double zeta) {
    const double sigma = sigma_coordinate(zidx, Nz);
    const double S = S_coordinate(hc, sigma, h, C);
    return zeta + (zeta + h) * S;
}

// _vertical_coordinate.pxd:41-43
__device__ __forceinline__ double S_from_z(double z, double h, double zeta) {
    const double num = z - zeta;
    const double den = zeta + h;
    if (den == 0.0) return 0.0;
    return num / den;
}

// _vertical_coordinate.pxd:45-48
__device__ __forceinline__ double sigma_from_Cidx(long long Cidx, double C_offset, int Nz) {
    const double zidx = (double)(int)Cidx - C_offset;
    return sigma_coordinate(zidx, Nz);
}

// The C levels the vertical search probes.  sigma_from_Cidx depends on the
// level only, so each block tabulates it (with C) in shared memory once:
// every probe then reads the same value the reference computes, minus one
// float64 division.  sigma == nullptr: compute on the fly from global C.
constexpr int kMaxLevels = 128;

struct Levels {
    const double *sigma;  // sigma_from_Cidx(k) for k < size, or nullptr
    const double *C;      // C[k]
    int size;             // C.shape[0]
    double C_offset;
    int Nz;
    bool monotone;        // sigma and C non-decreasing (checked on the device)
};

__device__ __forceinline__ double level_sigma(const Levels &L, int k) {
    return L.sigma ? L.sigma[k] : sigma_from_Cidx(k, L.C_offset, L.Nz);
}

// S(k) of sigma level k
__device__ __forceinline__ double S_level(const Levels &L, int k, double hc, double h) {
    return S_coordinate(hc, level_sigma(L, k), h, L.C[k]);
}

// Fill the shared tables and test monotonicity.  Every thread of the block
// must call this before any thread returns (it synchronises the block).
__device__ __forceinline__ Levels load_levels(const double *C_global, long long C_size, double C_offset, int Nz,
                                              double *s_sigma, double *s_C) {
    Levels L;
    L.size = (int)C_size;
    L.C_offset = C_offset;
    L.Nz = Nz;
    const bool fits = C_size <= kMaxLevels;
    if (fits) {
        for (int k = threadIdx.x; k < C_size; k += blockDim.x) {
            s_sigma[k] = sigma_from_Cidx(k, C_offset, Nz);
            s_C[k] = __ldg(C_global + k);
        }
        L.sigma = s_sigma;
        L.C = s_C;
    } else {
        L.sigma = nullptr;
        L.C = C_global;
    }
    __syncthreads();
    bool ok = fits && Nz > 0;
    if (fits)
        for (int k = threadIdx.x; k + 1 < C_size; k += blockDim.x)
            ok = ok && (s_sigma[k] <= s_sigma[k + 1]) && (s_C[k] <= s_C[k + 1]);
    L.monotone = __syncthreads_and(ok) != 0;
    return L;
}

// _vertical_coordinate.pxd:50-96 for a given S: the reference's binary
// search, visiting the same levels and making the same comparisons.  S(lo)
// and S(hi) are carried through the search so that the final interpolation
// reuses them (identical values: S_level is a pure function of the level).
__device__ __forceinline__ double zidx_from_S_search(double S, double h, double hc, const Levels &L) {
    const int C_size = L.size;
    int lo = 0, hi = C_size - 2;
    const double S0 = S_level(L, 0, hc, h);
    int Cidx;
    double S_low, S_high;
    if (S <= S0) {
        Cidx = 0;
        S_low = S0;
        S_high = S_level(L, 1, hc, h);
    } else {
        const double Sn = S_level(L, C_size - 2, hc, h);
        if (S >= Sn) {
            Cidx = C_size - 2;
            S_low = Sn;
            S_high = S_level(L, C_size - 1, hc, h);
        } else {
            double S_lo = S0, S_hi = Sn;
            while (lo < hi - 1) {
                const int mid = (lo + hi) / 2;
                const double S_mid = S_level(L, mid, hc, h);
                if (S_mid <= S) {
                    lo = mid;
                    S_lo = S_mid;
                } else {
                    hi = mid;
                    S_hi = S_mid;
                }
            }
            Cidx = lo;
            S_low = S_lo;
            // after the loop hi == lo + 1 unless the search never ran (hi <= lo + 1
            // from the start, i.e. C_size <= 3); recompute in that case
            S_high = (hi == lo + 1) ? S_hi : S_level(L, lo + 1, hc, h);
        }
    }
    // _vertical_coordinate.pxd:86-96
    const double num = S - S_low;
    const double den = S_high - S_low;
    if (den == 0.0) return 0.0;
    const double f = num / den;
    return ((double)Cidx - L.C_offset) + f;
}

// _vertical_coordinate.pxd:98-103: compute_zidx, as the reference computes it.
__device__ __forceinline__ double compute_zidx(double z, double h, double zeta, double hc, const Levels &L) {
    return zidx_from_S_search(S_from_z(z, h, zeta), h, hc, L);
}

// compute_zidx starting from a level hint (the particle's previous zidx).
//
// Same result as the reference's binary search, bit for bit.  When sigma and
// C are non-decreasing and hc, h >= 0 with hc + h > 0, every rounded S(k) =
// RN(RN(RN(hc sigma_k) + RN(h C_k)) / (hc + h)) is non-decreasing in k, and
// for S strictly between S(0) and S(C_size - 2) the binary search ends on the
// unique k with S(k) <= S < S(k + 1); at the ends it returns 0 for S <= S(0)
// (tested first) and C_size - 2 for S >= S(C_size - 2).  This function finds
// that same k by walking from the hint, which is almost always the right
// level already (particles move ~0.001 levels per step), so a call costs two
// S(k) evaluations instead of a whole search.  Anything outside those
// conditions -- a non-finite S or h, negative depths, a non-monotone table, a
// hint more than a few levels off -- runs the reference's search instead.
__device__ __forceinline__ double compute_zidx_hint(double z, double h, double zeta, double hc, const Levels &L,
                                                    double zidx_hint) {
    const double S = S_from_z(z, h, zeta);
    const int top = L.size - 2;
    if (!(L.monotone && top >= 1 && h >= 0.0 && hc >= 0.0 && hc + h > 0.0 && isfinite(S) && isfinite(h) &&
          isfinite(hc)))
        return zidx_from_S_search(S, h, hc, L);
    const double hk = zidx_hint + L.C_offset;
    int k = (hk >= 1.0 && hk < (double)top) ? (int)hk : (hk >= (double)top ? top : 0);
    constexpr int kMaxWalk = 3;
    int Cidx;
    double S_low, S_high;
    // S(k) and S(k + 1) are pure functions of the level: evaluated together, their divisions overlap
    // (the common case, the hint's own level, needs both)
    double lo_v = S_level(L, k, hc, h);
    const double up_v = S_level(L, k + 1, hc, h);  // k <= top, so k + 1 <= C_size - 1
    if (lo_v <= S && k < top && up_v > S) {
        Cidx = k;
        S_low = lo_v;
        S_high = up_v;
    } else if (lo_v > S) {  // walk down
        double hi_v = lo_v;
        int walked = 0;
        while (k > 0 && lo_v > S) {
            if (++walked > kMaxWalk) return zidx_from_S_search(S, h, hc, L);
            hi_v = lo_v;
            --k;
            lo_v = S_level(L, k, hc, h);
        }
        Cidx = k;
        S_low = lo_v;
        S_high = (walked > 0) ? hi_v : S_level(L, 1, hc, h);  // walked == 0 only when k == 0
    } else {  // walk up
        int walked = 0;
        for (;;) {
            if (k == top) {
                Cidx = top;
                S_low = lo_v;
                S_high = S_level(L, top + 1, hc, h);
                break;
            }
            const double hi_v = S_level(L, k + 1, hc, h);
            if (hi_v > S) {
                Cidx = k;
                S_low = lo_v;
                S_high = hi_v;
                break;
            }
            if (++walked > kMaxWalk) return zidx_from_S_search(S, h, hc, L);
            ++k;
            lo_v = hi_v;
        }
    }
    // the reference tests S <= S(0) first: on a plateau S(0) == ... == S(Cidx) == S it returns 0
    if (Cidx > 0 && S_low == S) {
        const double S0 = S_level(L, 0, hc, h);
        if (S <= S0) {
            Cidx = 0;
            S_low = S0;
            S_high = S_level(L, 1, hc, h);
        }
    }
    // _vertical_coordinate.pxd:86-96
    const double num = S - S_low;
    const double den = S_high - S_low;
    if (den == 0.0) return 0.0;
    const double f = num / den;
    return ((double)Cidx - L.C_offset) + f;
}

// x / 12.0 rounded to nearest, as the IEEE division gives it, in three
// floating-point operations: Markstein's correction step (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990; the final step of FMA-based
// division).  Theorem: if r is within half an ulp of 1/y and q within one ulp
// of x/y, then RN(q + RN(x - q y) r), with the remainder x - q y exact in an
// FMA, is RN(x/y).  Here y = 12 and r = RN(1/12) = (1/12)(1 - 2^-54) (RN(1/3)
// = (2^54 - 1) / (3 * 2^54)), so |x r - x/12| = |x/12| 2^-54 < ulp(x/12) / 2
// and q = RN(x r) is within one ulp.  Zeros (the sign of a zero quotient),
// infinities, NaN and magnitudes below 2^-960 (where the remainder could
// underflow) take the division itself.
__device__ __forceinline__ double div12(double x) {
    constexpr double kR = 0x1.5555555555555p-4;  // RN(1/12)
    if (!(fabs(x) >= 0x1p-960) || isinf(x)) return x / 12.0;
    const double q = x * kR;
    const double e = fma(-q, 12.0, x);
    return fma(e, kR, q);
}

// ----------------------------------------------------------------- status
__device__ __forceinline__ bool is_finite(double x) { return isfinite(x); }

// kernels/validation.pyx:21-77 for one active particle: finite_indices, then
// domain_bounds (validation_kernel = chain(finite, bounds), validation.pyx:124).
__device__ __forceinline__ uint8_t validate(uint8_t st, double zi, double yi, double xi, const double *b) {
    if (st & ST_INACTIVE) return st;
    if (!is_finite(zi) || !is_finite(yi) || !is_finite(xi)) return ST_NONFINITE;
    if (!(b[0] <= zi && zi <= b[1] && b[2] <= yi && yi <= b[3] && b[4] <= xi && xi <= b[5])) return ST_OUT_OF_DOMAIN;
    return st;
}

}  // namespace opb
