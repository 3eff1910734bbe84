// Device building blocks of the ROMS advection step, shared by every kernel.
//
// Arithmetic follows the reference's Cython in operation order; the
// translation units that include this header are compiled with -fmad=false so
// that no multiply-add is contracted, which makes every result bit-identical
// to the reference's x86-64 build (gcc -O3, SSE2, no FMA).
#pragma once

#include <cstdint>

#include "opb200.h"

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

struct DRoms {
    DField u, v, w, dx, dy, h, zeta, C;
};

struct DParticles {
    long long n;
    uint8_t *status;
    double *zidx, *yidx, *xidx, *z;
    double *dxidx0, *dyidx0, *dz0;
    double *dxidx1, *dyidx1, *dz1;
    double *dxidx2, *dyidx2, *dz2;
    uint32_t *err;
};

struct DScalars {
    double hc;
    int NZ;
    double dt, alpha;
    double bounds[6];
};

// ------------------------------------------------------------------ fields
// A field bound to one time selection: FieldData(array, offsets) of
// fields.py:12 whose array is the blend prev*gt + next*ft (fields.py:426-428),
// evaluated per gathered element instead of over the whole grid.
template <typename T>
struct View {
    const T *prev;
    const T *next;
    const double *stat;  // non-null: static float64 field
    T ft, gt;
    long long n0, n1, n2;
    double o0, o1, o2;

    // fields.py:423-428: both products and their sum in the storage dtype,
    // then widened to float64 (np.add(..., out=float64, casting="unsafe")
    // adds in the inputs' dtype).
    __device__ __forceinline__ double at(long long i) const {
        if (stat) return __ldg(stat + i);
        const T a = __ldg(prev + i) * gt;
        const T b = __ldg(next + i) * ft;
        return (double)(a + b);
    }
};

template <typename T>
__device__ __forceinline__ View<T> bind(const DField &f, const opb_time &t) {
    View<T> v;
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
    v.n0 = f.n0;
    v.n1 = f.n1;
    v.n2 = f.n2;
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

// linear.pxd:11-17
template <typename F>
__device__ __forceinline__ double linear(const F &f, double idx) {
    const long long I0 = trunc_index(idx, f.n0 - 2);
    const double f0 = idx - (double)I0;
    const double g0 = 1.0 - f0;
    return g0 * f.at(I0) + f0 * f.at(I0 + 1);
}

// linear.pxd:19-33
template <typename F>
__device__ __forceinline__ double bilinear(const F &f, double idx0, double idx1) {
    const long long I0 = trunc_index(idx0, f.n0 - 2);
    const long long I1 = trunc_index(idx1, f.n1 - 2);
    const double f0 = idx0 - (double)I0;
    const double f1 = idx1 - (double)I1;
    const double g0 = 1.0 - f0;
    const double g1 = 1.0 - f1;
    const long long b = I0 * f.n1 + I1;
    const double v00 = f.at(b);
    const double v01 = f.at(b + 1);
    const double v10 = f.at(b + f.n1);
    const double v11 = f.at(b + f.n1 + 1);
    return g0 * g1 * v00 + g0 * f1 * v01 + f0 * g1 * v10 + f0 * f1 * v11;
}

// linear.pxd:35-65
template <typename F>
__device__ __forceinline__ double trilinear(const F &f, double idx0, double idx1, double idx2) {
    const long long I0 = trunc_index(idx0, f.n0 - 2);
    const long long I1 = trunc_index(idx1, f.n1 - 2);
    const long long I2 = trunc_index(idx2, f.n2 - 2);
    const double f0 = idx0 - (double)I0;
    const double f1 = idx1 - (double)I1;
    const double f2 = idx2 - (double)I2;
    const double g0 = 1.0 - f0;
    const double g1 = 1.0 - f1;
    const double g2 = 1.0 - f2;
    const long long s1 = f.n2;
    const long long s0 = f.n1 * f.n2;
    const long long b = I0 * s0 + I1 * s1 + I2;
    const double v000 = f.at(b);
    const double v001 = f.at(b + 1);
    const double v010 = f.at(b + s1);
    const double v011 = f.at(b + s1 + 1);
    const double v100 = f.at(b + s0);
    const double v101 = f.at(b + s0 + 1);
    const double v110 = f.at(b + s0 + s1);
    const double v111 = f.at(b + s0 + s1 + 1);
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

// S(k) of sigma level k of the C table
__device__ __forceinline__ double S_level(long long k, const double *C, double C_offset, int NZ, double hc, double h) {
    return S_coordinate(hc, sigma_from_Cidx(k, C_offset, NZ), h, __ldg(C + k));
}

// _vertical_coordinate.pxd:50-103: compute_zidx.  The binary search visits
// the same levels and makes the same comparisons as the reference; S(lo) and
// S(hi) are carried through the search so that the final interpolation reuses
// them (identical values: S_level is a pure function of the level).
__device__ __forceinline__ double compute_zidx(double z, double h, double zeta, double hc, int NZ, const double *C,
                                               long long C_size, double C_offset) {
    const double S = S_from_z(z, h, zeta);
    long long lo = 0, hi = C_size - 2;
    const double S0 = S_level(0, C, C_offset, NZ, hc, h);
    long long Cidx;
    double S_low, S_high;
    if (S <= S0) {
        Cidx = 0;
        S_low = S0;
        S_high = S_level(1, C, C_offset, NZ, hc, h);
    } else {
        const double Sn = S_level(C_size - 2, C, C_offset, NZ, hc, h);
        if (S >= Sn) {
            Cidx = C_size - 2;
            S_low = Sn;
            S_high = S_level(C_size - 1, C, C_offset, NZ, hc, h);
        } else {
            double S_lo = S0, S_hi = Sn;
            while (lo < hi - 1) {
                const long long mid = (lo + hi) / 2;
                const double S_mid = S_level(mid, C, C_offset, NZ, hc, h);
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
            S_high = (hi == lo + 1) ? S_hi : S_level(lo + 1, C, C_offset, NZ, hc, h);
        }
    }
    // _vertical_coordinate.pxd:86-96
    const double num = S - S_low;
    const double den = S_high - S_low;
    if (den == 0.0) return 0.0;
    const double f = num / den;
    return ((double)Cidx - C_offset) + f;
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
