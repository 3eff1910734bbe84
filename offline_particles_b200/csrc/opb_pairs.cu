// Snapshot pairs: two consecutive snapshots of a time-dependent field
// interleaved element by element (out[2i] = a[i], out[2i + 1] = b[i]), the
// layout in which the float64 steppers fetch both values of a time blend with
// one load.  Snapshot quads extend each pair with its x-neighbour's
// ({a[i], b[i], a[i+1], b[i+1]}: one 16-byte load per two stencil corners), and
// x-pairs do the same for a static float64 field ({s[i], s[i+1]}).  Octets
// (and yx-pairs) add the next row's two elements: one 32-byte load per stencil
// face.  Pure data movement at HBM bandwidth.
#include <cuda_runtime.h>

#include <cstdint>

#include "opb200.h"
#include "opb_errors.h"

namespace {

constexpr int kBlock = 256;

// float32: four elements of a and b per thread -> two float4 stores
__global__ void __launch_bounds__(kBlock) k_pairs_f32(const float4 *__restrict__ a, const float4 *__restrict__ b,
                                                      float4 *__restrict__ out, long long n4) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += (long long)gridDim.x * blockDim.x) {
        const float4 x = __ldg(a + q), y = __ldg(b + q);
        out[2 * q] = make_float4(x.x, y.x, x.y, y.y);
        out[2 * q + 1] = make_float4(x.z, y.z, x.w, y.w);
    }
}

// float64: two elements of a and b per thread -> two double2 stores
__global__ void __launch_bounds__(kBlock) k_pairs_f64(const double2 *__restrict__ a, const double2 *__restrict__ b,
                                                      double2 *__restrict__ out, long long n2) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n2; q += (long long)gridDim.x * blockDim.x) {
        const double2 x = __ldg(a + q), y = __ldg(b + q);
        out[2 * q] = make_double2(x.x, y.x);
        out[2 * q + 1] = make_double2(x.y, y.y);
    }
}

// the elements the vector kernels leave (n not a multiple of the vector width, or unaligned buffers)
template <typename T>
__global__ void __launch_bounds__(kBlock) k_pairs_tail(const T *__restrict__ a, const T *__restrict__ b,
                                                       T *__restrict__ out, long long first, long long n) {
    const long long i = first + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[2 * i] = a[i];
    out[2 * i + 1] = b[i];
}

// float32 quads: four elements per thread (one float4 of a and of b, plus the
// next element of each) -> four float4 stores; the caller handles the tail
__global__ void __launch_bounds__(kBlock) k_quads_f32(const float *__restrict__ a, const float *__restrict__ b,
                                                      float4 *__restrict__ out, long long n4, long long n) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += (long long)gridDim.x * blockDim.x) {
        const long long i = 4 * q;
        const float4 x = __ldg((const float4 *)a + q), y = __ldg((const float4 *)b + q);
        const long long j = i + 4 < n ? i + 4 : n - 1;
        const float xn = __ldg(a + j), yn = __ldg(b + j);
        out[i] = make_float4(x.x, y.x, x.y, y.y);
        out[i + 1] = make_float4(x.y, y.y, x.z, y.z);
        out[i + 2] = make_float4(x.z, y.z, x.w, y.w);
        out[i + 3] = make_float4(x.w, y.w, xn, yn);
    }
}

__global__ void __launch_bounds__(kBlock) k_quads_tail(const float *__restrict__ a, const float *__restrict__ b,
                                                       float4 *__restrict__ out, long long first, long long n) {
    const long long i = first + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long j = i + 1 < n ? i + 1 : n - 1;
    out[i] = make_float4(a[i], b[i], a[j], b[j]);
}

// float64 x-pairs, one element per thread
__global__ void __launch_bounds__(kBlock) k_xpairs_f64(const double *__restrict__ s, double2 *__restrict__ out,
                                                       long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long j = i + 1 < n ? i + 1 : n - 1;
        out[i] = make_double2(__ldg(s + i), __ldg(s + j));
    }
}

// float32 octets, one element per thread: the pairs of i, i+1, i+row, i+row+1
// (indices past the end clamped to n - 1) -> two float4 stores
__global__ void __launch_bounds__(kBlock) k_octets_f32(const float *__restrict__ a, const float *__restrict__ b,
                                                       float4 *__restrict__ out, long long n, long long row) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long last = n - 1;
        const long long i1 = i + 1 < n ? i + 1 : last;
        const long long i2 = i + row < n ? i + row : last;
        const long long i3 = i + row + 1 < n ? i + row + 1 : last;
        out[2 * i] = make_float4(__ldg(a + i), __ldg(b + i), __ldg(a + i1), __ldg(b + i1));
        out[2 * i + 1] = make_float4(__ldg(a + i2), __ldg(b + i2), __ldg(a + i3), __ldg(b + i3));
    }
}

// float64 yx-pairs, one element per thread -> two double2 stores
__global__ void __launch_bounds__(kBlock) k_yxpairs_f64(const double *__restrict__ s, double2 *__restrict__ out,
                                                        long long n, long long row) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long last = n - 1;
        const long long i1 = i + 1 < n ? i + 1 : last;
        const long long i2 = i + row < n ? i + row : last;
        const long long i3 = i + row + 1 < n ? i + row + 1 : last;
        out[2 * i] = make_double2(__ldg(s + i), __ldg(s + i1));
        out[2 * i + 1] = make_double2(__ldg(s + i2), __ldg(s + i3));
    }
}

// zeta-with-h bundles, one element per thread: {h[i], (a[i], b[i]), h[j], (a[j], b[j])} as 64-bit
// words, j = i + 1 (the last element's neighbour is itself) -> two 16-byte stores
__device__ __forceinline__ unsigned long long pack_pair(float lo, float hi) {
    return (unsigned long long)__float_as_uint(lo) | ((unsigned long long)__float_as_uint(hi) << 32);
}

__global__ void __launch_bounds__(kBlock) k_bundle_zeta_h(const float *__restrict__ a, const float *__restrict__ b,
                                                          const double *__restrict__ h, ulonglong2 *__restrict__ out,
                                                          long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long j = i + 1 < n ? i + 1 : n - 1;
        out[2 * i] = make_ulonglong2((unsigned long long)__double_as_longlong(__ldg(h + i)),
                                     pack_pair(__ldg(a + i), __ldg(b + i)));
        out[2 * i + 1] = make_ulonglong2((unsigned long long)__double_as_longlong(__ldg(h + j)),
                                         pack_pair(__ldg(a + j), __ldg(b + j)));
    }
}

// dx-with-dy bundles, one element per thread: {dx[i], dy[i], dx[j], dy[j]}, j = i + 1 (clamped)
__global__ void __launch_bounds__(kBlock) k_bundle_dx_dy(const double *__restrict__ dx, const double *__restrict__ dy,
                                                         double2 *__restrict__ out, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long j = i + 1 < n ? i + 1 : n - 1;
        out[2 * i] = make_double2(__ldg(dx + i), __ldg(dy + i));
        out[2 * i + 1] = make_double2(__ldg(dx + j), __ldg(dy + j));
    }
}

int grid_for(long long work) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long want = (work + kBlock - 1) / kBlock;
    const long long cap = (long long)sms * 8;  // 8 resident CTAs of 256 per SM
    return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

}  // namespace

extern "C" {

int opb_interleave_pairs(const void *a, const void *b, void *out, int64_t n, int32_t dtype, void *stream) {
    const char *what = "opb_interleave_pairs";
    if (n < 0) return opb::fail(OPB_EINVAL, "%s: negative element count", what);
    if (n == 0) return OPB_OK;
    if (!a || !b || !out) return opb::fail(OPB_EINVAL, "%s: NULL buffer", what);
    if (dtype != OPB_F32 && dtype != OPB_F64) return opb::fail(OPB_EINVAL, "%s: dtype must be OPB_F32 or OPB_F64", what);
    cudaStream_t st = (cudaStream_t)stream;
    const bool aligned = ((((uintptr_t)a) | ((uintptr_t)b) | ((uintptr_t)out)) & 15) == 0;
    long long done = 0;
    if (dtype == OPB_F32) {
        if (aligned) {
            const long long n4 = n / 4;
            if (n4) k_pairs_f32<<<grid_for(n4), kBlock, 0, st>>>((const float4 *)a, (const float4 *)b, (float4 *)out, n4);
            done = n4 * 4;
        }
        if (done < n)
            k_pairs_tail<float><<<(unsigned)((n - done + kBlock - 1) / kBlock), kBlock, 0, st>>>(
                (const float *)a, (const float *)b, (float *)out, done, n);
    } else {
        if (aligned) {
            const long long n2 = n / 2;
            if (n2) k_pairs_f64<<<grid_for(n2), kBlock, 0, st>>>((const double2 *)a, (const double2 *)b, (double2 *)out, n2);
            done = n2 * 2;
        }
        if (done < n)
            k_pairs_tail<double><<<(unsigned)((n - done + kBlock - 1) / kBlock), kBlock, 0, st>>>(
                (const double *)a, (const double *)b, (double *)out, done, n);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return opb::fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    opb::clear_error();
    return OPB_OK;
}

int opb_interleave_quads(const float *a, const float *b, float *out, int64_t n, void *stream) {
    const char *what = "opb_interleave_quads";
    if (n < 0) return opb::fail(OPB_EINVAL, "%s: negative element count", what);
    if (n == 0) return OPB_OK;
    if (!a || !b || !out) return opb::fail(OPB_EINVAL, "%s: NULL buffer", what);
    if (((uintptr_t)out) & 15) return opb::fail(OPB_EINVAL, "%s: out is not 16-byte aligned", what);
    cudaStream_t st = (cudaStream_t)stream;
    const bool aligned = ((((uintptr_t)a) | ((uintptr_t)b)) & 15) == 0;
    long long done = 0;
    if (aligned) {
        const long long n4 = n / 4;
        if (n4) k_quads_f32<<<grid_for(n4), kBlock, 0, st>>>(a, b, (float4 *)out, n4, n);
        done = n4 * 4;
    }
    if (done < n)
        k_quads_tail<<<(unsigned)((n - done + kBlock - 1) / kBlock), kBlock, 0, st>>>(a, b, (float4 *)out, done, n);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return opb::fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    opb::clear_error();
    return OPB_OK;
}

int opb_neighbour_pairs(const double *s, double *out, int64_t n, void *stream) {
    const char *what = "opb_neighbour_pairs";
    if (n < 0) return opb::fail(OPB_EINVAL, "%s: negative element count", what);
    if (n == 0) return OPB_OK;
    if (!s || !out) return opb::fail(OPB_EINVAL, "%s: NULL buffer", what);
    if (((uintptr_t)out) & 15) return opb::fail(OPB_EINVAL, "%s: out is not 16-byte aligned", what);
    k_xpairs_f64<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(s, (double2 *)out, n);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return opb::fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    opb::clear_error();
    return OPB_OK;
}

int opb_interleave_octets(const float *a, const float *b, float *out, int64_t n, int64_t row, void *stream) {
    const char *what = "opb_interleave_octets";
    if (n < 0 || row < 0) return opb::fail(OPB_EINVAL, "%s: negative element count or row length", what);
    if (n == 0) return OPB_OK;
    if (!a || !b || !out) return opb::fail(OPB_EINVAL, "%s: NULL buffer", what);
    if (((uintptr_t)out) & 31) return opb::fail(OPB_EINVAL, "%s: out is not 32-byte aligned", what);
    k_octets_f32<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(a, b, (float4 *)out, n, row);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return opb::fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    opb::clear_error();
    return OPB_OK;
}

int opb_neighbour_quads(const double *s, double *out, int64_t n, int64_t row, void *stream) {
    const char *what = "opb_neighbour_quads";
    if (n < 0 || row < 0) return opb::fail(OPB_EINVAL, "%s: negative element count or row length", what);
    if (n == 0) return OPB_OK;
    if (!s || !out) return opb::fail(OPB_EINVAL, "%s: NULL buffer", what);
    if (((uintptr_t)out) & 31) return opb::fail(OPB_EINVAL, "%s: out is not 32-byte aligned", what);
    k_yxpairs_f64<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(s, (double2 *)out, n, row);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return opb::fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    opb::clear_error();
    return OPB_OK;
}

int opb_bundle_zeta_h(const float *a, const float *b, const double *h, void *out, int64_t n, void *stream) {
    const char *what = "opb_bundle_zeta_h";
    if (n < 0) return opb::fail(OPB_EINVAL, "%s: negative element count", what);
    if (n == 0) return OPB_OK;
    if (!a || !b || !h || !out) return opb::fail(OPB_EINVAL, "%s: NULL buffer", what);
    if (((uintptr_t)out) & 31) return opb::fail(OPB_EINVAL, "%s: out is not 32-byte aligned", what);
    k_bundle_zeta_h<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(a, b, h, (ulonglong2 *)out, n);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return opb::fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    opb::clear_error();
    return OPB_OK;
}

int opb_bundle_dx_dy(const double *dx, const double *dy, double *out, int64_t n, void *stream) {
    const char *what = "opb_bundle_dx_dy";
    if (n < 0) return opb::fail(OPB_EINVAL, "%s: negative element count", what);
    if (n == 0) return OPB_OK;
    if (!dx || !dy || !out) return opb::fail(OPB_EINVAL, "%s: NULL buffer", what);
    if (((uintptr_t)out) & 31) return opb::fail(OPB_EINVAL, "%s: out is not 32-byte aligned", what);
    k_bundle_dx_dy<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(dx, dy, (double2 *)out, n);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return opb::fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    opb::clear_error();
    return OPB_OK;
}

}  // extern "C"
