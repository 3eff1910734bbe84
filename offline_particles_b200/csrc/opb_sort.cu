// Spatial ordering of particles: Morton cell keys, radix sort, SoA gather.
//
// The advection kernels gather 8-corner stencils from fields far larger than
// L2.  Consecutive threads that hold spatially close particles share DRAM
// sectors and keep the in-flight working set in L2 across fused steps; this
// file produces that order.  Particles are independent, so the order changes
// no result -- only where each particle's state is stored.
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "opb200.h"
#include "opb_errors.h"
#include "opb_radix.cuh"

namespace opb_sort {
namespace {

constexpr int kBlock = 256;
constexpr uint32_t kInactiveKey = 0xFFFFFFFFu;
constexpr uint32_t kRangeKeyMask = 0x3FFFFFFFu;  // the cell key below the two range bits
constexpr int kMaxRanges = 4;

// spread the low 10 bits of v to every third bit
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ uint32_t cell(double idx, int n, int shift) {
    // the particle's cell, clamped into the grid (non-finite -> 0), quantised by 2^shift
    long long c = (idx >= 0.0 && idx < 9.0e18) ? (long long)idx : 0LL;
    if (c > n - 1) c = n - 1;
    return (uint32_t)(c >> shift);
}

struct KeyArgs {
    const uint8_t *status;
    const double *zidx, *yidx, *xidx;
    long long n;
    int nz, ny, nx;
    int sz, sy, sx;  // right shifts that bring each dimension under 2^10 (x additionally by 2)
    // id ranges kept in place (opb_sort_particles_ranges): with nbounds > 0 the particle whose id
    // (range_ids[i], or i without ids) is in [bound[r - 1], bound[r]) (bound[-1] = 0, bound[nbounds] =
    // n) sorts into the storage slots of that range
    const int64_t *range_ids;
    long long bound[kMaxRanges - 1];
    int nbounds;
};

__global__ void __launch_bounds__(kBlock) k_cell_keys(KeyArgs a, uint32_t *keys) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    uint32_t key = kInactiveKey;
    if (!(a.status[i] & OPB_STATUS_INACTIVE)) {
        const uint32_t z = cell(a.zidx[i], a.nz, a.sz);
        const uint32_t y = cell(a.yidx[i], a.ny, a.sy);
        const uint32_t x = cell(a.xidx[i], a.nx, a.sx);
        // x in the lowest bit of each triple: boxes of a Morton range are elongated along x,
        // the contiguous dimension of every field
        key = (spread3(z) << 2) | (spread3(y) << 1) | spread3(x);
    }
    if (a.nbounds > 0) {
        // the cell key fits 30 bits (three spread 10-bit values); the range index takes the top two, and
        // an inactive particle sorts last within its range
        const long long id = a.range_ids ? a.range_ids[i] : i;
        uint32_t r = 0;
        for (int j = 0; j < a.nbounds; ++j) r += id >= a.bound[j] ? 1u : 0u;
        key = (r << 30) | (key & kRangeKeyMask);
    }
    keys[i] = key;
}

struct GatherArgs {
    const uint8_t *s_status;
    uint8_t *d_status;
    const double *s[13];
    double *d[13];
    const int64_t *s_ids;
    int64_t *d_ids;
    int nf;
    long long n;
};

// d[j] = s[i] for every field of one particle.  All loads are issued before the first store: as far as the
// compiler knows the arrays may alias, so a loop of load-store pairs would wait out each load's latency in turn.
__device__ __forceinline__ void move_particle(const GatherArgs &a, long long i, long long j) {
    double v[13];
#pragma unroll
    for (int f = 0; f < 13; ++f)
        if (f < a.nf) v[f] = a.s[f][i];
    const uint8_t st = a.s_status[i];
    const int64_t id = a.d_ids ? a.s_ids[i] : 0;
#pragma unroll
    for (int f = 0; f < 13; ++f)
        if (f < a.nf) a.d[f][j] = v[f];
    a.d_status[j] = st;
    if (a.d_ids) a.d_ids[j] = id;
}

__global__ void __launch_bounds__(kBlock) k_gather(const __grid_constant__ GatherArgs a, const int32_t *perm) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= a.n) return;
    move_particle(a, perm[j], j);
}

int shift_for(int n, int extra) {
    int bits = 0;
    while ((1 << bits) < n) ++bits;
    int s = extra;
    while (bits - s > 10) ++s;
    return s;
}

using opb_radix::align256;

// ------------------------------------------------------------ segment sort
// Compact position q enumerates the segments' particles in storage order;
// seg_cstart[s] is the compact position of segment s's first particle.
struct SegArgs {
    KeyArgs k;
    const int64_t *seg_start;
    const int64_t *seg_cstart;
    int nseg;
    long long m;
};

__device__ __forceinline__ int segment_of(const int64_t *cstart, int nseg, long long q) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (cstart[mid] <= q) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(kBlock) k_segment_keys(SegArgs a, uint64_t *keys, int32_t *slot) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.m) return;
    const int s = segment_of(a.seg_cstart, a.nseg, q);
    const long long i = a.seg_start[s] + (q - a.seg_cstart[s]);
    uint32_t key = kInactiveKey;
    if (!(a.k.status[i] & OPB_STATUS_INACTIVE)) {
        const uint32_t z = cell(a.k.zidx[i], a.k.nz, a.k.sz);
        const uint32_t y = cell(a.k.yidx[i], a.k.ny, a.k.sy);
        const uint32_t x = cell(a.k.xidx[i], a.k.nx, a.k.sx);
        key = (spread3(z) << 2) | (spread3(y) << 1) | spread3(x);
    }
    keys[q] = ((uint64_t)s << 32) | key;
    slot[q] = (int32_t)i;
}

// scratch[q] <- arena[slot[perm[q]]]  (sorted compact order)
__global__ void __launch_bounds__(kBlock) k_segment_take(const __grid_constant__ GatherArgs a, const int32_t *perm,
                                                         const int32_t *slot) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.n) return;
    move_particle(a, slot[perm[q]], q);
}

// arena[slot[q]] <- scratch[q]
__global__ void __launch_bounds__(kBlock) k_segment_put(const __grid_constant__ GatherArgs a, const int32_t *slot) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.n) return;
    move_particle(a, q, slot[q]);
}

// bucket_bounds[s * (nb + 1) + b]: storage index of segment s's first particle
// whose cell key is >= b << shift (b = nb: the first inactive particle, or the
// segment's end).  Keys are sorted within the segment, so this is a lower bound.
__global__ void __launch_bounds__(kBlock) k_bucket_bounds(const uint64_t *keys, const int64_t *seg_start,
                                                          const int64_t *seg_cstart, long long m, int nseg, int nb,
                                                          int shift, int64_t *bounds) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nseg * (nb + 1)) return;
    const int s = (int)(t / (nb + 1));
    const int b = (int)(t % (nb + 1));
    const uint64_t threshold = b == nb ? 0x40000000ull : ((uint64_t)b << shift);
    long long lo = seg_cstart[s];
    long long hi = s + 1 < nseg ? seg_cstart[s + 1] : m;
    const long long first = lo;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if ((keys[mid] & 0xffffffffull) < threshold) lo = mid + 1;
        else hi = mid;
    }
    bounds[t] = seg_start[s] + (lo - first);
}

// right shift that leaves at most nb distinct buckets of the keys of this grid
int bucket_shift(const KeyArgs &k, int nb) {
    auto spread = [](uint32_t v) {
        uint32_t out = 0;
        for (int i = 0; i < 10; ++i) out |= ((v >> i) & 1u) << (3 * i);
        return out;
    };
    const uint32_t zmax = (uint32_t)((k.nz - 1) >> k.sz), ymax = (uint32_t)((k.ny - 1) >> k.sy);
    const uint32_t xmax = (uint32_t)((k.nx - 1) >> k.sx);
    // every key is below 2^bits, with bits the position of the top set bit of the largest key + 1
    const uint32_t top = (spread(zmax) << 2) | (spread(ymax) << 1) | spread(xmax);
    int bits = 0;
    while (bits < 32 && (top >> bits) != 0) ++bits;
    int lg = 0;
    while ((1 << lg) < nb) ++lg;
    return bits > lg ? bits - lg : 0;
}

// Pinned staging for small host tables copied to the device inside an
// asynchronous call: a copy from pageable memory would first wait for the
// stream to drain (CUDA's rule for pageable host-to-device copies), stalling
// the caller's host thread behind all queued work.  A ring of pinned slots per
// device; a slot is reused once the copy that last read it has completed.
struct PinnedRing {
    static constexpr int kSlots = 16;
    static constexpr size_t kSlotBytes = 1 << 20;
    char *host = nullptr;
    cudaEvent_t done[kSlots] = {};
    bool used[kSlots] = {};
    int next = 0;
};

// copy `bytes` from host `src` to device `dst` on stream st through pinned memory
cudaError_t stage_to_device(void *dst, const void *src, size_t bytes, cudaStream_t st) {
    static std::mutex mu;
    static std::map<int, PinnedRing> rings;
    if (bytes > PinnedRing::kSlotBytes) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    PinnedRing &R = rings[dev];
    if (!R.host) {
        e = cudaHostAlloc((void **)&R.host, PinnedRing::kSlots * PinnedRing::kSlotBytes, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            R.host = nullptr;
            return e;
        }
        for (int i = 0; i < PinnedRing::kSlots; ++i) {
            e = cudaEventCreateWithFlags(&R.done[i], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
    }
    const int k = R.next;
    R.next = (R.next + 1) % PinnedRing::kSlots;
    if (R.used[k] && (e = cudaEventSynchronize(R.done[k])) != cudaSuccess) return e;
    char *slot = R.host + (size_t)k * PinnedRing::kSlotBytes;
    std::memcpy(slot, src, bytes);
    if ((e = cudaMemcpyAsync(dst, slot, bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(R.done[k], st)) != cudaSuccess) return e;
    R.used[k] = true;
    return cudaSuccess;
}

int key_end_bit(int nseg) {
    int bits = 0;
    while ((1LL << bits) < (long long)nseg) ++bits;
    return 32 + bits;
}

// the pieces of a segment-sort workspace, in order
struct SegLayout {
    size_t keys_in, keys_out, ids_in, perm, slot, seg, status, fields, ids, temp, total;
};

SegLayout seg_layout(long long m, int nseg) {
    SegLayout L{};
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o += align256(bytes);
        return at;
    };
    L.keys_in = take((size_t)m * 8);
    L.keys_out = take((size_t)m * 8);
    L.ids_in = take((size_t)m * 4);
    L.perm = take((size_t)m * 4);
    L.slot = take((size_t)m * 4);
    L.seg = take((size_t)nseg * 16);
    L.status = take((size_t)m);
    L.fields = take((size_t)m * 8 * 13);
    L.ids = take((size_t)m * 8);
    L.temp = take(opb_radix::temp_bytes<uint64_t>(m));
    L.total = o;
    return L;
}

}  // namespace
}  // namespace opb_sort

using namespace opb_sort;
using opb::fail;

extern "C" {

size_t opb_sort_workspace_bytes(int64_t n) {
    if (n <= 0) return 0;
    return 3 * align256((size_t)n * 4) + opb_radix::temp_bytes<uint32_t>(n);
}

}  // extern "C"

namespace {

// opb_sort_particles, and with nranges > 1 opb_sort_particles_ranges (bounds: nranges + 1 host values)
int sort_particles(const char *what, const opb_particles *p, const int64_t shape[3], const int64_t *range_ids,
                   const int64_t *bounds, int nranges, int32_t *perm, void *workspace, size_t workspace_bytes,
                   void *stream) {
    if (!p) return fail(OPB_EINVAL, "%s: particles is NULL", what);
    if (p->n < 0 || p->n > 0x7fffffffLL) return fail(OPB_EINVAL, "%s: particle count out of range", what);
    if (p->n == 0) return OPB_OK;
    if (!p->status || !p->zidx || !p->yidx || !p->xidx || !perm || !shape)
        return fail(OPB_EINVAL, "%s: NULL argument", what);
    if (shape[0] < 1 || shape[1] < 1 || shape[2] < 1 || shape[0] > (1 << 30) || shape[1] > (1 << 30) ||
        shape[2] > (1 << 30))
        return fail(OPB_EINVAL, "%s: bad grid shape", what);
    if (nranges > 1) {
        if (!bounds || nranges > kMaxRanges) return fail(OPB_EINVAL, "%s: 1 to %d ranges", what, kMaxRanges);
        if (bounds[0] != 0 || bounds[nranges] != p->n)
            return fail(OPB_EINVAL, "%s: the range bounds must run from 0 to the particle count", what);
        for (int r = 0; r < nranges; ++r)
            if (bounds[r + 1] <= bounds[r]) return fail(OPB_EINVAL, "%s: the range bounds must increase", what);
    }
    const size_t need = opb_sort_workspace_bytes(p->n);
    if (!workspace || workspace_bytes < need)
        return fail(OPB_EINVAL, "%s: workspace of %zu bytes is smaller than the %zu needed", what,
                    workspace_bytes, need);
    const size_t a = align256((size_t)p->n * 4);
    char *ws = (char *)workspace;
    uint32_t *keys_in = (uint32_t *)ws;
    uint32_t *keys_out = (uint32_t *)(ws + a);
    int32_t *ids_in = (int32_t *)(ws + 2 * a);
    void *temp = ws + 3 * a;
    KeyArgs k{};
    k.status = p->status;
    k.zidx = p->zidx;
    k.yidx = p->yidx;
    k.xidx = p->xidx;
    k.n = p->n;
    k.nz = (int)shape[0];
    k.ny = (int)shape[1];
    k.nx = (int)shape[2];
    k.sz = shift_for(k.nz, 0);
    k.sy = shift_for(k.ny, 0);
    k.sx = shift_for(k.nx, 2);
    k.range_ids = range_ids;
    k.nbounds = nranges > 1 ? nranges - 1 : 0;
    for (int j = 0; j < k.nbounds; ++j) k.bound[j] = bounds[j + 1];
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned grid = (unsigned)((p->n + kBlock - 1) / kBlock);
    k_cell_keys<<<grid, kBlock, 0, st>>>(k, keys_in);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    e = opb_radix::radix_sort_index<uint32_t>(keys_in, keys_out, perm, ids_in, p->n, 32, temp, st, nullptr);
    if (e != cudaSuccess) return fail(OPB_ECUDA, "%s: radix sort: %s", what, cudaGetErrorString(e));
    opb::clear_error();
    return OPB_OK;
}

}  // namespace

extern "C" {

int opb_sort_particles(const opb_particles *p, const int64_t shape[3], int32_t *perm, void *workspace,
                       size_t workspace_bytes, void *stream) {
    return sort_particles("opb_sort_particles", p, shape, nullptr, nullptr, 1, perm, workspace, workspace_bytes,
                          stream);
}

int opb_sort_particles_ranges(const opb_particles *p, const int64_t shape[3], const int64_t *ids,
                              const int64_t *bounds, int32_t nranges, int32_t *perm, void *workspace,
                              size_t workspace_bytes, void *stream) {
    if (nranges < 1 || nranges > kMaxRanges || !bounds)
        return fail(OPB_EINVAL, "opb_sort_particles_ranges: 1 to %d ranges and their bounds", kMaxRanges);
    if (p && p->n > 0 && nranges == 1 && (bounds[0] != 0 || bounds[1] != p->n))
        return fail(OPB_EINVAL, "opb_sort_particles_ranges: the range bounds must run from 0 to the particle count");
    return sort_particles("opb_sort_particles_ranges", p, shape, ids, bounds, nranges, perm, workspace,
                          workspace_bytes, stream);
}

int opb_gather_particles(const opb_particles *src, const opb_particles *dst, const int32_t *perm,
                         const int64_t *src_ids, int64_t *dst_ids, void *stream) {
    if (!src || !dst || !perm) return fail(OPB_EINVAL, "opb_gather_particles: NULL argument");
    if (src->n != dst->n) return fail(OPB_EINVAL, "opb_gather_particles: particle counts differ");
    if (src->n < 0 || src->n > 0x7fffffffLL) return fail(OPB_EINVAL, "opb_gather_particles: bad particle count");
    if (src->n == 0) return OPB_OK;
    if (!src->status || !dst->status) return fail(OPB_EINVAL, "opb_gather_particles: status is NULL");
    if ((src_ids == nullptr) != (dst_ids == nullptr))
        return fail(OPB_EINVAL, "opb_gather_particles: give both id arrays or neither");
    GatherArgs g{};
    g.s_status = src->status;
    g.d_status = dst->status;
    const double *s[13] = {src->zidx, src->yidx, src->xidx, src->z, src->dxidx0, src->dyidx0, src->dz0,
                           src->dxidx1, src->dyidx1, src->dz1, src->dxidx2, src->dyidx2, src->dz2};
    double *d[13] = {dst->zidx, dst->yidx, dst->xidx, dst->z, dst->dxidx0, dst->dyidx0, dst->dz0,
                     dst->dxidx1, dst->dyidx1, dst->dz1, dst->dxidx2, dst->dyidx2, dst->dz2};
    int nf = 0;
    for (int f = 0; f < 13; ++f) {
        if ((s[f] == nullptr) != (d[f] == nullptr))
            return fail(OPB_EINVAL, "opb_gather_particles: source and destination fields differ");
        if (s[f]) {
            g.s[nf] = s[f];
            g.d[nf] = d[f];
            ++nf;
        }
    }
    g.nf = nf;
    g.n = src->n;
    g.s_ids = src_ids;
    g.d_ids = dst_ids;
    const unsigned grid = (unsigned)((src->n + kBlock - 1) / kBlock);
    k_gather<<<grid, kBlock, 0, (cudaStream_t)stream>>>(g, perm);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(OPB_ECUDA, "opb_gather_particles: %s", cudaGetErrorString(e));
    opb::clear_error();
    return OPB_OK;
}

size_t opb_sort_segments_workspace_bytes(int64_t total, int32_t nseg) {
    if (total <= 0 || nseg <= 0) return 0;
    return seg_layout(total, nseg).total;
}

int opb_sort_segments(const opb_particles *p, const int64_t shape[3], const int64_t *seg_start,
                      const int64_t *seg_count, int32_t nseg, int64_t *ids, int32_t nbuckets, int64_t *bucket_bounds,
                      void *workspace, size_t workspace_bytes, void *stream) {
    const char *what = "opb_sort_segments";
    if (!p) return fail(OPB_EINVAL, "%s: particles is NULL", what);
    if (p->n < 0 || p->n > 0x7fffffffLL) return fail(OPB_EINVAL, "%s: particle count out of range", what);
    if (nseg < 0) return fail(OPB_EINVAL, "%s: negative segment count", what);
    if (nseg == 0 || p->n == 0) return OPB_OK;
    if (!seg_start || !seg_count || !shape) return fail(OPB_EINVAL, "%s: NULL argument", what);
    if (bucket_bounds && (nbuckets < 1 || nbuckets > 65536 || (nbuckets & (nbuckets - 1))))
        return fail(OPB_EINVAL, "%s: nbuckets must be a power of two in [1, 65536]", what);
    if (!p->status || !p->zidx || !p->yidx || !p->xidx) return fail(OPB_EINVAL, "%s: NULL particle array", what);
    if (shape[0] < 1 || shape[1] < 1 || shape[2] < 1 || shape[0] > (1 << 30) || shape[1] > (1 << 30) ||
        shape[2] > (1 << 30))
        return fail(OPB_EINVAL, "%s: bad grid shape", what);
    // host-side checks: disjoint ascending in-range segments
    long long m = 0, end = 0;
    for (int s = 0; s < nseg; ++s) {
        if (seg_count[s] < 0 || seg_start[s] < end || seg_start[s] + seg_count[s] > p->n)
            return fail(OPB_EINVAL, "%s: segment %d [%lld, +%lld) is out of order or out of range", what, s,
                        (long long)seg_start[s], (long long)seg_count[s]);
        end = seg_start[s] + seg_count[s];
        m += seg_count[s];
    }
    if (m == 0) return OPB_OK;
    const SegLayout L = seg_layout(m, nseg);
    if (!workspace || workspace_bytes < L.total)
        return fail(OPB_EINVAL, "%s: workspace of %zu bytes is smaller than the %zu needed", what, workspace_bytes,
                    L.total);
    char *ws = (char *)workspace;
    cudaStream_t st = (cudaStream_t)stream;
    // segment table (start, compact start) -> device
    std::vector<int64_t> seg(2 * (size_t)nseg);
    long long c = 0;
    for (int s = 0; s < nseg; ++s) {
        seg[s] = seg_start[s];
        seg[nseg + s] = c;
        c += seg_count[s];
    }
    cudaError_t e = stage_to_device(ws + L.seg, seg.data(), seg.size() * 8, st);
    if (e != cudaSuccess) return fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    SegArgs a{};
    a.k.status = p->status;
    a.k.zidx = p->zidx;
    a.k.yidx = p->yidx;
    a.k.xidx = p->xidx;
    a.k.n = p->n;
    a.k.nz = (int)shape[0];
    a.k.ny = (int)shape[1];
    a.k.nx = (int)shape[2];
    a.k.sz = shift_for(a.k.nz, 0);
    a.k.sy = shift_for(a.k.ny, 0);
    a.k.sx = shift_for(a.k.nx, 2);
    a.seg_start = (const int64_t *)(ws + L.seg);
    a.seg_cstart = a.seg_start + nseg;
    a.nseg = nseg;
    a.m = m;
    uint64_t *keys_in = (uint64_t *)(ws + L.keys_in);
    uint64_t *keys_out = (uint64_t *)(ws + L.keys_out);
    int32_t *ids_in = (int32_t *)(ws + L.ids_in);
    int32_t *perm = (int32_t *)(ws + L.perm);
    int32_t *slot = (int32_t *)(ws + L.slot);
    const unsigned grid = (unsigned)((m + kBlock - 1) / kBlock);
    k_segment_keys<<<grid, kBlock, 0, st>>>(a, keys_in, slot);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    uint64_t *keys_sorted = nullptr;
    e = opb_radix::radix_sort_index<uint64_t>(keys_in, keys_out, perm, ids_in, m, key_end_bit(nseg), ws + L.temp, st,
                                              &keys_sorted);
    if (e != cudaSuccess) return fail(OPB_ECUDA, "%s: radix sort: %s", what, cudaGetErrorString(e));
    // arena -> scratch in sorted order -> arena
    const double *arena[13] = {p->zidx, p->yidx, p->xidx, p->z, p->dxidx0, p->dyidx0, p->dz0,
                               p->dxidx1, p->dyidx1, p->dz1, p->dxidx2, p->dyidx2, p->dz2};
    GatherArgs take{}, put{};
    take.s_status = p->status;
    take.d_status = (uint8_t *)(ws + L.status);
    put.s_status = take.d_status;
    put.d_status = p->status;
    int nf = 0;
    for (int f = 0; f < 13; ++f) {
        if (!arena[f]) continue;
        double *buf = (double *)(ws + L.fields) + (size_t)nf * m;
        take.s[nf] = arena[f];
        take.d[nf] = buf;
        put.s[nf] = buf;
        put.d[nf] = (double *)arena[f];
        ++nf;
    }
    take.nf = put.nf = nf;
    take.n = put.n = m;
    if (ids) {
        take.s_ids = ids;
        take.d_ids = (int64_t *)(ws + L.ids);
        put.s_ids = take.d_ids;
        put.d_ids = ids;
    }
    k_segment_take<<<grid, kBlock, 0, st>>>(take, perm, slot);
    k_segment_put<<<grid, kBlock, 0, st>>>(put, slot);
    if (bucket_bounds) {
        const long long nt = (long long)nseg * (nbuckets + 1);
        k_bucket_bounds<<<(unsigned)((nt + kBlock - 1) / kBlock), kBlock, 0, st>>>(
            keys_sorted, a.seg_start, a.seg_cstart, m, nseg, nbuckets, bucket_shift(a.k, nbuckets), bucket_bounds);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    opb::clear_error();
    return OPB_OK;
}

}  // extern "C"

// ====================================================================== no-alloc
// opb_sort_particles_noalloc: the same sort with its scratch in a static
// device array, for callers that cannot allocate device memory when they
// sort.  Sizes are stated in include/opb200.h (OPB_NOALLOC_*).
//
// Layout of the array: two key buffers and one id buffer of
// OPB_NOALLOC_MAX_PARTICLES entries each (the radix sort's double buffers; the
// caller's perm is the other id buffer), then OPB_NOALLOC_SORT_TEMP_BYTES for
// the radix sort's tile counts.
namespace opb_sort {
namespace {

constexpr size_t kNoAllocBuf = (size_t)OPB_NOALLOC_MAX_PARTICLES * 4;
constexpr size_t kNoAllocTempOffset = 3 * kNoAllocBuf;
static_assert(kNoAllocTempOffset + OPB_NOALLOC_SORT_TEMP_BYTES == OPB_NOALLOC_SCRATCH_BYTES, "scratch layout");

// Every GPU that loads this library holds this array until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[OPB_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[kMaxDevices] = {};

// Device address of the array on the current device.  In host code the
// array's name is only a host-side stand-in, never a device address; the
// runtime maps it the first time, once per device (which may load the module).
// Outside stream capture the address is looked up again on every call (a
// cheap table lookup once the module is loaded), so a context that was reset
// and re-created (cudaDeviceReset) never leaves a stale address behind;
// during capture the address cached by an earlier call is used.
int noalloc_scratch(void **out, cudaStream_t stream) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(OPB_ECUDA, "opb_sort_particles_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(OPB_EINVAL, "opb_sort_particles_noalloc: device %d out of range", dev);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess) {
        (void)cudaGetLastError();  // e.g. the legacy stream queried while another stream captures
        cap = cudaStreamCaptureStatusActive;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (cap != cudaStreamCaptureStatusActive || !g_noalloc_ptr[dev]) {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(OPB_ECUDA, "opb_sort_particles_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        g_noalloc_ptr[dev] = ptr;
    }
    *out = g_noalloc_ptr[dev];
    return OPB_OK;
}

}  // namespace
}  // namespace opb_sort

extern "C" int opb_sort_particles_noalloc(const opb_particles *p, const int64_t shape[3], int32_t *perm,
                                          void *stream) {
    if (!p) return fail(OPB_EINVAL, "opb_sort_particles_noalloc: particles is NULL");
    if (p->n < 0) return fail(OPB_EINVAL, "opb_sort_particles_noalloc: negative particle count");
    if (p->n > OPB_NOALLOC_MAX_PARTICLES)
        return fail(OPB_EINVAL,
                    "opb_sort_particles_noalloc: %lld particles exceed the static scratch limit of %d "
                    "(OPB_NOALLOC_MAX_PARTICLES); use opb_sort_particles with a caller-allocated workspace",
                    (long long)p->n, (int)OPB_NOALLOC_MAX_PARTICLES);
    if (p->n == 0) return OPB_OK;
    if (!p->status || !p->zidx || !p->yidx || !p->xidx || !perm || !shape)
        return fail(OPB_EINVAL, "opb_sort_particles_noalloc: NULL argument");
    if (shape[0] < 1 || shape[1] < 1 || shape[2] < 1 || shape[0] > (1 << 30) || shape[1] > (1 << 30) ||
        shape[2] > (1 << 30))
        return fail(OPB_EINVAL, "opb_sort_particles_noalloc: bad grid shape");
    void *base = nullptr;
    int rc = noalloc_scratch(&base, (cudaStream_t)stream);
    if (rc) return rc;
    char *ws = (char *)base;
    uint32_t *keys0 = (uint32_t *)ws;
    uint32_t *keys1 = (uint32_t *)(ws + kNoAllocBuf);
    int32_t *ids = (int32_t *)(ws + 2 * kNoAllocBuf);
    void *temp = ws + kNoAllocTempOffset;
    const long long n = p->n;
    const size_t temp_bytes = opb_radix::temp_bytes<uint32_t>(n);
    if (temp_bytes > OPB_NOALLOC_SORT_TEMP_BYTES)
        return fail(OPB_EINVAL, "opb_sort_particles_noalloc: radix sort needs %zu temporary bytes, the static "
                    "scratch reserves %zu", temp_bytes, (size_t)OPB_NOALLOC_SORT_TEMP_BYTES);
    KeyArgs k{};
    k.status = p->status;
    k.zidx = p->zidx;
    k.yidx = p->yidx;
    k.xidx = p->xidx;
    k.n = p->n;
    k.nz = (int)shape[0];
    k.ny = (int)shape[1];
    k.nx = (int)shape[2];
    k.sz = shift_for(k.nz, 0);
    k.sy = shift_for(k.ny, 0);
    k.sx = shift_for(k.nx, 2);
    cudaStream_t st = (cudaStream_t)stream;
    // keys0 is written in full before the sort reads it; every pass of the sort writes its outputs and its
    // tile counts in full before reading them, so no buffer of the array needs initial contents
    k_cell_keys<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock, 0, st>>>(k, keys0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(OPB_ECUDA, "opb_sort_particles_noalloc: %s", cudaGetErrorString(e));
    e = opb_radix::radix_sort_index<uint32_t>(keys0, keys1, perm, ids, n, 32, temp, st, nullptr);
    if (e != cudaSuccess) return fail(OPB_ECUDA, "opb_sort_particles_noalloc: radix sort: %s", cudaGetErrorString(e));
    opb::clear_error();
    return OPB_OK;
}
