// Batched release experiments for B200 (sm_100a): one persistent launch
// advances many releases, each in its own contiguous segment of a particle
// arena.  Compiled with -fmad=false like opb_roms.cu: the per-particle work is
// the same stage functions (opb_stages.cuh), so every release's results are
// bit-identical to the fused single-release steppers.
#include <cuda_runtime.h>

#include <type_traits>

#include "opb200.h"
#include "opb_device.cuh"
#include "opb_errors.h"
#include "opb_host.cuh"
#include "opb_stages.cuh"

// 1: the batched kernels keep the velocity history in shared memory (PState HS):
// measured 3 % faster than registers on config 4 (fewer spills at 128 registers)
#ifndef OPB_BATCH_HIST_SMEM
#define OPB_BATCH_HIST_SMEM 1
#endif
// Chunks a warp claims at once (and advances one after another): consecutive
// chunks lie in one Morton bucket, so claiming several keeps one region's
// field data in this SM's L1
#ifndef OPB_BATCH_CLAIM
#define OPB_BATCH_CLAIM 1
#endif

namespace opb {
namespace {

// One particle of experiment E through E.nsteps steps of its scheme: the loop
// bodies of k_rk2_steps / k_ab3_steps (opb_roms.cu) with E's dt, alpha and
// time table, reading the time-dependent fields as snapshot pairs or quads
// (LAYOUT).  SCHEME: OPB_SCHEME_RK2 or OPB_SCHEME_AB3 compiles one scheme only
// (smaller code, fewer live registers); 0 decides per experiment.
template <typename T, typename I, int SCHEME, int LAYOUT, bool B2>
__device__ __forceinline__ void batched_particle(const DParticles &p, long long i, const opb_experiment &E,
                                                 const DScalars &sc0, const DRoms &r, const opb_time *table,
                                                 const Levels &L, double *hs, int hstride) {
    constexpr bool HS = OPB_BATCH_HIST_SMEM != 0;
    PState<I, HS> s;
    s.hs = hs;
    s.hstride = hstride;
    s.status = p.status[i];
    if (s.status & ST_INACTIVE) return;
    DScalars sc = sc0;
    sc.dt = E.dt;
    sc.alpha = E.alpha;
    s.zidx = p.zidx[i];
    s.yidx = p.yidx[i];
    s.xidx = p.xidx[i];
    const bool ab3 = SCHEME == OPB_SCHEME_AB3 || (SCHEME == 0 && E.scheme == OPB_SCHEME_AB3);
    if (ab3) {
        s.set_k1(p.dxidx1[i], p.dyidx1[i], p.dz1[i]);
        s.set_k2(p.dxidx2[i], p.dyidx2[i], p.dz2[i]);
    }
    const uint8_t st0 = s.status;
    bool moved = false;
    const opb_time *tab = table + E.table_offset;
    for (int k = 0; k < E.nsteps; ++k) {
        if (E.validate) s.status = validate(s.status, s.zidx, s.yidx, s.xidx, sc.bounds);
        if (s.status & ST_INACTIVE) break;
        if (ab3) {
            const opb_time t1 = tab[2 * k], t2 = tab[2 * k + 1];
            const bool reuse = k > 0 && same_time(t1, tab[2 * k - 1]);  // the last post step's time
            if (!ab3_step(s, bind_all<T, I, true, LAYOUT, B2>(r, t1), sc, L, reuse, k > 0)) {
                raise_zero_division(p);
                break;
            }
            moved = true;
            ab3_post(s, bind_all<T, I, true, LAYOUT, B2>(r, t2), L, sc);
        } else {
            const opb_time t1 = tab[3 * k], t2 = tab[3 * k + 1], t3 = tab[3 * k + 2];
            const bool reuse = k > 0 && same_time(t1, tab[3 * k - 1]);  // the last update's time
            if (!rk2_stage1(s, bind_all<T, I, true, LAYOUT, B2>(r, t1), sc, L, reuse, k > 0)) {
                raise_zero_division(p);
                break;
            }
            moved = true;
            if (!rk2_stage2(s, bind_all<T, I, true, LAYOUT, B2>(r, t2), L, sc)) {
                raise_zero_division(p);
                break;
            }
            rk2_update(s, bind_all<T, I, true, LAYOUT, B2>(r, t3), L, sc);
        }
    }
    if (s.status != st0) p.status[i] = s.status;
    if (!moved) return;
    p.zidx[i] = s.zidx;
    p.yidx[i] = s.yidx;
    p.xidx[i] = s.xidx;
    p.z[i] = s.z;
    if (ab3) {
        s.get_k1(p.dxidx0[i], p.dyidx0[i], p.dz0[i]);
    }
    s.get_k1(p.dxidx1[i], p.dyidx1[i], p.dz1[i]);
    s.get_k2(p.dxidx2[i], p.dyidx2[i], p.dz2[i]);
}

// Interleaved work order: item t = (bucket t / nexp, experiment t % nexp)
// holds that experiment's particles in that Morton bucket; items[t] is the
// first chunk of item t (an exclusive prefix sum), items[nexp * nbuckets] and
// header->nchunks the total.  One CTA of 1024 threads.
constexpr int kPlanThreads = 1024;

__global__ void __launch_bounds__(kPlanThreads) k_plan_items(opb_batch_header *__restrict__ hdr,
                                                            const opb_experiment *__restrict__ exps,
                                                            const int64_t *__restrict__ bounds,
                                                            int64_t *__restrict__ items) {
    __shared__ long long warp_sum[kPlanThreads / 32];
    __shared__ long long carry;
    const int nexp = hdr->nexp, nb = hdr->nbuckets;
    if (nb <= 0) return;  // segment-major order: the caller's nchunks stands
    const long long n = (long long)nexp * nb;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long long base = 0; base < n; base += kPlanThreads) {
        const long long t = base + threadIdx.x;
        long long c = 0;
        if (t < n) {
            const int b = (int)(t / nexp), q = (int)(t % nexp);
            const opb_experiment &E = exps[q];
            if (E.nsteps > 0) {
                const int64_t *row = bounds + (long long)E.bucket_row * (nb + 1);
                const long long cnt = row[b + 1] - row[b];
                c = cnt > 0 ? (cnt + OPB_BATCH_CHUNK - 1) / OPB_BATCH_CHUNK : 0;
            }
        }
        // inclusive scan within the warp, then over the warp totals
        long long x = c;
        for (int d = 1; d < 32; d <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) warp_sum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            long long w = lane < kPlanThreads / 32 ? warp_sum[lane] : 0;
            for (int d = 1; d < 32; d <<= 1) {
                const long long y = __shfl_up_sync(0xffffffffu, w, d);
                if (lane >= d) w += y;
            }
            if (lane < kPlanThreads / 32) warp_sum[lane] = w;  // inclusive over warps
        }
        __syncthreads();
        const long long before = (warp > 0 ? warp_sum[warp - 1] : 0) + x - c;  // exclusive
        if (t < n) items[t] = carry + before;
        const long long block_total = warp_sum[kPlanThreads / 32 - 1];
        __syncthreads();
        if (threadIdx.x == 0) carry += block_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        items[n] = carry;
        hdr->nchunks = carry;
    }
}

// Persistent: every warp claims chunks of OPB_BATCH_CHUNK consecutive
// particles from the header's counter until none are left.  A chunk lies in
// one experiment's segment, so the 32 lanes of a warp share a scheme, a step
// count and a time table and never diverge on them.  MINB CTAs of BLOCK
// threads per SM: the register budget per thread is 65536 / (BLOCK * MINB).
template <typename T, typename I, int BLOCK, int MINB, int SCHEME, int LAYOUT, bool B2>
__global__ void __launch_bounds__(BLOCK, MINB) k_batched_steps(const __grid_constant__ DParticles p,
                                                            opb_batch_header *__restrict__ hdr,
                                                            const opb_experiment *__restrict__ exps,
                                                            const __grid_constant__ DScalars sc,
                                                            const __grid_constant__ DRoms r,
                                                            const opb_time *__restrict__ table,
                                                            const int64_t *__restrict__ bounds,
                                                            const int64_t *__restrict__ items) {
    OPB_LEVELS(r, sc);
    __shared__ double s_hist[OPB_BATCH_HIST_SMEM ? 6 * BLOCK : 1];
    const int nexp = hdr->nexp;
    const int nb = hdr->nbuckets;
    const long long nchunks = hdr->nchunks;
    const int lane = threadIdx.x & 31;
    unsigned long long *counter = (unsigned long long *)&hdr->next_chunk;
    for (;;) {
        unsigned long long c0 = 0;
        if (lane == 0) c0 = atomicAdd(counter, (unsigned long long)OPB_BATCH_CLAIM);
        c0 = __shfl_sync(0xffffffffu, c0, 0);
        if ((long long)c0 >= nchunks) break;
        for (unsigned long long c = c0; c < c0 + OPB_BATCH_CLAIM && (long long)c < nchunks; ++c) {
            long long i, end;
            int q;
            if (nb == 0) {
                // segment-major: the experiment owning chunk c is the last one whose first_chunk <= c
                int lo = 0, hi = nexp - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (exps[mid].first_chunk <= (long long)c) lo = mid;
                    else hi = mid - 1;
                }
                q = lo;
                i = exps[q].start + ((long long)c - exps[q].first_chunk) * OPB_BATCH_CHUNK + lane;
                end = exps[q].start + exps[q].count;
            } else {
                // interleaved: the item owning chunk c is the last one whose first chunk <= c
                long long lo = 0, hi = (long long)nexp * nb - 1;
                while (lo < hi) {
                    const long long mid = (lo + hi + 1) >> 1;
                    if (items[mid] <= (long long)c) lo = mid;
                    else hi = mid - 1;
                }
                q = (int)(lo % nexp);
                const int b = (int)(lo / nexp);
                const int64_t *row = bounds + (long long)exps[q].bucket_row * (nb + 1);
                i = row[b] + ((long long)c - items[lo]) * OPB_BATCH_CHUNK + lane;
                end = row[b + 1];
            }
            const opb_experiment E = exps[q];
            if (i >= end || i < E.start || i >= E.start + E.count || E.nsteps <= 0) continue;
            if (i < 0 || i >= p.n) continue;
            if (SCHEME != 0 && E.scheme != SCHEME) continue;  // another launch's experiment
            batched_particle<T, I, SCHEME, LAYOUT, B2>(p, i, E, sc, r, table, L, s_hist + threadIdx.x, BLOCK);
        }
    }
}

// launch the <BLOCK, MINB> instance; false if the shape is not compiled
template <typename T, typename I, int SCHEME, int LAYOUT, bool B2>
bool launch_batched(int block, int warps_per_sm, int ctas, cudaStream_t st, const DParticles &dp,
                    opb_batch_header *hdr, const opb_experiment *exps, const DScalars &ds, const DRoms &dr,
                    const opb_time *table, const int64_t *bounds, const int64_t *items, int *launched) {
    auto go = [&](auto kernel, int B) {
        const int g = ctas > 0 ? ctas : resident_ctas((const void *)kernel, B);
        if (g <= 0) return true;
        kernel<<<g, B, 0, st>>>(dp, hdr, exps, ds, dr, table, bounds, items);
        *launched = 1;
        return true;
    };
    const int key = block * 100 + warps_per_sm;
    // the combined kernel (SCHEME 0) only at 16 warps: its register budget already spills at 80
    if (SCHEME == 0 && warps_per_sm != 16) return false;
    switch (key) {
        case 12816: return go(k_batched_steps<T, I, 128, 4, SCHEME, LAYOUT, B2>, 128);
        case 25616: return go(k_batched_steps<T, I, 256, 2, SCHEME, LAYOUT, B2>, 256);
        case 25624: return go(k_batched_steps<T, I, 256, 3, SCHEME != 0 ? SCHEME : OPB_SCHEME_RK2, LAYOUT, B2>, 256);
        case 25632: return go(k_batched_steps<T, I, 256, 4, SCHEME != 0 ? SCHEME : OPB_SCHEME_RK2, LAYOUT, B2>, 256);
        default: return false;
    }
}

}  // namespace
}  // namespace opb

using namespace opb;

extern "C" {

int opb_batched_steps(const opb_particles *p, opb_batch_header *header, const opb_experiment *experiments,
                      const opb_scalars *s, const opb_roms_fields *f, const opb_time *table,
                      const int64_t *bucket_bounds, int64_t *item_scratch, int32_t scheme, int32_t block,
                      int32_t warps_per_sm, int32_t ctas, void *stream) {
    const char *what = "opb_batched_steps";
    DParticles dp;
    DScalars ds;
    DRoms dr;
    int dtype, rc;
    if ((rc = convert_particles(p, dp, what, true))) return rc;
    if (!s) return fail(OPB_EINVAL, "%s: scalars is NULL", what);
    convert_scalars(s, ds);
    // time-dependent fields come as snapshot pairs or quads: check, then convert with the element dtype
    opb_roms_fields g;
    int layout = LAYOUT_PLAIN;
    bool bundled = false;
    if ((rc = unpair_fields(f, g, layout, bundled, what))) return rc;
    if (layout == LAYOUT_PLAIN && !(g.u.is_static && g.v.is_static && g.w.is_static && g.zeta.is_static))
        return fail(OPB_EINVAL, "%s: time-dependent fields must be snapshot pairs (OPB_F32_PAIRS or OPB_F64_PAIRS), "
                    "quads (OPB_F32_QUADS) or octets (OPB_F32_OCTS)", what);
    if ((rc = convert_fields(&g, dr, what, true, &dtype))) return rc;
    if (!header || !experiments || !table) return fail(OPB_EINVAL, "%s: NULL device array", what);
    const bool shape_ok = (block == 128 && warps_per_sm == 16) ||
                          (block == 256 && (warps_per_sm == 16 || warps_per_sm == 24 || warps_per_sm == 32));
    if (!shape_ok || (scheme == 0 && warps_per_sm != 16))
        return fail(OPB_EINVAL, "%s: launch shapes are block 256 with 16, 24 or 32 warps per SM, or block 128 with "
                    "16 (scheme 0: 16 warps only)", what);
    if (ctas < 0) return fail(OPB_EINVAL, "%s: negative CTA count", what);
    if (scheme != 0 && scheme != OPB_SCHEME_RK2 && scheme != OPB_SCHEME_AB3)
        return fail(OPB_EINVAL, "%s: scheme must be 0, OPB_SCHEME_RK2 or OPB_SCHEME_AB3", what);
    if (!roms_layout(dr))
        return fail(OPB_EINVAL, "%s: fields must have the ROMS layout (u, v, w, zeta time-dependent; h, dx, dy, C "
                    "static) and geometry (u, v, w staggered on the Arakawa C grid)", what);
    rc = need_fields(p, what, {{"z", p->z}, {"_dxidx1", p->dxidx1}, {"_dyidx1", p->dyidx1}, {"_dz1", p->dz1},
                               {"_dxidx2", p->dxidx2}, {"_dyidx2", p->dyidx2}, {"_dz2", p->dz2},
                               {"_dxidx0", p->dxidx0}, {"_dyidx0", p->dyidx0}, {"_dz0", p->dz0}});
    if (rc) return rc;
    if ((bucket_bounds == nullptr) != (item_scratch == nullptr))
        return fail(OPB_EINVAL, "%s: give both bucket_bounds and item_scratch or neither", what);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(&header->next_chunk, 0, sizeof(header->next_chunk), st);
    if (e != cudaSuccess) return fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    if (dp.n == 0) return OPB_OK;
    // interleaved order (header->nbuckets > 0, read on the device): the plan kernel fills the item table
    // and header->nchunks; with nbuckets = 0 it returns at once
    if (bucket_bounds) {
        k_plan_items<<<1, kPlanThreads, 0, st>>>(header, experiments, bucket_bounds, item_scratch);
        e = cudaGetLastError();
        if (e != cudaSuccess) return fail(OPB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    }
    int launched = 0;
    auto go = [&](auto tv, auto iv, auto lv, auto bv) {
        using T = decltype(tv);
        using I = decltype(iv);
        constexpr int LAYOUT = decltype(lv)::value;
        constexpr bool B2 = decltype(bv)::value;
        if (scheme == OPB_SCHEME_RK2)
            launch_batched<T, I, OPB_SCHEME_RK2, LAYOUT, B2>(block, warps_per_sm, ctas, st, dp, header, experiments,
                                                             ds, dr, table, bucket_bounds, item_scratch, &launched);
        else if (scheme == OPB_SCHEME_AB3)
            launch_batched<T, I, OPB_SCHEME_AB3, LAYOUT, B2>(block, warps_per_sm, ctas, st, dp, header, experiments,
                                                             ds, dr, table, bucket_bounds, item_scratch, &launched);
        else
            launch_batched<T, I, 0, LAYOUT, B2>(block, warps_per_sm, ctas, st, dp, header, experiments, ds, dr, table,
                                                bucket_bounds, item_scratch, &launched);
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
    } else {
        // snapshot pairs (roms_layout above rules out the all-static fields that passed the layout check)
        dispatch(dtype, small, [&](auto tv, auto iv) {
            go(tv, iv, std::integral_constant<int, LAYOUT_PAIRS>{}, NoB{});
        });
    }
    if (!launched) return fail(OPB_ECUDA, "%s: occupancy query failed", what);
    return check_launch(what);
}

}  // extern "C"
