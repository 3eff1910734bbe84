/*
 * opb200.h -- C ABI of liboffline_particles_b200.so, the B200 (sm_100a)
 * implementation of offline_particles' ROMS particle-advection hot path.
 *
 * Reference interface.  In offline_particles every particle kernel is a
 * ParticleKernel wrapping  fn(particles, scalars, fielddata) -> None  that
 * mutates the particle arrays in place (kernels/_kernels.py:12,22-44,85-93);
 * Launcher.launch_kernel builds `scalars` and `fielddata` and calls it
 * (launcher.py:167-174).  Each entry point below is the device-side
 * replacement of one such function, with the same three arguments as plain C
 * structs:
 *   particles -> opb_particles  (device SoA, Particles / particles.py:76-92)
 *   scalars   -> opb_scalars    (hc, NZ, _dt, _RK2_alpha, *idx_min/max)
 *   fielddata -> opb_roms_fields + opb_time (FieldData(array, offsets) of
 *                fields.py:12 with the time blend of fields.py:394-430 left
 *                unmaterialised: the kernels blend each gathered corner)
 * All pointers in these structs are DEVICE pointers; `stream` is a
 * cudaStream_t (NULL = legacy default stream).  Every call is asynchronous.
 *
 * Return value: 0 on success, otherwise an OPB_E* code; opb_last_error()
 * then describes the failure.  Per-particle problems are not errors: as in
 * the reference they become status codes (kernels/status.pxd:1-14).  A zero
 * grid spacing in a velocity division -- ZeroDivisionError in the reference
 * (Cython cdivision=False) -- sets OPB_ERRF_ZERO_DIVISION in *particles->err
 * on the device; the host reads that word when it synchronises.
 *
 * Numerics: float64 arithmetic in the reference's operation order with no
 * FMA contraction, so results are bit-identical to the reference's x86-64
 * build on the same inputs.
 */
#ifndef OPB200_H
#define OPB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OPB_ABI_VERSION 5
#define OPB_MAX_SLOTS 8

/* storage dtypes of time-dependent fields (the float64-exact entry points take
 * OPB_F64 and OPB_F32; the *_fp32 entry points also take OPB_BF16 / OPB_F16
 * with per-level scales) */
#define OPB_F64 0
#define OPB_F32 1
#define OPB_BF16 2
#define OPB_F16 3
/* snapshot pairs (opb_batched_steps and the float64 fused steppers
 * opb_rk2/ab3_w_advection_steps, ROMS field layout): data[k] holds two consecutive
 * snapshots interleaved element by element (element 2i from the earlier, 2i+1
 * from the later), so one load fetches both values a time blend needs; an
 * opb_time selects the pair with prev (next == prev) */
#define OPB_F64_PAIRS 4
#define OPB_F32_PAIRS 5
/* snapshot quads (the same entry points, float32 storage): data[k] holds, for
 * element i, the four floats {a[i], b[i], a[i+1], b[i+1]} of the earlier (a) and
 * later (b) snapshot, so one 16-byte load fetches a stencil's two x-neighbouring
 * corners with both values of their time blends.  Quads come with x-pairs of the
 * static fields h, dx and dy (OPB_F64_XPAIRS; C stays OPB_F64) */
#define OPB_F32_QUADS 6
/* x-pairs of a static float64 field: data[0] holds {s[i], s[i+1]} for element i */
#define OPB_F64_XPAIRS 7
/* snapshot octets (the same entry points, float32 storage): data[k] holds, for
 * element i, the earlier/later pairs of elements i, i+1, i+R and i+R+1 (R: the
 * field's last dimension), so one 32-byte load fetches the four corners of a
 * stencil face with both values of their time blends.  Octets come with yx-pairs
 * of h, dx and dy (OPB_F64_YXPAIRS; C stays OPB_F64).  Pair buffers must be
 * aligned to their load: 8 bytes (OPB_F32_PAIRS), 16 (OPB_F64_PAIRS, quads,
 * x-pairs) or 32 (octets, yx-pairs) */
#define OPB_F32_OCTS 8
/* yx-pairs of a static float64 field: data[0] holds {s[i], s[i+1], s[i+R], s[i+R+1]} */
#define OPB_F64_YXPAIRS 9
/* 2-D bundles (with snapshot pairs or quads of float32 u, v, w): h, zeta, dx and
 * dy share one stagger, so two of them can share one load per two stencil
 * corners.  zeta as OPB_F32_ZETA_H: data[k] holds, per element i, the 64-bit
 * words {h[i], zeta pair[i], h[i+1], zeta pair[i+1]} (a zeta pair: the earlier
 * snapshot's float in the low half, the later's in the high half; pair slot k as
 * for OPB_F32_PAIRS), with h as OPB_F64_IN_ZETA (read from zeta's bundle; same
 * shape and offsets).  dx as OPB_F64_DX_DY: data[0] holds {dx[i], dy[i], dx[i+1],
 * dy[i+1]}, with dy as OPB_F64_IN_DX (same shape and offsets).  Bundle buffers
 * are 32-byte aligned; all four codes come together. */
#define OPB_F32_ZETA_H 10
#define OPB_F64_IN_ZETA 11
#define OPB_F64_DX_DY 12
#define OPB_F64_IN_DX 13

/* return codes */
#define OPB_OK 0
#define OPB_EINVAL 1  /* bad argument (sizes, dtype, NULL pointer, slot index) */
#define OPB_ECUDA 2   /* a CUDA runtime call failed */

/* bits of the device error word (opb_particles.err) */
#define OPB_ERRF_ZERO_DIVISION 1u

/* particle status codes: kernels/status.pxd:1-14 */
#define OPB_STATUS_INACTIVE 0x80
#define OPB_STATUS_NORMAL 0x00
#define OPB_STATUS_NONFINITE 0x81
#define OPB_STATUS_OUT_OF_DOMAIN 0x82
#define OPB_STATUS_MULTISTEP_1 10
#define OPB_STATUS_MULTISTEP_2 11

/* A field: FieldData(array, offsets) of fields.py:12.
 * Time-dependent fields (is_static == 0) give the device snapshot buffers
 * `data[0..nslots-1]` in storage dtype `dtype`; an opb_time picks the two
 * snapshots and the blend weights.  Static fields (is_static == 1) give one
 * float64 buffer in data[0] (the reference casts every field to float64,
 * kernels/_core.pyx:5-24).  Arrays are C-contiguous over the `ndim` active
 * dimensions (slowest first); `offset` is added to the particle index of each
 * active dimension (spatial_arrays.py:29-41,224-225). */
typedef struct {
    const void *data[OPB_MAX_SLOTS];
    int32_t dtype;
    int32_t ndim;
    int64_t shape[3];
    double offset[3];
    int32_t is_static;
    int32_t nslots;
    /* OPB_BF16 / OPB_F16 storage: scale[k][l] multiplies the stored values of
     * slot k at level l (the first active dimension; 2-D fields use l = 0);
     * NULL for unscaled storage */
    const float *scale[OPB_MAX_SLOTS];
} opb_field;

/* The simulation fields of the ROMS w-advection kernels
 * (kernels/roms/rk2_w_advection.pyx:386-395, ab3_w_advection.pyx:265-274). */
typedef struct {
    opb_field u, v, w, dx, dy, h, zeta, C;
} opb_roms_fields;

/* Time selection for one launch: It, ft = divmod(time_index, 1)
 * (fields.py:409-424).  prev/next are slot indices of snapshots It and It+1;
 * ft and gt = 1 - ft are already rounded to the storage dtype. */
typedef struct {
    int32_t prev, next;
    double ft, gt;
} opb_time;

/* Particle SoA (kernels/_kernels.py:14-19 plus the kernels' own fields).
 * RK2 uses k1 = (dxidx1, dyidx1, dz1) and k2 = (dxidx2, dyidx2, dz2)
 * (rk2_w_advection.pyx:377-410); AB3 uses the 0/1/2 history
 * (ab3_w_advection.pyx:250-258).  Unused pointers may be NULL. */
typedef struct {
    int64_t n;
    uint8_t *status;
    double *zidx, *yidx, *xidx, *z;
    double *dxidx0, *dyidx0, *dz0;
    double *dxidx1, *dyidx1, *dz1;
    double *dxidx2, *dyidx2, *dz2;
    uint32_t *err; /* device error word (OPB_ERRF_*), may be NULL */
    double *rho_t; /* target density of the isopycnal follower (ab3_isopycnal_following.pyx:41), or NULL */
} opb_particles;

/* Scalars the ROMS kernels declare (rk2_w_advection.pyx:382-385,412-417;
 * validation.pyx:113-120): hc, NZ, _dt, _RK2_alpha, zidx/yidx/xidx min/max. */
typedef struct {
    double hc;
    int32_t NZ;
    int32_t _pad;
    double dt;
    double alpha;
    double bounds[6]; /* zmin, zmax, ymin, ymax, xmin, xmax */
    double w_max;     /* isopycnal follower (ab3_isopycnal_following.pyx:54-55) */
    double rho_scale;
} opb_scalars;

/* ---- one entry point per reference kernel function ---------------------- */

/* kernels/validation.pyx:21-43 (finite_indices) */
int opb_finite_indices(const opb_particles *p, void *stream);
/* kernels/validation.pyx:45-77 (domain_bounds) */
int opb_domain_bounds(const opb_particles *p, const opb_scalars *s, void *stream);
/* kernels/validation.pyx:124 (validation_kernel = finite_indices, domain_bounds) */
int opb_validation(const opb_particles *p, const opb_scalars *s, void *stream);
/* kernels/roms/_roms_core.pyx:17-73 (compute_z_kernel): z into `out` */
int opb_compute_z(const opb_particles *p, double *out, const opb_scalars *s, const opb_roms_fields *f,
                  const opb_time *t, void *stream);
/* kernels/roms/rk2_w_advection.pyx:31-153 (rk2_w_advection_step_1) */
int opb_rk2_w_advection_step_1(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                               const opb_time *t, void *stream);
/* kernels/roms/rk2_w_advection.pyx:155-275 (rk2_w_advection_step_2) */
int opb_rk2_w_advection_step_2(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                               const opb_time *t, void *stream);
/* kernels/roms/rk2_w_advection.pyx:278-354 (rk2_w_advection_update) */
int opb_rk2_w_advection_update(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                               const opb_time *t, void *stream);
/* kernels/roms/ab3_w_advection.pyx:20-178 (ab3_w_advection) */
int opb_ab3_w_advection(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                        const opb_time *t, void *stream);
/* kernels/roms/ab3_w_advection.pyx:180-229 (ab3_post_w_advection) */
int opb_ab3_post_w_advection(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                             const opb_time *t, void *stream);

/* kernels/roms/ab3_isopycnal_following.pyx:26-192 (ab3_isopycnal_following):
 * the AB3 step with dz0 = w_max * drho / (rho_scale + |drho|), drho = rho -
 * rho_t.  The density field is passed in f->w (staggered at rho points),
 * p->rho_t and s->w_max, s->rho_scale are required.  The post step
 * (ab3_isopycnal_following.pyx:194-241) is the same computation as
 * opb_ab3_post_w_advection, which serves it. */
int opb_ab3_isopycnal_following(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                                const opb_time *t, void *stream);

/* ---- snapshot pairs ------------------------------------------------------------
 * No reference counterpart (a layout of this library): out[2i] = a[i],
 * out[2i + 1] = b[i] for i < n, a/b/out DEVICE buffers of dtype OPB_F32 or
 * OPB_F64 (out holds 2n elements): the snapshot pair of snapshots a and b. */
int opb_interleave_pairs(const void *a, const void *b, void *out, int64_t n, int32_t dtype, void *stream);

/* No reference counterpart (a layout of this library): the snapshot quads of
 * float32 snapshots a and b, out[4i .. 4i+3] = a[i], b[i], a[i+1], b[i+1] for
 * i < n - 1 and a[n-1], b[n-1], a[n-1], b[n-1] for the last element (out holds
 * 4n floats; DEVICE buffers, out 16-byte aligned). */
int opb_interleave_quads(const float *a, const float *b, float *out, int64_t n, void *stream);

/* No reference counterpart: the x-pairs of a static float64 field s,
 * out[2i] = s[i], out[2i+1] = s[i+1] for i < n - 1 and s[n-1] twice for the last
 * element (out holds 2n doubles; DEVICE buffers, out 16-byte aligned). */
int opb_neighbour_pairs(const double *s, double *out, int64_t n, void *stream);

/* No reference counterpart: the snapshot octets of float32 snapshots a and b with
 * row length `row`, out[8i .. 8i+7] = a[j], b[j] for j = i, i+1, i+row, i+row+1 in
 * turn, each j past the end replaced by n - 1 (out holds 8n floats; DEVICE
 * buffers, out 32-byte aligned). */
int opb_interleave_octets(const float *a, const float *b, float *out, int64_t n, int64_t row, void *stream);

/* No reference counterpart: the yx-pairs of a static float64 field s with row
 * length `row`, out[4i .. 4i+3] = s[i], s[i+1], s[i+row], s[i+row+1], each index
 * past the end replaced by n - 1 (out holds 4n doubles; DEVICE buffers, out
 * 32-byte aligned). */
int opb_neighbour_quads(const double *s, double *out, int64_t n, int64_t row, void *stream);

/* No reference counterpart: the zeta-with-h bundle of float32 zeta snapshots a
 * (earlier) and b (later) and float64 h, n elements each (OPB_F32_ZETA_H; out
 * holds 32 bytes per element, 32-byte aligned; the last element's neighbour is
 * itself). */
int opb_bundle_zeta_h(const float *a, const float *b, const double *h, void *out, int64_t n, void *stream);

/* No reference counterpart: the dx-with-dy bundle of float64 dx and dy, n
 * elements each (OPB_F64_DX_DY; out holds 4n doubles, 32-byte aligned). */
int opb_bundle_dx_dy(const double *dx, const double *dy, double *out, int64_t n, void *stream);

/* ---- batched release experiments ---------------------------------------------
 * No single reference counterpart: the reference advances one release per
 * Simulation (simulation.py:27-229).  Here many releases share one particle
 * arena, each in its own contiguous segment, and advance in one launch; each
 * release runs exactly the steps its own Simulation would run with the ROMS
 * presets (timesteppers.py:241-257 / :296-305), so its results are the same. */
#define OPB_SCHEME_RK2 1
#define OPB_SCHEME_AB3 2
#define OPB_BATCH_CHUNK 32 /* particles a warp claims at a time */

/* One experiment's work in a launch.  Its steps read table[table_offset ...]:
 * 3 opb_time entries per RK2 step (t, t + alpha dt, t + dt), 2 per AB3 step
 * (t, t + dt).  Chunks: experiment e owns chunks [first_chunk, first_chunk +
 * ceil(count / OPB_BATCH_CHUNK)); first_chunk ascends through the table. */
typedef struct {
    int64_t start;       /* first storage index of the experiment's segment */
    int64_t count;       /* particles in the segment */
    int64_t first_chunk; /* chunks of the experiments before this one */
    int32_t scheme;      /* OPB_SCHEME_RK2 or OPB_SCHEME_AB3 */
    int32_t nsteps;      /* steps in this launch (>= 1) */
    int32_t table_offset;
    int32_t validate;    /* 1: the validation kernel runs before every step */
    double dt;
    double alpha;        /* RK2 only */
    int32_t bucket_row;  /* row of the experiment in the bucket-bounds table (interleaved order) */
    int32_t _pad;
} opb_experiment;

/* Per-launch header, in DEVICE memory next to the tables (so one captured
 * CUDA graph serves every launch: only device contents change). */
typedef struct {
    int32_t nexp;        /* experiments in the table */
    int32_t nbuckets;    /* 0: segment-major work order; else spatially interleaved over this many buckets */
    int64_t nchunks;     /* total chunks (segment-major: set by the caller; interleaved: by the launch) */
    uint64_t next_chunk; /* work counter: zeroed by opb_batched_steps before its kernel */
} opb_batch_header;

/* Advance the experiments of `header`/`experiments`/`table` (DEVICE arrays)
 * over the particle arena p (all AB3 history pointers required).  A
 * persistent grid (`ctas` CTAs of `block` threads; ctas = 0: as many as stay
 * resident) in which each warp claims chunks until none are left.  Shapes:
 * block 256 with warps_per_sm 16, 24 or 32 (register budget per thread 128,
 * 80 or 64), or block 128 with 16; scheme 0 takes 16 only.  Work order: header->nbuckets = 0 walks each
 * experiment's segment in turn (chunks from first_chunk); nbuckets > 0 walks
 * Morton buckets in turn and, within a bucket, every experiment's particles in
 * it (bucket_bounds as written by opb_sort_segments, row bucket_row per
 * experiment; item_scratch: nexp * nbuckets + 1 int64 of DEVICE scratch), so
 * particles of all experiments that share a region are advanced together and
 * share the field data in L2.  The time-dependent fields (u, v, w, zeta) come
 * as snapshot pairs (OPB_F32_PAIRS / OPB_F64_PAIRS).  scheme: 0 advances every experiment of the
 * table with one kernel; OPB_SCHEME_RK2 / OPB_SCHEME_AB3 compiles that scheme
 * alone (smaller code, fewer registers) and skips experiments of the other.
 * Fields must have the ROMS layout (u, v, w,
 * zeta time-dependent; h, dx, dy, C static).  Results equal running each
 * experiment alone with opb_rk2/ab3_w_advection_steps. */
int opb_batched_steps(const opb_particles *p, opb_batch_header *header, const opb_experiment *experiments,
                      const opb_scalars *s, const opb_roms_fields *f, const opb_time *table,
                      const int64_t *bucket_bounds, int64_t *item_scratch, int32_t scheme, int32_t block,
                      int32_t warps_per_sm, int32_t ctas, void *stream);

/* Spatially sort particles WITHIN each of nseg segments [start, start+count)
 * (host arrays; segments disjoint and ascending).  Each segment is reordered
 * by the Morton key of opb_sort_particles (inactive last, stable); particles
 * never leave their segment.  ids (int64, DEVICE, one per arena particle, or
 * NULL) is permuted with the particles.  bucket_bounds (DEVICE, nseg rows of
 * nbuckets + 1 int64, or NULL): row s, entry b = storage index of segment s's
 * first particle in Morton bucket >= b (nbuckets equal power-of-two key
 * ranges covering the grid; entry nbuckets = the first inactive particle or
 * the segment's end).  No reference counterpart (the reference never
 * reorders particles). */
size_t opb_sort_segments_workspace_bytes(int64_t total, int32_t nseg);
int opb_sort_segments(const opb_particles *p, const int64_t shape[3], const int64_t *seg_start,
                      const int64_t *seg_count, int32_t nseg, int64_t *ids, int32_t nbuckets, int64_t *bucket_bounds,
                      void *workspace, size_t workspace_bytes, void *stream);

/* ---- reduced-precision steppers --------------------------------------------
 * The precision variant of the fused steppers: float32 interpolation and
 * updates, fractional x/y indices kept as compensated float32 pairs, float64
 * only for z = zeta + (zeta + h) S and its inverse in columns with h < 100 m.
 * Time-dependent fields may be stored as float32, or as bfloat16 / float16
 * with per-level scales (opb_field.scale).  Not bit-identical to the
 * reference: its error is measured as trajectory separation in metres against
 * the float64 entry points. */
int opb_rk2_w_advection_steps_fp32(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                                   const opb_time *table, int32_t nsteps, int32_t validate, void *stream);
int opb_ab3_w_advection_steps_fp32(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                                   const opb_time *table, int32_t nsteps, int32_t validate, void *stream);
/* Quantise `nsnap` float32 snapshots of `nlev` levels x `per_level` values each
 * (C order) into `dtype` (OPB_BF16 or OPB_F16) at `dst`, writing one scale per
 * (snapshot, level) to `scales` (nsnap x nlev): value ~= stored * scale,
 * scale = max |value| of the level / 32768 (1 for an all-zero level). */
int opb_quantize_levels(const float *src, int64_t nsnap, int64_t nlev, int64_t per_level, int32_t dtype, void *dst,
                        float *scales, void *stream);

/* ---- output sampling (kernels/output/linear_interpolation.pyx:34-136) ----- */

/* out[i] = linear interpolation of a 1-D field at idx[i] + offset, for active
 * particles (linear_interpolation_kernel_function, :34-68) */
int opb_linear_interpolation(const opb_particles *p, const double *idx, const opb_field *f, const opb_time *t,
                             double *out, void *stream);
/* out[i] = bilinear interpolation of a 2-D field at (idx0[i], idx1[i]) + offsets
 * (bilinear_interpolation_kernel_function, :70-103) */
int opb_bilinear_interpolation(const opb_particles *p, const double *idx0, const double *idx1, const opb_field *f,
                               const opb_time *t, double *out, void *stream);
/* out[i] = trilinear interpolation of a 3-D field at (zidx, yidx, xidx) + offsets
 * (trilinear_interpolation_kernel_function, :105-136) */
int opb_trilinear_interpolation(const opb_particles *p, const opb_field *f, const opb_time *t, double *out,
                                void *stream);

/* ---- fused steppers ------------------------------------------------------ */

/* Step tables of the fused entry points (the *_steps functions, float64 and
 * float32): a DEVICE array, or a HOST array (pageable or pinned) of at most
 * OPB_INLINE_TABLE entries, which the call copies into the launch's parameters.
 * A host table needs no copy engine, so the launch does not queue behind
 * host-to-device copies issued before it (snapshot uploads); the caller may
 * reuse the array as soon as the call returns.  Every entry of a host table
 * is checked (slots within the fields' nslots; OPB_EINVAL otherwise); a device
 * table is the caller's to get right. */
#define OPB_INLINE_TABLE 720

/* `nsteps` whole RK2 steps in one launch: per step, the preset's validation
 * pre-step, step_1 at t, step_2 at t + alpha dt, update at t + dt
 * (timesteppers.py:241-257; models/roms/__init__.py:37-62).  `table` is an
 * array of 3*nsteps opb_time entries (t, t + alpha dt, t + dt per step), on the
 * device or on the host (OPB_INLINE_TABLE).  validate = 0 drops the pre-step.  Results equal `nsteps` rounds of
 * the stage entry points; k1/k2 and z hold the last step's values. */
int opb_rk2_w_advection_steps(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                              const opb_time *table, int32_t nsteps, int32_t validate, void *stream);
/* `nsteps` whole AB3 steps in one launch: validation pre-step, ab3 at t,
 * ab3_post at t + dt (timesteppers.py:296-305; models/roms/__init__.py:65-96).
 * `table`: 2*nsteps opb_time entries (t, t + dt per step), on the device or on
 * the host (OPB_INLINE_TABLE). */
int opb_ab3_w_advection_steps(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                              const opb_time *table, int32_t nsteps, int32_t validate, void *stream);

/* Particle state recorded after chosen steps of one fused launch, for the
 * events that fall inside it (output events: Simulation._invoke_events,
 * simulation.py:169-176, fires them between steps; here they replay after the
 * launch on the recorded state, so they no longer end the launch).  Bit k of
 * mask[k / 64] asks for the state after step k (k < nsteps <= 256); the r-th
 * recorded step (in step order) of particle i goes to index r * stride + i of
 * each array (stride >= n; DEVICE pointers).  The state is what the particle
 * arrays would hold at that point: status, zidx, yidx, xidx and z (a particle
 * that stopped, or was inactive from the start, records its unchanged state).
 * No reference counterpart. */
typedef struct {
    uint64_t mask[4];
    int64_t stride;
    double *zidx, *yidx, *xidx, *z;
    uint8_t *status;
} opb_records;

/* The three fused entry points above, with `rec` (NULL: none) recorded. */
int opb_rk2_w_advection_steps_rec(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                                  const opb_time *table, int32_t nsteps, int32_t validate, const opb_records *rec,
                                  void *stream);
int opb_ab3_w_advection_steps_rec(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                                  const opb_time *table, int32_t nsteps, int32_t validate, const opb_records *rec,
                                  void *stream);
int opb_ab3_isopycnal_following_steps_rec(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                                          const opb_time *table, int32_t nsteps, int32_t validate,
                                          const opb_records *rec, void *stream);

/* ABTimestepper.timestep_particles with ab3_isopycnal_following_timestepper's
 * kernels (models/roms/__init__.py:109-141): nsteps fused steps, as
 * opb_ab3_w_advection_steps with the isopycnal follower's vertical velocity. */
int opb_ab3_isopycnal_following_steps(const opb_particles *p, const opb_scalars *s, const opb_roms_fields *f,
                                      const opb_time *table, int32_t nsteps, int32_t validate, void *stream);

/* ---- spatial ordering ------------------------------------------------------
 * No counterpart in the reference, which keeps particles in release order and
 * splits them statically over OpenMP threads (rk2_w_advection.pyx:85-91).
 * Every kernel is per particle, so storage order changes no result; a
 * Morton order by cell makes neighbouring threads gather neighbouring field
 * corners, which is what lets the fused kernels reuse L1/L2. */

/* Bytes of device workspace opb_sort_particles needs for n particles. */
size_t opb_sort_workspace_bytes(int64_t n);
/* perm[j] = index of the particle that belongs at position j: active particles
 * in Morton order of their cell on the centred (z, y, x) grid of `shape`,
 * inactive particles last, ties in index order.  `workspace` is a device buffer
 * of at least opb_sort_workspace_bytes(n) bytes, used as scratch. */
int opb_sort_particles(const opb_particles *p, const int64_t shape[3], int32_t *perm, void *workspace,
                       size_t workspace_bytes, void *stream);
/* As opb_sort_particles, within id ranges: the particle in slot i has id
 * ids[i] (int64, DEVICE; NULL: id = i), and the particles with ids in
 * [bounds[r], bounds[r + 1]) are ordered among themselves into the positions
 * [bounds[r], bounds[r + 1]).  bounds: HOST array of nranges + 1 increasing
 * values from 0 to n, nranges 1 to 4 (the range index takes the top two bits
 * of the cell key).  With ids a permutation of 0..n-1 whose range r occupies
 * those slots already (an earlier call with the same bounds, or the identity),
 * every particle stays in its range: a caller can then read back the particles
 * of one range as soon as the launches over its slots are done.  Same
 * workspace as opb_sort_particles. */
int opb_sort_particles_ranges(const opb_particles *p, const int64_t shape[3], const int64_t *ids,
                              const int64_t *bounds, int32_t nranges, int32_t *perm, void *workspace,
                              size_t workspace_bytes, void *stream);
/* dst.f[j] = src.f[perm[j]] for status and every float64 field present in
 * both (src and dst must not alias), and dst_ids[j] = src_ids[perm[j]] when
 * id arrays are given. */
int opb_gather_particles(const opb_particles *src, const opb_particles *dst, const int32_t *perm,
                         const int64_t *src_ids, int64_t *dst_ids, void *stream);

/* ---- sorting without device allocation ---------------------------------------
 * No counterpart in the reference (which has no GPU and no device memory).
 * Some callers cannot allocate device memory at the moment they sort: a host
 * runtime that reserved all device memory up front for its own pool, or a
 * latency-critical loop in which a cudaMalloc / cudaFree pair would
 * synchronise the device and stall the work already queued.  For them,
 * opb_sort_particles_noalloc gives the same permutation as
 * opb_sort_particles but takes its scratch from a static device array inside
 * this library instead of a caller workspace, and calls no allocating routine.
 *
 *   - The array is OPB_NOALLOC_SCRATCH_BYTES (13 MiB).  Every GPU that loads
 *     the library holds it until the process exits.
 *   - At most OPB_NOALLOC_MAX_PARTICLES particles per call; more is rejected
 *     with OPB_EINVAL and a message (use opb_sort_particles then).
 *   - The first call on a device looks up the array's device address (with
 *     that device current); make that first call before any stream capture.
 *     With lazy module loading (the CUDA default) that first call may also
 *     load this library's device code on that device, which places the array
 *     in device memory then: a caller that reserves device memory for its own
 *     pool should make one call (n = 0 is not enough; any n >= 1 is) before
 *     reserving.  Later calls allocate nothing.
 *   - Outside stream capture every call looks the address up again, so a
 *     device reset (cudaDeviceReset) between calls is safe; during capture
 *     the address found by an earlier call on that device is used, so do not
 *     capture a call after a reset without an uncaptured call in between.
 *   - Every call on a device shares the one array, which keeps the last call's
 *     contents (nothing in it has to start at zero: each call writes its keys
 *     and ids in full before reading them).  Calls that overlap on the GPU
 *     race on it: issue them on one stream, or wait for one before the next. */
#define OPB_NOALLOC_MAX_PARTICLES (1 << 20)
#define OPB_NOALLOC_SORT_TEMP_BYTES (1u << 20)
#define OPB_NOALLOC_SCRATCH_BYTES ((size_t)12 * OPB_NOALLOC_MAX_PARTICLES + OPB_NOALLOC_SORT_TEMP_BYTES)

int opb_sort_particles_noalloc(const opb_particles *p, const int64_t shape[3], int32_t *perm, void *stream);

/* ---- library ------------------------------------------------------------- */

/* Message of the last failed call on this host thread ("" if none). */
const char *opb_last_error(void);
/* Self-check of the AB3 update's division by 12 (three floating-point
 * operations instead of the IEEE division; the same bits by Markstein's
 * theorem): adds to *mismatches (DEVICE, uint64) the number of x[i] (DEVICE)
 * for which the two quotients differ in any bit.  No reference counterpart. */
int opb_check_div12(const double *x, int64_t n, uint64_t *mismatches, void *stream);

/* OPB_ABI_VERSION of the loaded library. */
int opb_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* OPB200_H */
