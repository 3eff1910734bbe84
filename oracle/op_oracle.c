/*
 * CPU oracle for the ROMS particle-advection step -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's Cython kernels, used by tests/,
 * the smoke check and the CPU-baseline leg of bench.py as the checker.  It is
 * never linked into, called by or shipped with the product library.
 *
 * Every function below states the reference file:line it follows (paths are
 * relative to the reference package root, src/offline_particles/).  The
 * arithmetic is written in the reference's operation order and compiled with
 * -ffp-contract=off so that it is bit-identical to the reference's x86-64
 * release build (gcc -O3, no FMA).
 *
 * Fields arrive already blended in time and cast to float64, exactly what the
 * reference's kernels receive from Field.get_field_data + unpack_fielddata_*
 * (fields.py:394-430, kernels/_core.pyx:5-24); the blend itself is done by
 * oracle/oracle.py in numpy, mirroring fields.py:419-428.
 *
 * Error behaviour (from the C that Cython 3 generates for the reference with
 * cdivision=False):
 *   - a zero divisor inside the `noexcept nogil` helpers of
 *     kernels/roms/_vertical_coordinate.pxd makes THAT helper return 0.0;
 *   - a zero divisor in a loop body (u/dx, v/dy) raises ZeroDivisionError.
 *     Here such a particle is counted and the caller raises.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define OST_INACTIVE 0x80u     /* kernels/status.pxd:3 */
#define OST_NORMAL 0u          /* kernels/status.pxd:6 */
#define OST_NONFINITE 0x81u    /* kernels/status.pxd:9 */
#define OST_OUT_OF_DOMAIN 0x82u/* kernels/status.pxd:10 */
#define OST_MULTISTEP_1 10u    /* kernels/status.pxd:13 */
#define OST_MULTISTEP_2 11u    /* kernels/status.pxd:14 */

typedef struct { const double *a; int64_t n0; double o0; } of1;
typedef struct { const double *a; int64_t n0, n1; double o0, o1; } of2;
typedef struct { const double *a; int64_t n0, n1, n2; double o0, o1, o2; } of3;

/* Field bundle of the ROMS w-advection kernels (rk2_w_advection.pyx:386-395). */
typedef struct {
    of3 u, v, w;
    of2 dx, dy, h, zeta;
    of1 C;
} oroms_fields;

/* Particle SoA (kernels/_kernels.py:14-19 plus the kernels' own fields). */
typedef struct {
    int64_t n;
    uint8_t *status;
    double *zidx, *yidx, *xidx, *z;
    double *dxidx0, *dyidx0, *dz0; /* AB3 k(n)      ab3_w_advection.pyx:250-258 */
    double *dxidx1, *dyidx1, *dz1; /* RK2 k1 / AB3 k(n-1) */
    double *dxidx2, *dyidx2, *dz2; /* RK2 k2 / AB3 k(n-2) */
} oparticles;

typedef struct {
    double hc;
    int32_t NZ;
    double dt;
    double alpha;
    double bounds[6]; /* zmin zmax ymin ymax xmin xmax (fieldset.py:45-70) */
} oscalars;

/* kernels/_interpolation/linear.pxd:3-9.  `(Py_ssize_t)idx` on x86-64 is
 * cvttsd2si: NaN and out-of-range values give INT64_MIN, which clamps to 0. */
static inline int64_t o_trunc(double idx, int64_t max_idx) {
    int64_t i = (int64_t)idx;
    if (i < 0) i = 0;
    else if (i > max_idx) i = max_idx;
    return i;
}

/* linear.pxd:11-17 */
static inline double o_lin(const of1 *f, double idx) {
    int64_t I0 = o_trunc(idx, f->n0 - 2);
    double f0 = idx - (double)I0;
    double g0 = 1.0 - f0;
    return g0 * f->a[I0] + f0 * f->a[I0 + 1];
}

/* linear.pxd:19-33 */
static inline double o_bilin(const of2 *f, double idx0, double idx1) {
    int64_t I0 = o_trunc(idx0, f->n0 - 2);
    int64_t I1 = o_trunc(idx1, f->n1 - 2);
    double f0 = idx0 - (double)I0, f1 = idx1 - (double)I1;
    double g0 = 1.0 - f0, g1 = 1.0 - f1;
    const double *r0 = f->a + I0 * f->n1, *r1 = r0 + f->n1;
    double v00 = r0[I1], v01 = r0[I1 + 1], v10 = r1[I1], v11 = r1[I1 + 1];
    return g0 * g1 * v00 + g0 * f1 * v01 + f0 * g1 * v10 + f0 * f1 * v11;
}

/* linear.pxd:35-65 */
static inline double o_trilin(const of3 *f, double idx0, double idx1, double idx2) {
    int64_t I0 = o_trunc(idx0, f->n0 - 2);
    int64_t I1 = o_trunc(idx1, f->n1 - 2);
    int64_t I2 = o_trunc(idx2, f->n2 - 2);
    double f0 = idx0 - (double)I0, f1 = idx1 - (double)I1, f2 = idx2 - (double)I2;
    double g0 = 1.0 - f0, g1 = 1.0 - f1, g2 = 1.0 - f2;
    int64_t s1 = f->n2, s0 = f->n1 * f->n2;
    const double *p = f->a + I0 * s0 + I1 * s1 + I2;
    double v000 = p[0], v001 = p[1], v010 = p[s1], v011 = p[s1 + 1];
    double v100 = p[s0], v101 = p[s0 + 1], v110 = p[s0 + s1], v111 = p[s0 + s1 + 1];
    return (g0 * g1 * g2 * v000 +
            g0 * g1 * f2 * v001 +
            g0 * f1 * g2 * v010 +
            g0 * f1 * f2 * v011 +
            f0 * g1 * g2 * v100 +
            f0 * g1 * f2 * v101 +
            f0 * f1 * g2 * v110 +
            f0 * f1 * f2 * v111);
}

/* kernels/roms/_vertical_coordinate.pxd:19-21 */
static inline double o_sigma(double zidx, int32_t Nz) {
    double num = zidx + 0.5;
    if (Nz == 0) return 0.0;
    return num / (double)Nz - 1.0;
}

/* _vertical_coordinate.pxd:23-25 */
static inline double o_S(double hc, double sigma, double h, double C) {
    double num = hc * sigma + h * C;
    double den = hc + h;
    if (den == 0.0) return 0.0;
    return num / den;
}

/* _vertical_coordinate.pxd:31-35 */
static inline double o_compute_z(double zidx, int32_t Nz, double hc, double h, double C, double zeta) {
    double sigma = o_sigma(zidx, Nz);
    double S = o_S(hc, sigma, h, C);
    return zeta + (zeta + h) * S;
}

/* _vertical_coordinate.pxd:41-43 */
static inline double o_S_from_z(double z, double h, double zeta) {
    double num = z - zeta;
    double den = zeta + h;
    if (den == 0.0) return 0.0;
    return num / den;
}

/* _vertical_coordinate.pxd:45-48 */
static inline double o_sigma_from_Cidx(int64_t Cidx, double C_offset, int32_t Nz) {
    double zidx = (double)Cidx - C_offset;
    return o_sigma(zidx, Nz);
}

/* _vertical_coordinate.pxd:50-84 (binary search over the C levels) */
static inline int64_t o_Cidx_from_S(double S, double hc, int32_t NZ, double h, const of1 *C, double C_offset) {
    int64_t C_size = C->n0;
    int64_t lo = 0, hi = C_size - 2, mid;
    double S_mid;
    if (S <= o_S(hc, o_sigma_from_Cidx(0, C_offset, NZ), h, C->a[0])) return 0;
    else if (S >= o_S(hc, o_sigma_from_Cidx(C_size - 2, C_offset, NZ), h, C->a[C_size - 2])) return C_size - 2;
    while (lo < hi - 1) {
        mid = (lo + hi) / 2; /* non-negative: Python floor division == C division */
        S_mid = o_S(hc, o_sigma_from_Cidx(mid, C_offset, NZ), h, C->a[mid]);
        if (S_mid <= S) lo = mid;
        else hi = mid;
    }
    return lo;
}

/* _vertical_coordinate.pxd:86-96 */
static inline double o_zidx_from_S(double S, double hc, int32_t NZ, double h, const of1 *C, double C_offset) {
    int64_t Cidx = o_Cidx_from_S(S, hc, NZ, h, C, C_offset);
    double S_low = o_S(hc, o_sigma_from_Cidx(Cidx, C_offset, NZ), h, C->a[Cidx]);
    double S_high = o_S(hc, o_sigma_from_Cidx(Cidx + 1, C_offset, NZ), h, C->a[Cidx + 1]);
    double num = S - S_low;
    double den = S_high - S_low;
    if (den == 0.0) return 0.0;
    double f = num / den;
    return ((double)Cidx - C_offset) + f;
}

/* _vertical_coordinate.pxd:98-103 */
static inline double o_compute_zidx(double z, double h, double zeta, double hc, int32_t NZ, const of1 *C, double C_offset) {
    double S = o_S_from_z(z, h, zeta);
    return o_zidx_from_S(S, hc, NZ, h, C, C_offset);
}

/* ---------------------------------------------------------------- kernels */

/* kernels/validation.pyx:21-43 */
int oracle_finite_indices(const oparticles *p) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < p->n; ++i) {
        if (p->status[i] & OST_INACTIVE) continue;
        if (!isfinite(p->zidx[i]) || !isfinite(p->yidx[i]) || !isfinite(p->xidx[i]))
            p->status[i] = OST_NONFINITE;
    }
    return 0;
}

/* kernels/validation.pyx:45-77 */
int oracle_domain_bounds(const oparticles *p, const oscalars *s) {
    const double zmin = s->bounds[0], zmax = s->bounds[1];
    const double ymin = s->bounds[2], ymax = s->bounds[3];
    const double xmin = s->bounds[4], xmax = s->bounds[5];
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < p->n; ++i) {
        if (p->status[i] & OST_INACTIVE) continue;
        if (!(zmin <= p->zidx[i] && p->zidx[i] <= zmax &&
              ymin <= p->yidx[i] && p->yidx[i] <= ymax &&
              xmin <= p->xidx[i] && p->xidx[i] <= xmax))
            p->status[i] = OST_OUT_OF_DOMAIN;
    }
    return 0;
}

/* kernels/roms/_roms_core.pyx:17-73 (writes into `out`, the kernel's particle_field) */
int oracle_compute_z(const oparticles *p, double *out, const oscalars *s, const oroms_fields *F) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < p->n; ++i) {
        if (p->status[i] & OST_INACTIVE) continue;
        double h = o_bilin(&F->h, p->yidx[i] + F->h.o0, p->xidx[i] + F->h.o1);
        double zeta = o_bilin(&F->zeta, p->yidx[i] + F->zeta.o0, p->xidx[i] + F->zeta.o1);
        double C = o_lin(&F->C, p->zidx[i] + F->C.o0);
        out[i] = o_compute_z(p->zidx[i], s->NZ, s->hc, h, C, zeta);
    }
    return 0;
}

/* kernels/roms/rk2_w_advection.pyx:31-153 */
int oracle_rk2_step_1(const oparticles *p, const oscalars *s, const oroms_fields *F) {
    int64_t nzero = 0;
    #pragma omp parallel for schedule(static) reduction(+:nzero)
    for (int64_t i = 0; i < p->n; ++i) {
        if (p->status[i] & OST_INACTIVE) continue;
        double zi = p->zidx[i], yi = p->yidx[i], xi = p->xidx[i];
        double h = o_bilin(&F->h, yi + F->h.o0, xi + F->h.o1);
        double zeta = o_bilin(&F->zeta, yi + F->zeta.o0, xi + F->zeta.o1);
        double C = o_lin(&F->C, zi + F->C.o0);
        p->z[i] = o_compute_z(zi, s->NZ, s->hc, h, C, zeta);
        double u = o_trilin(&F->u, zi + F->u.o0, yi + F->u.o1, xi + F->u.o2);
        double v = o_trilin(&F->v, zi + F->v.o0, yi + F->v.o1, xi + F->v.o2);
        double dx = o_bilin(&F->dx, yi + F->dx.o0, xi + F->dx.o1);
        double dy = o_bilin(&F->dy, yi + F->dy.o0, xi + F->dy.o1);
        if (dx == 0.0 || dy == 0.0) { nzero++; continue; }
        p->dxidx1[i] = u / dx;
        p->dyidx1[i] = v / dy;
        p->dz1[i] = o_trilin(&F->w, zi + F->w.o0, yi + F->w.o1, xi + F->w.o2);
    }
    return (int)(nzero > 0x7fffffff ? 0x7fffffff : nzero);
}

/* kernels/roms/rk2_w_advection.pyx:155-275 */
int oracle_rk2_step_2(const oparticles *p, const oscalars *s, const oroms_fields *F) {
    int64_t nzero = 0;
    const double adt = s->alpha * s->dt;
    #pragma omp parallel for schedule(static) reduction(+:nzero)
    for (int64_t i = 0; i < p->n; ++i) {
        if (p->status[i] & OST_INACTIVE) continue;
        double z_int = p->z[i] + adt * p->dz1[i];
        double y_int = p->yidx[i] + adt * p->dyidx1[i];
        double x_int = p->xidx[i] + adt * p->dxidx1[i];
        double h = o_bilin(&F->h, y_int + F->h.o0, x_int + F->h.o1);
        double zeta = o_bilin(&F->zeta, y_int + F->zeta.o0, x_int + F->zeta.o1);
        double z_idx = o_compute_zidx(z_int, h, zeta, s->hc, s->NZ, &F->C, F->C.o0);
        double u = o_trilin(&F->u, z_idx + F->u.o0, y_int + F->u.o1, x_int + F->u.o2);
        double v = o_trilin(&F->v, z_idx + F->v.o0, y_int + F->v.o1, x_int + F->v.o2);
        double dx = o_bilin(&F->dx, y_int + F->dx.o0, x_int + F->dx.o1);
        double dy = o_bilin(&F->dy, y_int + F->dy.o0, x_int + F->dy.o1);
        if (dx == 0.0 || dy == 0.0) { nzero++; continue; }
        p->dxidx2[i] = u / dx;
        p->dyidx2[i] = v / dy;
        p->dz2[i] = o_trilin(&F->w, z_idx + F->w.o0, y_int + F->w.o1, x_int + F->w.o2);
    }
    return (int)(nzero > 0x7fffffff ? 0x7fffffff : nzero);
}

/* kernels/roms/rk2_w_advection.pyx:278-354.  b1 = 1/(2 alpha) weights k1
 * (rk2_w_advection.pyx:317-318), the reference's own convention. */
int oracle_rk2_update(const oparticles *p, const oscalars *s, const oroms_fields *F) {
    const double b1 = 1.0 / (2.0 * s->alpha);
    const double b2 = 1.0 - b1;
    const double b1dt = b1 * s->dt, b2dt = b2 * s->dt;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < p->n; ++i) {
        if (p->status[i] & OST_INACTIVE) continue;
        p->z[i] = p->z[i] + b1dt * p->dz1[i] + b2dt * p->dz2[i];
        p->yidx[i] = p->yidx[i] + b1dt * p->dyidx1[i] + b2dt * p->dyidx2[i];
        p->xidx[i] = p->xidx[i] + b1dt * p->dxidx1[i] + b2dt * p->dxidx2[i];
        double h = o_bilin(&F->h, p->yidx[i] + F->h.o0, p->xidx[i] + F->h.o1);
        double zeta = o_bilin(&F->zeta, p->yidx[i] + F->zeta.o0, p->xidx[i] + F->zeta.o1);
        p->zidx[i] = o_compute_zidx(p->z[i], h, zeta, s->hc, s->NZ, &F->C, F->C.o0);
    }
    return 0;
}

/* kernels/roms/ab3_w_advection.pyx:20-178 */
int oracle_ab3(const oparticles *p, const oscalars *s, const oroms_fields *F) {
    int64_t nzero = 0;
    const double dt = s->dt;
    #pragma omp parallel for schedule(static) reduction(+:nzero)
    for (int64_t i = 0; i < p->n; ++i) {
        if (p->status[i] & OST_INACTIVE) continue;
        double zi = p->zidx[i], yi = p->yidx[i], xi = p->xidx[i];
        double u = o_trilin(&F->u, zi + F->u.o0, yi + F->u.o1, xi + F->u.o2);
        double dx = o_bilin(&F->dx, yi + F->dx.o0, xi + F->dx.o1);
        if (dx == 0.0) { nzero++; continue; }
        p->dxidx0[i] = u / dx;
        double v = o_trilin(&F->v, zi + F->v.o0, yi + F->v.o1, xi + F->v.o2);
        double dy = o_bilin(&F->dy, yi + F->dy.o0, xi + F->dy.o1);
        if (dy == 0.0) { nzero++; continue; }
        p->dyidx0[i] = v / dy;
        p->dz0[i] = o_trilin(&F->w, zi + F->w.o0, yi + F->w.o1, xi + F->w.o2);
        if (p->status[i] == OST_MULTISTEP_1) {
            p->dxidx1[i] = p->dxidx0[i]; p->dyidx1[i] = p->dyidx0[i]; p->dz1[i] = p->dz0[i];
            p->dxidx2[i] = p->dxidx0[i]; p->dyidx2[i] = p->dyidx0[i]; p->dz2[i] = p->dz0[i];
            p->status[i] = OST_MULTISTEP_2;
        } else if (p->status[i] == OST_MULTISTEP_2) {
            p->dxidx2[i] = -p->dxidx0[i] + 2.0 * p->dxidx1[i];
            p->dyidx2[i] = -p->dyidx0[i] + 2.0 * p->dyidx1[i];
            p->dz2[i] = -p->dz0[i] + 2.0 * p->dz1[i];
            p->status[i] = OST_NORMAL;
        }
        double h = o_bilin(&F->h, yi + F->h.o0, xi + F->h.o1);
        double zeta = o_bilin(&F->zeta, yi + F->zeta.o0, xi + F->zeta.o1);
        double C = o_lin(&F->C, zi + F->C.o0);
        p->z[i] = o_compute_z(zi, s->NZ, s->hc, h, C, zeta);
        p->z[i] += dt * (23.0 * p->dz0[i] - 16.0 * p->dz1[i] + 5.0 * p->dz2[i]) / 12.0;
        p->yidx[i] += dt * (23.0 * p->dyidx0[i] - 16.0 * p->dyidx1[i] + 5.0 * p->dyidx2[i]) / 12.0;
        p->xidx[i] += dt * (23.0 * p->dxidx0[i] - 16.0 * p->dxidx1[i] + 5.0 * p->dxidx2[i]) / 12.0;
        p->dz2[i] = p->dz1[i]; p->dxidx2[i] = p->dxidx1[i]; p->dyidx2[i] = p->dyidx1[i];
        p->dz1[i] = p->dz0[i]; p->dxidx1[i] = p->dxidx0[i]; p->dyidx1[i] = p->dyidx0[i];
    }
    return (int)(nzero > 0x7fffffff ? 0x7fffffff : nzero);
}

/* kernels/roms/ab3_isopycnal_following.pyx:26-192: ab3_w_advection's step with
 * the vertical velocity of an isopycnal follower, dz0 = w_max * drho /
 * (rho_scale + |drho|), drho = rho(x) - rho_t (:124-132).  F->w holds rho.
 * A zero divisor (dx, dy, or rho_scale + |drho|) skips the particle and is
 * counted: the reference raises ZeroDivisionError (cdivision=False). */
int oracle_ab3_isopycnal(const oparticles *p, const oscalars *s, const oroms_fields *F, const double *rho_t,
                         double w_max, double rho_scale) {
    int64_t nzero = 0;
    const double dt = s->dt;
    #pragma omp parallel for schedule(static) reduction(+:nzero)
    for (int64_t i = 0; i < p->n; ++i) {
        if (p->status[i] & OST_INACTIVE) continue;
        double zi = p->zidx[i], yi = p->yidx[i], xi = p->xidx[i];
        double u = o_trilin(&F->u, zi + F->u.o0, yi + F->u.o1, xi + F->u.o2);
        double dx = o_bilin(&F->dx, yi + F->dx.o0, xi + F->dx.o1);
        if (dx == 0.0) { nzero++; continue; }
        p->dxidx0[i] = u / dx;
        double v = o_trilin(&F->v, zi + F->v.o0, yi + F->v.o1, xi + F->v.o2);
        double dy = o_bilin(&F->dy, yi + F->dy.o0, xi + F->dy.o1);
        if (dy == 0.0) { nzero++; continue; }
        p->dyidx0[i] = v / dy;
        double rho = o_trilin(&F->w, zi + F->w.o0, yi + F->w.o1, xi + F->w.o2);
        double drho = rho - rho_t[i];
        double den = rho_scale + fabs(drho);
        if (den == 0.0) { nzero++; continue; }
        p->dz0[i] = w_max * drho / den;
        if (p->status[i] == OST_MULTISTEP_1) {
            p->dxidx1[i] = p->dxidx0[i]; p->dyidx1[i] = p->dyidx0[i]; p->dz1[i] = p->dz0[i];
            p->dxidx2[i] = p->dxidx0[i]; p->dyidx2[i] = p->dyidx0[i]; p->dz2[i] = p->dz0[i];
            p->status[i] = OST_MULTISTEP_2;
        } else if (p->status[i] == OST_MULTISTEP_2) {
            p->dxidx2[i] = -p->dxidx0[i] + 2.0 * p->dxidx1[i];
            p->dyidx2[i] = -p->dyidx0[i] + 2.0 * p->dyidx1[i];
            p->dz2[i] = -p->dz0[i] + 2.0 * p->dz1[i];
            p->status[i] = OST_NORMAL;
        }
        double h = o_bilin(&F->h, yi + F->h.o0, xi + F->h.o1);
        double zeta = o_bilin(&F->zeta, yi + F->zeta.o0, xi + F->zeta.o1);
        double C = o_lin(&F->C, zi + F->C.o0);
        p->z[i] = o_compute_z(zi, s->NZ, s->hc, h, C, zeta);
        p->z[i] += dt * (23.0 * p->dz0[i] - 16.0 * p->dz1[i] + 5.0 * p->dz2[i]) / 12.0;
        p->yidx[i] += dt * (23.0 * p->dyidx0[i] - 16.0 * p->dyidx1[i] + 5.0 * p->dyidx2[i]) / 12.0;
        p->xidx[i] += dt * (23.0 * p->dxidx0[i] - 16.0 * p->dxidx1[i] + 5.0 * p->dxidx2[i]) / 12.0;
        p->dz2[i] = p->dz1[i]; p->dxidx2[i] = p->dxidx1[i]; p->dyidx2[i] = p->dyidx1[i];
        p->dz1[i] = p->dz0[i]; p->dxidx1[i] = p->dxidx0[i]; p->dyidx1[i] = p->dyidx0[i];
    }
    return (int)(nzero > 0x7fffffff ? 0x7fffffff : nzero);
}

/* kernels/roms/ab3_w_advection.pyx:180-229 (and ab3_isopycnal_following.pyx:194-241, the same post step) */
int oracle_ab3_post(const oparticles *p, const oscalars *s, const oroms_fields *F) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < p->n; ++i) {
        if (p->status[i] & OST_INACTIVE) continue;
        double h = o_bilin(&F->h, p->yidx[i] + F->h.o0, p->xidx[i] + F->h.o1);
        double zeta = o_bilin(&F->zeta, p->yidx[i] + F->zeta.o0, p->xidx[i] + F->zeta.o1);
        p->zidx[i] = o_compute_zidx(p->z[i], h, zeta, s->hc, s->NZ, &F->C, F->C.o0);
    }
    return 0;
}

/* The primitives, exported for known-answer tests of the oracle itself. */
double oracle_trilinear(const of3 *f, double i0, double i1, double i2) { return o_trilin(f, i0, i1, i2); }
double oracle_bilinear(const of2 *f, double i0, double i1) { return o_bilin(f, i0, i1); }
double oracle_linear(const of1 *f, double i0) { return o_lin(f, i0); }
double oracle_compute_z_scalar(double zidx, int32_t Nz, double hc, double h, double C, double zeta) {
    return o_compute_z(zidx, Nz, hc, h, C, zeta);
}
double oracle_compute_zidx_scalar(double z, double h, double zeta, double hc, int32_t NZ, const of1 *C) {
    return o_compute_zidx(z, h, zeta, hc, NZ, C, C->o0);
}
