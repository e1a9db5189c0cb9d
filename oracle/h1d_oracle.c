/*
 * h1d_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the hybrid_1d per-step hot path
 * of kyungguk1/hybrid_code-hfemic_wave, used as the checker of the CUDA implementation.
 * Nothing in the product links, loads or calls this file; only tests/, the smoke check and
 * the CPU-baseline leg of bench.py do.
 *
 * It restates, with runtime sizes instead of the reference's template constants:
 *   Domain_CAMCL::advance_by / cycle / subcycle / current_advance  (src/hybrid_1d/Core/Domain_CAMCL.cc:21-193)
 *   Domain_PC::advance_by / predictor_step / corrector_step         (Core/Domain_PC.cc:21-205)
 *   Domain::collect_smooth                                          (Core/Domain.hh:35-74)
 *   PartSpecies::update_vel/update_pos/collect_part/collect_all     (Core/PartSpecies.cc:27-34, 105-244)
 *   PartSpecies::impl_update_weight, equilibrium moments            (Core/PartSpecies.cc:82-89, 115-143, 178-208;
 *                                                                    VDF/{Maxwellian,Losscone,PartialShell,CounterBeam}VDF)
 *   ColdSpecies::update_vel/collect_part/collect_all                (Core/ColdSpecies.cc:31-77)
 *   BField::update, EField::update, Charge/Current/Lambda/Gamma     (Core/BField.cc:24-74, EField.cc:41-126,
 *                                                                    Charge.cc:26-36, Current.cc:29-52)
 *   BorisPush::non_relativistic, Shape<1..3>, GridArray interp/deposit/smooth, MaskingFunction,
 *   CurviBasis/MFABasis/MirrorGeometry                              (LibPIC/PIC headers)
 *   Delegate particle partition / periodic / reflecting pass, ghost pass and gather semantics of
 *   SubdomainDelegate with a single subdomain (Boundary/Delegate.cc:51-156,
 *   Boundary/SubdomainDelegate.cc:58-181)
 *   EnergyRecorder::dump                                            (Recorder/EnergyRecorder.cc:98-140)
 *
 * Every floating-point expression keeps the reference's evaluation order, and the particle
 * container keeps the reference's std::deque order (std::partition is the two-pointer
 * partition of libstdc++ for bidirectional iterators), so that with -ffp-contract=off on both
 * sides this code reproduces the compiled reference bit for bit.  The one deliberate
 * difference: gyro-phase randomisation of reflected particles draws from a counter-based hash
 * instead of std::random_device (Delegate.cc:148), so that it is reproducible.
 */
#define _DEFAULT_SOURCE
#include "../include/h1d_gpu.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define P H1D_PAD

typedef struct {
    double x, y, z;
} V3;

typedef struct {
    int64_t  n, cap;
    double  *q1, *vx, *vy, *vz, *w;
    int64_t *pid;
    double  *real_f, *marker; /* Particle::PSD (Particle.h:26-34) */
} Bucket;

typedef struct orc_run {
    h1d_params p;
    long       Nx, M; /* M = Nx + 2P */
    double     full_min, full_len, half_min; /* extents (ParamSet.cc:22-23) */
    /* geometry (MirrorGeometry.cc:13-22, CurviBasis.h:32-35, MFABasis.h:29-32) */
    double xi, xi2, D1, D2, D3, inv_D1, inv_D2, inv_D3, sqrt_g;
    int    homogeneous;
    /* grids, GridArray layout (M elements, ghosts included) */
    double *B, *B1, *E, *E1;             /* CartVector */
    double *charge, *charge1, *rho, *lambda; /* Scalar */
    double *current, *current1, *J, *gamma;  /* CartVector */
    double *smooth_buf;                  /* CartVector-sized scratch for smooth_assign */
    double *Bprev, *Ecovar;              /* BField internals */
    double *Pe, *dPe, *Je, *covar, *contr; /* EField internals */
    /* kinetic species */
    Bucket  part[H1D_MAX_KINETIC];
    Bucket  pred;            /* Domain_PC::part_predict bucket */
    double *mom0[H1D_MAX_KINETIC], *mom1[H1D_MAX_KINETIC], *mom2[H1D_MAX_KINETIC];
    double *eq0[H1D_MAX_KINETIC], *eq2[H1D_MAX_KINETIC]; /* PartSpecies::equilibrium_mom0/2 (nV0 = 0) */
    double *pmom0, *pmom1;   /* predictor moments */
    /* cold species */
    double *cn_full[H1D_MAX_COLD], *cnV_full[H1D_MAX_COLD];
    double *cmom0[H1D_MAX_COLD], *cmom1[H1D_MAX_COLD], *cmom2[H1D_MAX_COLD];
    double *pc_n_full, *pc_nV_full;
    /* external sources: moment<0> (always zero) and moment<1> of the last update */
    double *smom0[H1D_MAX_SOURCES], *smom1[H1D_MAX_SOURCES];
    /* bucket buffers of the delegate */
    Bucket  bufL, bufR;
    int     recurring;
    int64_t step;
    char    msg[512];
} orc_run;

/* ------------------------------------------------------------------------------------------------
 * small helpers
 */
static inline double *at1(double *g, long i) { return g + (i + P); }
static inline double *at3(double *g, long i) { return g + 3 * (i + P); }
static inline double *at6(double *g, long i) { return g + 6 * (i + P); }

static void *xcalloc(size_t n, size_t sz)
{
    void *p = calloc(n ? n : 1, sz);
    if (!p) {
        fprintf(stderr, "oracle: out of memory\n");
        abort();
    }
    return p;
}

static void bucket_reserve(Bucket *b, int64_t cap)
{
    if (cap <= b->cap)
        return;
    int64_t nc = b->cap ? b->cap : 64;
    while (nc < cap)
        nc *= 2;
    b->q1  = realloc(b->q1, sizeof(double) * nc);
    b->vx  = realloc(b->vx, sizeof(double) * nc);
    b->vy  = realloc(b->vy, sizeof(double) * nc);
    b->vz  = realloc(b->vz, sizeof(double) * nc);
    b->w   = realloc(b->w, sizeof(double) * nc);
    b->pid = realloc(b->pid, sizeof(int64_t) * nc);
    b->real_f = realloc(b->real_f, sizeof(double) * nc);
    b->marker = realloc(b->marker, sizeof(double) * nc);
    if (!b->q1 || !b->vx || !b->vy || !b->vz || !b->w || !b->pid || !b->real_f || !b->marker) {
        fprintf(stderr, "oracle: out of memory\n");
        abort();
    }
    b->cap = nc;
}
static void bucket_free(Bucket *b)
{
    free(b->q1), free(b->vx), free(b->vy), free(b->vz), free(b->w), free(b->pid);
    free(b->real_f), free(b->marker);
    memset(b, 0, sizeof *b);
}
static void bucket_swap_elems(Bucket *b, int64_t i, int64_t j)
{
    double t;
    t = b->q1[i], b->q1[i] = b->q1[j], b->q1[j] = t;
    t = b->vx[i], b->vx[i] = b->vx[j], b->vx[j] = t;
    t = b->vy[i], b->vy[i] = b->vy[j], b->vy[j] = t;
    t = b->vz[i], b->vz[i] = b->vz[j], b->vz[j] = t;
    t = b->w[i], b->w[i] = b->w[j], b->w[j] = t;
    t = b->real_f[i], b->real_f[i] = b->real_f[j], b->real_f[j] = t;
    t = b->marker[i], b->marker[i] = b->marker[j], b->marker[j] = t;
    int64_t u = b->pid[i];
    b->pid[i] = b->pid[j], b->pid[j] = u;
}
static void bucket_push(Bucket *dst, Bucket const *src, int64_t k)
{
    bucket_reserve(dst, dst->n + 1);
    int64_t i   = dst->n++;
    dst->q1[i]  = src->q1[k];
    dst->vx[i]  = src->vx[k];
    dst->vy[i]  = src->vy[k];
    dst->vz[i]  = src->vz[k];
    dst->w[i]   = src->w[k];
    dst->pid[i] = src->pid[k];
    dst->real_f[i] = src->real_f[k];
    dst->marker[i] = src->marker[k];
}
static void bucket_copy(Bucket *dst, Bucket const *src)
{
    bucket_reserve(dst, src->n);
    dst->n = src->n;
    memcpy(dst->q1, src->q1, sizeof(double) * src->n);
    memcpy(dst->vx, src->vx, sizeof(double) * src->n);
    memcpy(dst->vy, src->vy, sizeof(double) * src->n);
    memcpy(dst->vz, src->vz, sizeof(double) * src->n);
    memcpy(dst->w, src->w, sizeof(double) * src->n);
    memcpy(dst->pid, src->pid, sizeof(int64_t) * src->n);
    memcpy(dst->real_f, src->real_f, sizeof(double) * src->n);
    memcpy(dst->marker, src->marker, sizeof(double) * src->n);
}

/* ------------------------------------------------------------------------------------------------
 * geometry (LibPIC/PIC/Geometry/CurviBasis.h, MFABasis.h, MirrorGeometry.cc)
 */
/* inv_sqrt_BOB0(CurviCoord) = cos(xi*D1*q1)   (CurviBasis.h:42, MFABasis.h:39) */
static inline double g_cos(orc_run const *R, double q1) { return cos(R->xi * R->D1 * q1); }
/* BOB0(CurviCoord) = pow2(1/inv_sqrt_BOB0)     (CurviBasis.h:43) */
static inline double g_BOB0(orc_run const *R, double q1)
{
    double t = 1 / g_cos(R, q1);
    return t * t;
}
/* symmetric tensor {xx,yy,zz,0,0,0} . vector  (TensorTemplate.h:294-301) */
static inline V3 tdot(double xx, double yy, double zz, V3 b)
{
    double const xy = 0, yz = 0, zx = 0;
    V3 r = { xx * b.x + xy * b.y + zx * b.z, xy * b.x + yy * b.y + yz * b.z,
             zx * b.x + yz * b.y + zz * b.z };
    return r;
}
/* cart_to_covar(v, pos) = covar_basis<0>(pos) . v   (CurviBasis.h:52-56, 158, 204) */
static inline V3 g_cart_to_covar(orc_run const *R, V3 v, double q1)
{
    double tmp = g_cos(R, q1);
    return tdot(R->D1 / (tmp * tmp), R->D2 * tmp, R->D3 * tmp, v);
}
/* cart_to_contr(v, pos) = contr_basis<0>(pos) . v   (CurviBasis.h:65-69, 146, 188) */
static inline V3 g_cart_to_contr(orc_run const *R, V3 v, double q1)
{
    double tmp = g_cos(R, q1);
    return tdot(R->inv_D1 * (tmp * tmp), R->inv_D2 / tmp, R->inv_D3 / tmp, v);
}
/* contr_to_cart = v . covar_basis<0>   (CurviBasis.h:152, 196) */
static inline V3 g_contr_to_cart(orc_run const *R, V3 v, double q1) { return g_cart_to_covar(R, v, q1); }
/* covar_to_cart = v . contr_basis<0>   (CurviBasis.h:164, 212) */
static inline V3 g_covar_to_cart(orc_run const *R, V3 v, double q1) { return g_cart_to_contr(R, v, q1); }
/* Bcart(CurviCoord) = {BOB0, 0, 0} * O0   (MFABasis.h:47, Geometry.h:44) */
static inline V3 g_Bcart(orc_run const *R, double q1)
{
    double const O0 = R->p.O0;
    V3 r = { g_BOB0(R, q1) * O0, 0 * O0, 0 * O0 };
    return r;
}
/* Bcontr(CurviCoord) = {1/D1, 0, 0} * O0   (MFABasis.h:43, Geometry.h:36) */
static inline V3 g_Bcontr(orc_run const *R)
{
    double const O0 = R->p.O0;
    V3 r = { R->inv_D1 * O0, 0 * O0, 0 * O0 };
    return r;
}
/* curvilinear -> Cartesian x (MirrorGeometry.cc:34-47) */
static inline double g_curvi_to_cart(orc_run const *R, double q1)
{
    if (R->homogeneous) {
        double const D1q1 = q1 * R->D1;
        return D1q1 * (1 + R->xi * R->xi * D1q1 * D1q1 / 3);
    } else {
        double const xiD1q1 = R->xi * R->D1 * q1;
        return tan(xiD1q1) / R->xi;
    }
}
/* Bcart(CurviCoord, y, z) = Bcart_div_B0(cotrans(pos), y, z) * B0  (MirrorGeometry.h:68-71, MFABasis.h:72-75) */
static inline V3 g_Bcart_yz(orc_run const *R, double q1, double y, double z)
{
    double const x  = g_curvi_to_cart(R, q1);
    double const O0 = R->p.O0;
    V3 r = { (1 + R->xi2 * (x * x)) * O0, -R->xi2 * x * y * O0, -R->xi2 * x * z * O0 };
    return r;
}

/* MaskingFunction::operator() (MaskingFunction.h:28-35) */
static inline double mask_fn(long inset, double factor, double offset)
{
    double const a = offset < 0 ? -offset : offset;
    if (0 == inset || a > (double)inset)
        return 1;
    double const tmp = factor * (1 - a / (double)inset);
    return (1 - tmp) * (1 + tmp);
}
/* BField::mask / EField::mask (BField.cc:40-48, EField.cc:52-61): whole-domain subdomain, offsets 0 */
static void mask_grid(orc_run const *R, double *g, int ncomp, long inset, double factor)
{
    long const N = R->Nx;
    for (long i = 0, first = 0, last = N - 1; i < N; ++i) {
        double const f = mask_fn(inset, factor, 0.0 + (double)i);
        double *a = g + ncomp * (first++ + P);
        for (int c = 0; c < ncomp; ++c)
            a[c] *= f;
        double *b = g + ncomp * (last-- + P);
        for (int c = 0; c < ncomp; ++c)
            b[c] *= f;
    }
}

/* ------------------------------------------------------------------------------------------------
 * shape functions (LibPIC/PIC/Shape.h)
 */
typedef struct {
    long   i[4];
    double w[4];
} Shp;

static inline void shape1(Shp *s, double x)
{
    s->i[0] = s->i[1] = (long)floor(x);
    s->i[1] += 1;
    s->w[1] = x - (double)s->i[0];
    s->w[0] = 1 - s->w[1];
}
static inline void shape2(Shp *s, double x)
{
    double const half = 0.5, f3_4 = 0.75;
    s->i[0] = s->i[1] = s->i[2] = (long)round(x);
    s->i[0] -= 1;
    s->i[2] += 1;
    x       = (double)s->i[1] - x;
    s->w[1] = f3_4 - (x * x);
    x += half;
    s->w[0] = half * (x * x);
    s->w[2] = 1 - (s->w[0] + s->w[1]);
}
static inline void shape3(Shp *s, double x)
{
    s->w[0] = s->w[1] = s->w[2] = s->w[3] = 1. / 6;
    s->i[0]                              = (long)ceil(x) - 2;
    s->i[1]                              = s->i[0] + 1;
    s->i[2]                              = s->i[1] + 1;
    s->i[3]                              = s->i[2] + 1;
    double tmp;
    tmp = 2 + ((double)s->i[0] - x);
    s->w[0] *= tmp * tmp * tmp;
    tmp = 2 - ((double)s->i[3] - x);
    s->w[3] *= tmp * tmp * tmp;
    tmp = x - (double)s->i[1];
    s->w[1] *= 4 + 3 * tmp * tmp * (tmp - 2);
    s->w[2] = 1 - (s->w[0] + s->w[1] + s->w[3]);
}
static inline void shape(Shp *s, int order, double x)
{
    if (order == 1)
        shape1(s, x);
    else if (order == 2)
        shape2(s, x);
    else
        shape3(s, x);
}
/* GridArray::interp (GridArray.h:110-119) for a CartVector grid */
static inline V3 interp3(double *g, Shp const *s, int order)
{
    V3 y = { 0, 0, 0 };
    for (int j = 0; j <= order; ++j) {
        double const *a = at3(g, s->i[j]);
        y.x += a[0] * s->w[j];
        y.y += a[1] * s->w[j];
        y.z += a[2] * s->w[j];
    }
    return y;
}

/* ------------------------------------------------------------------------------------------------
 * Boris push (LibPIC/PIC/BorisPush.h:25-30, 57-73, 99-102)
 */
typedef struct {
    double dtOc_2O0, cDtOc_2O0;
} Boris;
static inline Boris boris_make(double dt, double c, double O0, double Oc)
{
    Boris b;
    double const dt_2 = 0.5 * dt;
    b.dtOc_2O0  = Oc * dt_2 / O0;
    b.cDtOc_2O0 = c * b.dtOc_2O0;
    return b;
}
static inline V3 cross3(V3 A, V3 B)
{
    V3 r = { A.y * B.z - A.z * B.y, A.z * B.x - A.x * B.z, A.x * B.y - A.y * B.x };
    return r;
}
static inline void boris_push(Boris const *b, V3 *v, V3 B, V3 E)
{
    B.x *= b->dtOc_2O0, B.y *= b->dtOc_2O0, B.z *= b->dtOc_2O0;
    E.x *= b->cDtOc_2O0, E.y *= b->cDtOc_2O0, E.z *= b->cDtOc_2O0;
    v->x += E.x, v->y += E.y, v->z += E.z;
    /* rotate: cross(v + cross(v, B), (2 / (1 + dot(B, B))) * B) */
    V3 const     vxB = cross3(*v, B);
    V3 const     u   = { v->x + vxB.x, v->y + vxB.y, v->z + vxB.z };
    double const s   = 2 / (1 + (B.x * B.x + B.y * B.y + B.z * B.z));
    V3 const     sB  = { B.x * s, B.y * s, B.z * s };
    V3 const     r   = cross3(u, sB);
    v->x += r.x, v->y += r.y, v->z += r.z;
    v->x += E.x, v->y += E.y, v->z += E.z;
}

/* ------------------------------------------------------------------------------------------------
 * ghost pass / gather with one subdomain (SubdomainDelegate.cc:58-89, 122-181)
 */
static void pass_grid(orc_run const *R, double *g, int nc)
{
    long const N = R->Nx;
    /* recv into [end, end+P) from [begin, begin+P); then [begin-P, begin) from [end-P, end) */
    for (long k = 0; k < P; ++k)
        for (int c = 0; c < nc; ++c)
            g[nc * (N + k + P) + c] = g[nc * (k + P) + c];
    for (long k = -P; k < 0; ++k)
        for (int c = 0; c < nc; ++c)
            g[nc * (k + P) + c] = g[nc * (N + k + P) + c];
}
static void gather_grid(orc_run const *R, double *g, int nc)
{
    long const N = R->Nx;
    if (R->p.particle_bc == H1D_BC_REFLECTING || R->p.particle_bc == H1D_BC_ABSORBING) {
        /* moments accumulate at the first/last grid point (SubdomainDelegate.cc:130-141) */
        for (long i = -P; i < 0; ++i)
            for (int c = 0; c < nc; ++c) {
                g[nc * (i + 1 + P) + c] += g[nc * (i + P) + c];
                g[nc * (i + P) + c] = 0;
            }
        for (long i = N + P - 1; i >= N; --i)
            for (int c = 0; c < nc; ++c) {
                g[nc * (i - 1 + P) + c] += g[nc * (i + P) + c];
                g[nc * (i + P) + c] = 0;
            }
    }
    /* mpi_gather with self as both neighbours: payloads are taken before accumulation */
    double left[6 * P], right[6 * P];
    for (long k = 0; k < P; ++k)
        for (int c = 0; c < nc; ++c) {
            left[nc * k + c]  = g[nc * (-P + k + P) + c];
            right[nc * k + c] = g[nc * (N + k + P) + c];
        }
    for (long k = 0; k < P; ++k)
        for (int c = 0; c < nc; ++c)
            g[nc * (N - P + k + P) + c] = g[nc * (N - P + k + P) + c] + left[nc * k + c];
    for (long k = 0; k < P; ++k)
        for (int c = 0; c < nc; ++c)
            g[nc * (k + P) + c] = g[nc * (k + P) + c] + right[nc * k + c];
}

/* Charge::smooth / Current::smooth: swap(buffer.smooth_assign(*this)) (GridArray.h:134-142).
 * The ghost cells of the result are stale in the reference and are always refilled by the next
 * boundary_pass before being read; here they keep the old values. */
static void smooth_grid(orc_run *R, double *g, int nc)
{
    long const N   = R->Nx;
    double    *buf = R->smooth_buf;
    for (long i = 0; i < N; ++i)
        for (int c = 0; c < nc; ++c)
            buf[nc * (i + P) + c]
                = (g[nc * (i - 1 + P) + c] + 2 * g[nc * (i + P) + c] + g[nc * (i + 1 + P) + c]) * .25;
    for (long i = 0; i < N; ++i)
        for (int c = 0; c < nc; ++c)
            g[nc * (i + P) + c] = buf[nc * (i + P) + c];
}

/* ------------------------------------------------------------------------------------------------
 * species helpers
 */
static double cdcf(orc_run const *R, double Oc, double op) { return ((op * op) * R->p.O0) / Oc; } /* Species.h:42-45 */
static double ccf(orc_run const *R, double Oc, double op) { return cdcf(R, Oc, op) / R->p.c; }   /* Species.h:46-49 */

/* half_grid (PartSpecies.cc:27-34): B averaged onto the half grid; last ghost NaN */
static void half_grid(orc_run const *R, double *full, double const *half)
{
    long const N = R->Nx;
    for (long i = -P; i < N - 1 + P; ++i)
        for (int c = 0; c < 3; ++c)
            full[3 * (i + P) + c] = (half[3 * (i + 1 + P) + c] + half[3 * (i + P) + c]) * 0.5;
    for (int c = 0; c < 3; ++c)
        full[3 * (R->M - 1) + c] = NAN;
}

/* PartSpecies::impl_update_velocity<O> (PartSpecies.cc:161-176) */
static void update_weight(orc_run const *R, Bucket *b, h1d_kinetic_desc const *d, double dt);
static int  evolves_psd(h1d_kinetic_desc const *d);
static void update_velocity(orc_run *R, Bucket *b, h1d_kinetic_desc const *d, double *dB, double *E, double dt)
{
    Boris const  boris = boris_make(dt, R->p.c, R->p.O0, d->Oc);
    double const q1min = R->half_min;
    int const    O     = (int)d->shape_order;
    for (int64_t k = 0; k < b->n; ++k) {
        Shp sx;
        shape(&sx, O, b->q1[k] - q1min);
        double const Oc   = d->Oc * g_BOB0(R, b->q1[k]);
        double const rL_y = -b->vz[k] / Oc;
        double const rL_z = +b->vy[k] / Oc;
        V3 const     B0   = g_Bcart_yz(R, b->q1[k], rL_y, rL_z);
        V3 const     dBi  = interp3(dB, &sx, O);
        V3 const     Bt   = { B0.x + dBi.x, B0.y + dBi.y, B0.z + dBi.z };
        V3 const     Ei   = interp3(E, &sx, O);
        V3           v    = { b->vx[k], b->vy[k], b->vz[k] };
        boris_push(&boris, &v, Bt, Ei);
        b->vx[k] = v.x, b->vy[k] = v.y, b->vz[k] = v.z;
    }
    if (evolves_psd(d))
        update_weight(R, b, d, dt);
}
/* The equilibrium distribution a species' weights refer to (h1d_kinetic_desc::vdf): n0(q1), the
 * diagonal of nvv0(q1) (field-aligned = Cartesian on the axis) and the physical f0(vel, q1).
 *   MaxwellianVDF    (VDF/MaxwellianVDF.cc:33-86, .h:56-70)
 *   LossconeVDF      (VDF/LossconeVDF.cc:15-117, .h:69-83)
 *   PartialShellVDF  (VDF/PartialShellVDF.cc:14-145, .h:62-76)
 *   CounterBeamVDF   (VDF/CounterBeamVDF.cc:14-178, .h:62-75) */

/* Dawson's integral F(x), x > 0 (CounterBeamVDF's B(nu) = 2 nu F(1/nu)); the reference evaluates it
 * with the Faddeeva package (Misc/Faddeeva.cc).  Here: Maclaurin series below 0.2, Rybicki's
 * sampling-theorem sum pi^-1/2 sum_{n odd} exp(-(x - n h)^2)/n with h = 0.2 up to 50 (G. B. Rybicki,
 * Computers in Physics 3(2), 85 (1989)), the asymptotic series beyond; relative error < 2e-15. */
static double orc_dawson(double x)
{
    if (x < 0.2) {
        double t = x, sum = x;
        for (int n = 1; n < 40; ++n)
            sum += (t *= -2 * x * x / (2 * n + 1));
        return sum;
    }
    if (x > 50) {
        double const r = 1 / (2 * x * x);
        double       t = 1, sum = 1;
        for (int k = 1; k < 12; ++k)
            sum += (t *= (2 * k - 1) * r);
        return sum / (2 * x);
    }
    long const lo  = (long)floor((x - 7) / 0.2) | 1, hi = (long)ceil((x + 7) / 0.2);
    double     sum = 0;
    for (long n = lo; n <= hi; n += 2)
        sum += exp(-(x - (double)n * 0.2) * (x - (double)n * 0.2)) / (double)n;
    return sum / sqrt(M_PI);
}
static double bnu(double nu) { return 2 * nu * orc_dawson(1 / nu); }

/* loss-cone beta kept 1e-10 away from 0 and 1 (LossconeVDF.cc:25-30, 68-76) */
static double lc_nudge(double beta) { return fabs(beta - 1) < 1e-10 ? beta + copysign(1e-10, beta - 1) : beta; }
static double lc_beta_eq(h1d_kinetic_desc const *d) { return d->vdf_param[0] < 1e-10 ? 1e-10 : lc_nudge(d->vdf_param[0]); }

/* speed normalisation A(xs) and T / vth^2 of the shell distributions (PartialShellVDF.cc:14-22,
 * CounterBeamVDF.cc:20-35) */
static void shell_params(double xs, double *Ab, double *T_vth2)
{
    *Ab     = .5 * (xs * exp(-xs * xs) + 2 / M_2_SQRTPI * (.5 + xs * xs) * erfc(-xs));
    *T_vth2 = .5 / *Ab * (xs * (2.5 + xs * xs) * exp(-xs * xs) + 2 / M_2_SQRTPI * (0.75 + xs * xs * (3 + xs * xs)) * erfc(-xs));
}

static double vdf_cos(orc_run const *R, double q1) { return cos(R->xi * R->D1 * q1); }
/* n0(q1) and, when vv is given, the diagonal of nvv0(q1) */
static double vdf_n0(orc_run const *R, h1d_kinetic_desc const *d, double q1, double vv[3])
{
    double const cs = vdf_cos(R, q1);
    switch (d->vdf) {
        case H1D_VDF_LOSSCONE: {
            double const beq   = lc_beta_eq(d), X = d->T2_T1 / (1 + beq);
            double const eta   = 1 / (X + (1 - X) * cs * cs);
            double const tmp   = beq * X;
            double const eta_b = 1 / (tmp + (1 - tmp) * cs * cs);
            double const n0    = 1 * (eta - beq * eta_b) / (1 - beq);
            if (vv) {
                double const T2OT1 = (1 + lc_nudge(beq * eta_b / eta)) * (X * eta);
                double const h     = .5 * d->vth1 * d->vth1;
                vv[0] = (1 * h) * n0, vv[1] = (T2OT1 * h) * n0, vv[2] = (T2OT1 * h) * n0;
            }
            return n0;
        }
        case H1D_VDF_PARTIAL_SHELL: {
            long const   zeta = (long)d->vdf_param[0];
            double const n0   = 1 * (zeta == 0 ? 1 : pow(cs, (double)zeta));
            if (vv) {
                double Ab, T_vth2;
                shell_params(d->vdf_param[1] / d->vth1, &Ab, &T_vth2);
                double const T1    = T_vth2 / (double)(3 + zeta) * (d->vth1 * d->vth1);
                double const T2OT1 = (double)(2 + zeta) / 2;
                vv[0] = (1 * T1) * n0, vv[1] = (T2OT1 * T1) * n0, vv[2] = (T2OT1 * T1) * n0;
            }
            return n0;
        }
        case H1D_VDF_COUNTER_BEAM: {
            double const nu0 = d->vdf_param[0], nu = nu0 * sqrt((1 / cs) * (1 / cs));
            double const n0  = 1 * (bnu(nu) / bnu(nu0));
            if (vv) {
                double Ab, T_vth2;
                shell_params(d->vdf_param[1] / d->vth1, &Ab, &T_vth2);
                double const T1OT = 0.5 * nu * (1 / orc_dawson(1 / nu) - nu), T2OT = 0.5 * (1 - T1OT);
                double const nT   = n0 * T_vth2 * (d->vth1 * d->vth1);
                vv[0] = T1OT * nT, vv[1] = T2OT * nT, vv[2] = T2OT * nT;
            }
            return n0;
        }
        default: {
            double const eta = 1 / (d->T2_T1 + (1 - d->T2_T1) * cs * cs);
            if (vv) {
                double const T = d->T2_T1 * eta, hv2 = .5 * (d->vth1 * d->vth1);
                vv[0] = (1 * hv2) * eta, vv[1] = (T * hv2) * eta, vv[2] = (T * hv2) * eta;
            }
            return 1 * eta;
        }
    }
}
static double vdf_f0(orc_run const *R, h1d_kinetic_desc const *d, V3 v, double q1)
{
    double const vth1 = d->vth1, vth1_cubed = vth1 * vth1 * vth1;
    double const x1 = v.x / vth1, x2 = v.y / vth1, x3 = v.z / vth1; /* cart_to_mfa is the identity on the axis */
    double const n0 = vdf_n0(R, d, q1, NULL);
    double const cs = vdf_cos(R, q1);
    switch (d->vdf) {
        case H1D_VDF_LOSSCONE: {
            double const beq   = lc_beta_eq(d), X = d->T2_T1 / (1 + beq);
            double const eta   = 1 / (X + (1 - X) * cs * cs);
            double const tmp   = beq * X;
            double const eta_b = 1 / (tmp + (1 - tmp) * cs * cs);
            double const beta  = lc_nudge(beq * eta_b / eta);
            double const xth2  = X * eta;
            double const f1    = exp(-x1 * x1) * M_2_SQRTPI * .5;
            double const y     = (x2 * x2 + x3 * x3) / xth2;
            double const f2    = ((1 - 0 * beta) * exp(-y) - (1 - 0) * exp(-y / beta)) / (M_PI * xth2 * (1 - beta));
            return n0 * ((f1 * f2) / vth1_cubed);
        }
        case H1D_VDF_PARTIAL_SHELL:
        case H1D_VDF_COUNTER_BEAM: {
            double Ab, T_vth2;
            shell_params(d->vdf_param[1] / vth1, &Ab, &T_vth2);
            double const x  = sqrt(x1 * x1 + x2 * x2 + x3 * x3);
            double const t  = x - d->vdf_param[1] / vth1;
            double const fv = exp(-t * t) / Ab;
            double const u  = x1 / x;
            if (d->vdf == H1D_VDF_PARTIAL_SHELL) {
                long const   zeta = (long)d->vdf_param[0];
                double const Bz   = 2 / M_2_SQRTPI * tgamma(1 + .5 * (double)zeta) / tgamma(1.5 + .5 * (double)zeta);
                double const fa   = (zeta == 0 ? 1 : pow((1 - u) * (1 + u), .5 * (double)zeta)) / Bz;
                return n0 * (.5 * fv * fa / (M_PI * vth1_cubed));
            }
            double const nu = d->vdf_param[0] * sqrt((1 / cs) * (1 / cs));
            double const fa = exp(-((1 - u) * (1 + u)) / (nu * nu)) / bnu(nu);
            return n0 * (fv * fa / (2 * M_PI * vth1_cubed));
        }
        default: {
            double const T2OT1 = d->T2_T1 * n0;
            double const f1    = exp(-x1 * x1) * M_2_SQRTPI * .5;
            double const xx    = x2 * x2 + x3 * x3;
            double const f2    = exp(-xx / T2OT1) / (M_PI * T2OT1);
            return n0 * ((f1 * f2) / vth1_cubed);
        }
    }
}
static int evolves_psd(h1d_kinetic_desc const *d) { return d->scheme == H1D_DELTA_F || d->psd_refresh_frequency != 0; }

/* PartSpecies::impl_update_weight (PartSpecies.cc:178-208) with nu_dt = psd_refresh_frequency * dt */
static void update_weight(orc_run const *R, Bucket *b, h1d_kinetic_desc const *d, double dt)
{
    double const nu_dt   = d->psd_refresh_frequency * dt;
    int const    refresh = d->psd_refresh_frequency != 0;
    if (d->scheme == H1D_FULL_F) {
        if (!refresh)
            return;
        for (int64_t k = 0; k < b->n; ++k) {
            V3 const v  = { b->vx[k], b->vy[k], b->vz[k] };
            b->real_f[k] = (b->real_f[k] + nu_dt * vdf_f0(R, d, v, b->q1[k])) / (1 + nu_dt);
            b->w[k]      = b->real_f[k] / b->marker[k];
        }
    } else {
        for (int64_t k = 0; k < b->n; ++k) {
            V3 const     v  = { b->vx[k], b->vy[k], b->vz[k] };
            double const f0 = vdf_f0(R, d, v, b->q1[k]);
            if (refresh)
                b->real_f[k] = (b->real_f[k] + nu_dt * f0) / (1 + nu_dt);
            b->w[k] = (b->real_f[k] - f0) / b->marker[k];
        }
    }
}

/* the equilibrium moments cached by PartSpecies::populate (PartSpecies.cc:82-89) at the interior
 * half-grid points; ghost cells stay zero */
static void cache_equilibrium(orc_run *R, int s)
{
    h1d_kinetic_desc const *d = &R->p.kinetic[s];
    double const            q1min = R->half_min;
    for (long i = 0; i < R->Nx; ++i) {
        double const q1 = (double)i + q1min;
        double       vv[3];
        *at1(R->eq0[s], i) = vdf_n0(R, d, q1, vv);
        double *e = at6(R->eq2[s], i);
        e[0] = vv[0], e[1] = vv[1], e[2] = vv[2], e[3] = 0, e[4] = 0, e[5] = 0;
    }
}
/* delta-f: moments += equilibrium * m_moment_weighting_factor (PartSpecies.cc:115-143), over all
 * cells (GridArray dead_begin..dead_end) */
static void add_equilibrium(orc_run const *R, int s, double *n, double *nV, double *nvv)
{
    if (R->p.kinetic[s].scheme != H1D_DELTA_F)
        return;
    for (long i = 0; i < R->M; ++i)
        n[i] = n[i] + R->eq0[s][i] * 1.0;
    for (long i = 0; i < 3 * R->M; ++i)
        nV[i] = nV[i] + 0.0 * 1.0;
    if (nvv)
        for (long i = 0; i < 6 * R->M; ++i)
            nvv[i] = nvv[i] + R->eq2[s][i] * 1.0;
}

/* PartSpecies::impl_update_pos (PartSpecies.cc:147-159): returns 1 if nothing moved too far */
static int update_pos(orc_run *R, Bucket *b, double dt, double fraction)
{
    double const scale = 1.0 / fraction;
    int          ok    = 1;
    for (int64_t k = 0; k < b->n; ++k) {
        V3 const v     = { b->vx[k], b->vy[k], b->vz[k] };
        double   moved = g_cart_to_contr(R, v, b->q1[k]).x * dt;
        b->q1[k] += moved;
        moved *= scale;
        ok &= 0 == (long)moved;
    }
    return ok;
}
static void add_equilibrium(orc_run const *R, int s, double *n, double *nV, double *nvv);
/* PartSpecies::impl_collect_part<O> (PartSpecies.cc:210-224), then the delta-f equilibrium */
static void collect_part(orc_run *R, Bucket const *b, h1d_kinetic_desc const *d, double *n, double *nV)
{
    double const q1min = R->half_min;
    int const    O     = (int)d->shape_order;
    memset(n, 0, sizeof(double) * R->M);
    memset(nV, 0, sizeof(double) * 3 * R->M);
    for (int64_t k = 0; k < b->n; ++k) {
        Shp sx;
        shape(&sx, O, b->q1[k] - q1min);
        double const w  = b->w[k];
        V3 const     vw = { b->vx[k] * w, b->vy[k] * w, b->vz[k] * w };
        for (int j = 0; j <= O; ++j)
            *at1(n, sx.i[j]) += w * sx.w[j];
        for (int j = 0; j <= O; ++j) {
            double *a = at3(nV, sx.i[j]);
            a[0] += vw.x * sx.w[j];
            a[1] += vw.y * sx.w[j];
            a[2] += vw.z * sx.w[j];
        }
    }
    double const s = 1.0 / d->moment_norm;
    for (long i = 0; i < R->M; ++i)
        n[i] *= s;
    for (long i = 0; i < 3 * R->M; ++i)
        nV[i] *= s;
    add_equilibrium(R, (int)(d - R->p.kinetic), n, nV, NULL);
}
/* PartSpecies::impl_collect_all (PartSpecies.cc:225-244): always CIC */
static void collect_all(orc_run *R, Bucket const *b, h1d_kinetic_desc const *d, double *n, double *nV, double *nvv)
{
    double const q1min = R->half_min;
    memset(n, 0, sizeof(double) * R->M);
    memset(nV, 0, sizeof(double) * 3 * R->M);
    memset(nvv, 0, sizeof(double) * 6 * R->M);
    for (int64_t k = 0; k < b->n; ++k) {
        Shp sx;
        shape1(&sx, b->q1[k] - q1min);
        double const w  = b->w[k];
        double const vx = b->vx[k], vy = b->vy[k], vz = b->vz[k];
        V3 const     vw = { vx * w, vy * w, vz * w };
        for (int j = 0; j <= 1; ++j)
            *at1(n, sx.i[j]) += w * sx.w[j];
        for (int j = 0; j <= 1; ++j) {
            double *a = at3(nV, sx.i[j]);
            a[0] += vw.x * sx.w[j], a[1] += vw.y * sx.w[j], a[2] += vw.z * sx.w[j];
        }
        double t[6] = { vx * vx, vy * vy, vz * vz, vx * vy, vy * vz, vz * vx };
        for (int c = 0; c < 6; ++c)
            t[c] *= w;
        for (int j = 0; j <= 1; ++j) {
            double *a = at6(nvv, sx.i[j]);
            for (int c = 0; c < 6; ++c)
                a[c] += t[c] * sx.w[j];
        }
    }
    double const s = 1.0 / d->moment_norm;
    for (long i = 0; i < R->M; ++i)
        n[i] *= s;
    for (long i = 0; i < 3 * R->M; ++i)
        nV[i] *= s;
    for (long i = 0; i < 6 * R->M; ++i)
        nvv[i] *= s;
    add_equilibrium(R, (int)(d - R->p.kinetic), n, nV, nvv);
}

/* counter-based gyro-phase draw in [-pi, pi) replacing the std::random_device-seeded
 * generator of Delegate::randomize_gyrophase (Delegate.cc:146-156) */
static inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
double orc_gyrophase(uint64_t seed, uint64_t counter, uint64_t species, uint64_t pid)
{
    uint64_t h = mix64(seed + 0x9e3779b97f4a7c15ULL);
    h          = mix64(h ^ (counter * 0xd1b54a32d192ed03ULL));
    h          = mix64(h ^ (species * 0x8cb92ba72f3d8dd7ULL) ^ pid);
    double const u = (double)(h >> 11) * (1.0 / 9007199254740992.0);
    return -M_PI + u * (2 * M_PI);
}

/* Delegate::boundary_pass(Domain, PartSpecies) with partition + periodic/reflecting pass
 * (Delegate.cc:51-74, 101-145) and SubdomainDelegate's self-exchange (SubdomainDelegate.cc:183-251) */
static int64_t partition(Bucket *b, int64_t first, int64_t last, int (*pred)(double, double), double ref)
{ /* libstdc++ __partition for bidirectional iterators (two-pointer) */
    for (;;) {
        for (;;) {
            if (first == last)
                return first;
            else if (pred(b->q1[first], ref))
                ++first;
            else
                break;
        }
        --last;
        for (;;) {
            if (first == last)
                return first;
            else if (!pred(b->q1[last], ref))
                --last;
            else
                break;
        }
        bucket_swap_elems(b, first, last);
        ++first;
    }
}
static int pred_ge(double q1, double LB) { return q1 >= LB; }
static int pred_lt(double q1, double RB) { return q1 < RB; }

static void particle_bc(orc_run *R, Bucket *b, int species, uint64_t counter)
{
    double const LB = R->full_min, RB = R->full_min + R->full_len, len = R->full_len;
    Bucket *L = &R->bufL, *Rb = &R->bufR;
    L->n = Rb->n = 0;
    int64_t it = partition(b, 0, b->n, pred_ge, LB);
    for (int64_t k = it; k < b->n; ++k)
        bucket_push(L, b, k);
    b->n = it;
    it   = partition(b, 0, b->n, pred_lt, RB);
    for (int64_t k = it; k < b->n; ++k)
        bucket_push(Rb, b, k);
    b->n = it;

    int const bc = R->p.particle_bc;
    if (bc == H1D_BC_PERIODIC) {
        for (int64_t k = 0; k < L->n; ++k)
            if (!(L->q1[k] >= LB && L->q1[k] < RB))
                L->q1[k] += len;
        for (int64_t k = 0; k < Rb->n; ++k)
            if (!(Rb->q1[k] >= LB && Rb->q1[k] < RB))
                Rb->q1[k] -= len;
    } else if (bc == H1D_BC_REFLECTING) {
        for (int pass = 0; pass < 2; ++pass) {
            Bucket      *B   = pass == 0 ? L : Rb;
            double const ext = pass == 0 ? LB : RB;
            for (int64_t k = 0; k < B->n; ++k) {
                if (B->q1[k] >= LB && B->q1[k] < RB)
                    continue;
                B->q1[k] += 2 * (ext - B->q1[k]);
                double const d = B->vx[k] * 1 + B->vy[k] * 0 + B->vz[k] * 0;
                double const s = 2 * d;
                B->vx[k]       = B->vx[k] - s * 1;
                B->vy[k]       = B->vy[k] - s * 0;
                B->vz[k]       = B->vz[k] - s * 0;
                if (R->p.randomize_gyrophase) {
                    double const ph = orc_gyrophase(R->p.gyrophase_seed, counter, (uint64_t)species, (uint64_t)B->pid[k]);
                    double const c = cos(ph), s2 = sin(ph);
                    double const vy = B->vy[k], vz = B->vz[k];
                    B->vy[k] = vy * c - vz * s2;
                    B->vz[k] = vy * s2 + vz * c;
                }
            }
        }
    } else { /* absorbing: crossing particles leave the system */
        L->n = Rb->n = 0;
    }
    /* swap_bucket, then append L then R (Delegate.cc:61, 72-73) */
    for (int64_t k = 0; k < Rb->n; ++k)
        bucket_push(b, Rb, k);
    for (int64_t k = 0; k < L->n; ++k)
        bucket_push(b, L, k);
}

/* ------------------------------------------------------------------------------------------------
 * collect_smooth (Domain.hh:35-74) with the charge/current conversion factors
 */
static void add_scaled(double *dst, double const *src, long count, double f)
{
    for (long i = 0; i < count; ++i)
        dst[i] += src[i] * f;
}
static void addto(double *dst, double const *src, long count)
{
    for (long i = 0; i < count; ++i)
        dst[i] += src[i];
}
static double const *collect_smooth_rho_f(orc_run *R, double const *mom0, double factor, long n_smooth)
{
    memset(R->rho, 0, sizeof(double) * R->M);
    add_scaled(R->rho, mom0, R->M, factor);
    gather_grid(R, R->rho, 1);
    for (long i = 0; i < n_smooth; ++i) {
        pass_grid(R, R->rho, 1);
        smooth_grid(R, R->rho, 1);
    }
    pass_grid(R, R->rho, 1);
    return R->rho;
}
static double const *collect_smooth_J_f(orc_run *R, double const *mom1, double factor, long n_smooth)
{
    memset(R->J, 0, sizeof(double) * 3 * R->M);
    add_scaled(R->J, mom1, 3 * R->M, factor);
    gather_grid(R, R->J, 3);
    for (long i = 0; i < n_smooth; ++i) {
        pass_grid(R, R->J, 3);
        smooth_grid(R, R->J, 3);
    }
    pass_grid(R, R->J, 3);
    return R->J;
}
/* Domain::collect_smooth (Domain.hh:35-74) with the species' conversion factors (Species.h:42-49) */
static double const *collect_smooth_rho(orc_run *R, double const *mom0, double Oc, double op, long n_smooth)
{
    return collect_smooth_rho_f(R, mom0, cdcf(R, Oc, op), n_smooth);
}
static double const *collect_smooth_J(orc_run *R, double const *mom1, double Oc, double op, long n_smooth)
{
    return collect_smooth_J_f(R, mom1, ccf(R, Oc, op), n_smooth);
}

/* ------------------------------------------------------------------------------------------------
 * EField::update (EField.cc:41-126)
 */
static void efield_update(orc_run *R, double *E, double const *B, double const *rho, double const *Ji)
{
    long const            N  = R->Nx;
    h1d_efluid_desc const ef = R->p.efluid;
    double const          O0 = R->p.O0;
    /* impl_update_dPe */
    double const O02beO2   = (O0 * O0) * ef.beta * 0.5;
    double const mOeOO0oe2 = -ef.Oc / (O0 * (ef.op * ef.op));
    for (long i = -P; i < N + P; ++i)
        R->Pe[i + P] = pow(mOeOO0oe2 * rho[i + P], ef.gamma) * O02beO2;
    double const cO2 = R->p.c / 2;
    for (long i = 0; i < N; ++i) {
        double *d = at3(R->dPe, i);
        d[0]      = (R->Pe[i + 1 + P] - R->Pe[i - 1 + P]) * cO2;
        d[1] = d[2] = 0;
    }
    mask_grid(R, R->dPe, 3, R->p.phase_retardation_inset, R->p.phase_retardation_factor);
    /* impl_update_Je with B_covar */
    for (long i = -1; i < N + 1; ++i) {
        V3 const b = { B[3 * (i + P)], B[3 * (i + P) + 1], B[3 * (i + P) + 2] };
        V3 const c = g_cart_to_covar(R, b, (double)i + R->full_min);
        double  *o = at3(R->covar, i);
        o[0] = c.x, o[1] = c.y, o[2] = c.z;
    }
    double const cOsqrtg = R->p.c / R->sqrt_g;
    for (long i = 0; i < N; ++i) {
        double const *B1 = at3(R->covar, i + 1), *B0 = at3(R->covar, i);
        V3 const      curl = { 0, (-B1[2] + B0[2]) * cOsqrtg, (+B1[1] - B0[1]) * cOsqrtg };
        V3 const      j    = { Ji[3 * (i + P)], Ji[3 * (i + P) + 1], Ji[3 * (i + P) + 2] };
        V3 const      jc   = g_cart_to_contr(R, j, (double)i + R->half_min);
        double       *o    = at3(R->Je, i);
        o[0] = curl.x - jc.x, o[1] = curl.y - jc.y, o[2] = curl.z - jc.z;
    }
    mask_grid(R, R->Je, 3, R->p.phase_retardation_inset, R->p.phase_retardation_factor);
    /* impl_update_E with dB_contr */
    for (long i = -1; i < N + 1; ++i) {
        V3 const b = { B[3 * (i + P)], B[3 * (i + P) + 1], B[3 * (i + P) + 2] };
        V3 const c = g_cart_to_contr(R, b, (double)i + R->full_min);
        double  *o = at3(R->contr, i);
        o[0] = c.x, o[1] = c.y, o[2] = c.z;
    }
    V3 const Bc0 = g_Bcontr(R);
    for (long i = 0; i < N; ++i) {
        double const  pos = (double)i + R->half_min;
        double const *d1 = at3(R->contr, i + 1), *d0 = at3(R->contr, i);
        V3 const      Bc = { Bc0.x + (d1[0] + d0[0]) * 0.5, Bc0.y + (d1[1] + d0[1]) * 0.5,
                             Bc0.z + (d1[2] + d0[2]) * 0.5 };
        double const *je = at3(R->Je, i);
        V3 const      J  = { je[0], je[1], je[2] };
        V3            lz = cross3(J, Bc);
        lz.x *= R->sqrt_g, lz.y *= R->sqrt_g, lz.z *= R->sqrt_g;
        double const *g  = at3(R->dPe, i);
        double const  r  = rho[i + P];
        V3 const      Ec = { (lz.x - g[0]) / r, (lz.y - g[1]) / r, (lz.z - g[2]) / r };
        V3 const      Ee = g_covar_to_cart(R, Ec, pos);
        double       *o  = at3(E, i);
        o[0] = Ee.x, o[1] = Ee.y, o[2] = Ee.z;
    }
    mask_grid(R, E, 3, R->p.amplitude_damping_inset, R->p.amplitude_damping_factor);
}

/* BField::update (BField.cc:24-74) */
static void bfield_update(orc_run *R, double *B, double const *E, double dt)
{
    long const   N         = R->Nx;
    double const cdtOsqrtg = dt * R->p.c / R->sqrt_g;
    memcpy(R->Bprev, B, sizeof(double) * 3 * R->M);
    memset(B, 0, sizeof(double) * 3 * R->M);
    for (long i = -1; i < N + 1; ++i) {
        V3 const e = { E[3 * (i + P)], E[3 * (i + P) + 1], E[3 * (i + P) + 2] };
        V3 const c = g_cart_to_covar(R, e, (double)i + R->half_min);
        double  *o = at3(R->Ecovar, i);
        o[0] = c.x, o[1] = c.y, o[2] = c.z;
    }
    for (long i = 0; i < N; ++i) {
        double const *E1 = at3(R->Ecovar, i), *E0 = at3(R->Ecovar, i - 1);
        V3 const      Bc = { 0, (-E1[2] + E0[2]) * cdtOsqrtg, (+E1[1] - E0[1]) * cdtOsqrtg };
        V3 const      Bk = g_contr_to_cart(R, Bc, (double)i + R->full_min);
        double       *o  = at3(B, i);
        o[0] -= Bk.x, o[1] -= Bk.y, o[2] -= Bk.z;
    }
    mask_grid(R, B, 3, R->p.phase_retardation_inset, R->p.phase_retardation_factor);
    for (long i = 0; i < N; ++i)
        for (int c = 0; c < 3; ++c)
            B[3 * (i + P) + c] = B[3 * (i + P) + c] + R->Bprev[3 * (i + P) + c];
    mask_grid(R, B, 3, R->p.amplitude_damping_inset, R->p.amplitude_damping_factor);
}

/* Current::impl_advance (Current.cc:45-52) on a zeroed J */
static void current_advance_impl(orc_run *R, double *J, double const *L, double const *G, double const *B, double const *E, double dt)
{
    long const N = R->Nx;
    for (long i = 0; i < N; ++i) {
        double const  pos = (double)i + R->half_min;
        V3 const      b0  = g_Bcart(R, pos);
        double const *d1 = at3((double *)B, i + 1), *d0 = at3((double *)B, i);
        V3 const      Bi = { b0.x + (d1[0] + d0[0]) * 0.5, b0.y + (d1[1] + d0[1]) * 0.5, b0.z + (d1[2] + d0[2]) * 0.5 };
        double const *e  = at3((double *)E, i);
        double const  l  = L[i + P];
        double const *g  = at3((double *)G, i);
        V3 const      Gv = { g[0], g[1], g[2] };
        V3 const      gx = cross3(Gv, Bi);
        double       *o  = at3(J, i);
        o[0] += (e[0] * l + gx.x) * dt;
        o[1] += (e[1] * l + gx.y) * dt;
        o[2] += (e[2] * l + gx.z) * dt;
    }
}
/* Domain_CAMCL::current_advance (Domain_CAMCL.cc:131-151); Lambda / Gamma take the charge / current
 * conversion factors times Oc/O0 (Charge.cc:31-36, Current.cc:34-39) */
static double const *current_advance_f(orc_run *R, double const *mom0, double const *mom1, double lam_f, double gam_f,
                                       long n_smooth, double dt_2)
{
    long const M = R->M;
    memset(R->lambda, 0, sizeof(double) * M);
    add_scaled(R->lambda, mom0, M, lam_f);
    gather_grid(R, R->lambda, 1);
    memset(R->gamma, 0, sizeof(double) * 3 * M);
    add_scaled(R->gamma, mom1, 3 * M, gam_f);
    gather_grid(R, R->gamma, 3);
    memset(R->J, 0, sizeof(double) * 3 * M);
    current_advance_impl(R, R->J, R->lambda, R->gamma, R->B, R->E, dt_2);
    for (long i = 0; i < n_smooth; ++i) {
        pass_grid(R, R->J, 3);
        smooth_grid(R, R->J, 3);
    }
    pass_grid(R, R->J, 3);
    return R->J;
}
static double const *current_advance(orc_run *R, double const *mom0, double const *mom1, double Oc, double op, long n_smooth, double dt_2)
{
    return current_advance_f(R, mom0, mom1, cdcf(R, Oc, op) * Oc / R->p.O0, ccf(R, Oc, op) * Oc / R->p.O0, n_smooth, dt_2);
}

/* ------------------------------------------------------------------------------------------------
 * ExternalSource (Core/ExternalSource.cc:12-66, ExternalSource.hh:16-33): a species whose Oc is O0
 * and op is 0, with charge / current conversion factors 0 / 1 (ExternalSource.h:36-38), so it adds
 * its moment<1> to the current, J x B dt/2 to the advanced current, and nothing to the charge.
 */
static double src_envelope(h1d_source_desc const *d, double t)
{
    double const eps      = 1e-15;
    double const slope_in = M_PI / (d->ease_in > eps ? d->ease_in : 1.0);
    double const slope_out = M_PI / (d->ease_out > eps ? d->ease_out : 1.0);
    t -= d->start;
    if (t < -d->ease_in) /* before ease-in */
        return 0;
    if (t < 0) /* ease-in */
        return .5 * (1 + cos(slope_in * t));
    if (t < d->duration) /* middle */
        return 1;
    if ((t -= d->duration) < d->ease_out) /* ease-out */
        return .5 * (1 + cos(slope_out * t));
    return 0;
}
/* ExternalSource::collect: moment<1> = sum over source points inside the half-grid extent of the
 * Cartesian current (field-aligned = Cartesian on the field line) times envelope x weighting,
 * deposited with Shape<1> */
static void src_collect(orc_run *R, int e, double t)
{
    h1d_source_desc const *d = &R->p.sources[e];
    memset(R->smom0[e], 0, sizeof(double) * R->M);
    memset(R->smom1[e], 0, sizeof(double) * 3 * R->M);
    double const lo = R->half_min, hi = R->half_min + R->full_len;
    for (int64_t i = 0; i < d->n_points; ++i) {
        double const pos = d->pos[i];
        if (!(pos >= lo && pos < hi))
            continue;
        Shp sx;
        shape1(&sx, pos - lo);
        double const phase = -d->omega * (t - d->start);
        double const c = cos(phase), sn = sin(phase);
        double const f  = src_envelope(d, t) * R->p.moment_weighting;
        double const J[3] = { d->J0re[i][0] * c - d->J0im[i][0] * sn, d->J0re[i][1] * c - d->J0im[i][1] * sn,
                              d->J0re[i][2] * c - d->J0im[i][2] * sn };
        double const v[3] = { J[0] * f, J[1] * f, J[2] * f };
        for (int j = 0; j <= 1; ++j) {
            double *a = at3(R->smom1[e], sx.i[j]);
            a[0] += v[0] * sx.w[j];
            a[1] += v[1] * sx.w[j];
            a[2] += v[2] * sx.w[j];
        }
    }
}
/* the source's contribution to a charge / current pair (collect_smooth with factors 0 and 1) */
static void src_add(orc_run *R, int e, double *charge, double *current)
{
    long const n_smooth = R->p.sources[e].n_smooth;
    addto(current, collect_smooth_J_f(R, R->smom1[e], 1.0, n_smooth), 3 * R->M);
    addto(charge, collect_smooth_rho_f(R, R->smom0[e], 0.0, n_smooth), R->M);
}

/* ColdSpecies::impl_update_nV (ColdSpecies.cc:35-42) */
static void cold_update_vel(orc_run *R, int ci, double const *E, double dt)
{
    h1d_cold_desc const *d     = &R->p.cold[ci];
    Boris const          boris = boris_make(dt, R->p.c, R->p.O0, d->Oc);
    double              *nV = R->cnV_full[ci], *n = R->cn_full[ci];
    for (long i = 0; i < R->Nx; ++i) {
        double const pos = (double)i + R->half_min;
        double const ni  = n[i + P];
        double const *e  = at3((double *)E, i);
        V3 const      En = { e[0] * ni, e[1] * ni, e[2] * ni };
        double       *v  = at3(nV, i);
        V3            vv = { v[0], v[1], v[2] };
        boris_push(&boris, &vv, g_Bcart(R, pos), En);
        v[0] = vv.x, v[1] = vv.y, v[2] = vv.z;
    }
}
/* ColdSpecies::impl_collect_part (ColdSpecies.cc:53-65) */
static void cold_collect_part(orc_run *R, double const *n_full, double const *nV_full, double *n, double *nV)
{
    double const w = R->p.moment_weighting;
    memset(n, 0, sizeof(double) * R->M);
    memset(nV, 0, sizeof(double) * 3 * R->M);
    for (long i = 0; i < R->Nx; ++i) {
        n[i + P] = n_full[i + P] * w;
        for (int c = 0; c < 3; ++c)
            nV[3 * (i + P) + c] = nV_full[3 * (i + P) + c] * w;
    }
}

/* ------------------------------------------------------------------------------------------------
 * Domain_CAMCL::cycle (Domain_CAMCL.cc:57-130) and subcycle (:152-193)
 */
static int camcl_cycle(orc_run *R)
{
    long const   M  = R->M;
    double const dt = R->p.dt;
    int          ok = 1;
    memset(R->current, 0, sizeof(double) * 3 * M);
    memset(R->current1, 0, sizeof(double) * 3 * M);
    memset(R->charge, 0, sizeof(double) * M);
    memset(R->charge1, 0, sizeof(double) * M);
    for (int s = 0; s < R->p.n_kinetic; ++s) {
        h1d_kinetic_desc const *d = &R->p.kinetic[s];
        half_grid(R, R->mom1[s], R->B);
        update_velocity(R, &R->part[s], d, R->mom1[s], R->E, dt);
        collect_part(R, &R->part[s], d, R->mom0[s], R->mom1[s]);
        addto(R->current, collect_smooth_J(R, R->mom1[s], d->Oc, d->op, d->n_smooth), 3 * M);
        addto(R->charge, collect_smooth_rho(R, R->mom0[s], d->Oc, d->op, d->n_smooth), M);
        ok &= update_pos(R, &R->part[s], dt, 1);
        particle_bc(R, &R->part[s], s, (uint64_t)R->step * 8);
        collect_part(R, &R->part[s], d, R->mom0[s], R->mom1[s]);
        addto(R->current1, collect_smooth_J(R, R->mom1[s], d->Oc, d->op, d->n_smooth), 3 * M);
        addto(R->charge1, collect_smooth_rho(R, R->mom0[s], d->Oc, d->op, d->n_smooth), M);
    }
    for (int ci = 0; ci < R->p.n_cold; ++ci) {
        h1d_cold_desc const *d = &R->p.cold[ci];
        cold_update_vel(R, ci, R->E, dt);
        cold_collect_part(R, R->cn_full[ci], R->cnV_full[ci], R->cmom0[ci], R->cmom1[ci]);
        addto(R->current, collect_smooth_J(R, R->cmom1[ci], d->Oc, d->op, d->n_smooth), 3 * M);
        addto(R->charge, collect_smooth_rho(R, R->cmom0[ci], d->Oc, d->op, d->n_smooth), M);
        addto(R->current1, collect_smooth_J(R, R->cmom1[ci], d->Oc, d->op, d->n_smooth), 3 * M);
        addto(R->charge1, collect_smooth_rho(R, R->cmom0[ci], d->Oc, d->op, d->n_smooth), M);
    }
    for (int e = 0; e < R->p.n_sources; ++e) { /* update(0.5 dt): at the half-time step */
        src_collect(R, e, (double)R->step * dt + 0.5 * dt);
        src_add(R, e, R->charge, R->current);
        src_add(R, e, R->charge1, R->current1);
    }
    /* average */
    for (long i = 0; i < M; ++i)
        R->charge[i] = (R->charge[i] + R->charge1[i]) * .5;
    for (long i = 0; i < 3 * M; ++i)
        R->current[i] = (R->current[i] + R->current1[i]) * .5;
    /* subcycle */
    {
        long const   m      = R->p.n_subcycles;
        double const sdt    = dt / m;
        double const dt_x_2 = sdt * 2.0;
        double      *b0 = R->B, *b1 = R->B1;
        memcpy(b1, b0, sizeof(double) * 3 * M);
        efield_update(R, R->E, b0, R->charge, R->current);
        pass_grid(R, R->E, 3);
        bfield_update(R, b1, R->E, sdt);
        pass_grid(R, b1, 3);
        for (long i = 1; i < m; ++i) {
            efield_update(R, R->E, b1, R->charge, R->current);
            pass_grid(R, R->E, 3);
            bfield_update(R, b0, R->E, dt_x_2);
            pass_grid(R, b0, 3);
            double *t = b0;
            b0 = b1, b1 = t;
        }
        efield_update(R, R->E, b1, R->charge, R->current);
        pass_grid(R, R->E, 3);
        bfield_update(R, b0, R->E, sdt);
        pass_grid(R, b0, 3);
        for (long i = 0; i < 3 * M; ++i)
            b0[i] = (b0[i] + b1[i]) * .5;
        R->B = b0, R->B1 = b1;
    }
    efield_update(R, R->E, R->B, R->charge1, R->current);
    pass_grid(R, R->E, 3);
    for (int s = 0; s < R->p.n_kinetic; ++s) {
        h1d_kinetic_desc const *d = &R->p.kinetic[s];
        addto(R->current1, current_advance(R, R->mom0[s], R->mom1[s], d->Oc, d->op, d->n_smooth, 0.5 * dt), 3 * M);
    }
    for (int ci = 0; ci < R->p.n_cold; ++ci) {
        h1d_cold_desc const *d = &R->p.cold[ci];
        addto(R->current1, current_advance(R, R->cmom0[ci], R->cmom1[ci], d->Oc, d->op, d->n_smooth, 0.5 * dt), 3 * M);
    }
    for (int e = 0; e < R->p.n_sources; ++e) /* Oc = O0: Lambda factor 0 * O0/O0, Gamma factor 1 * O0/O0 */
        addto(R->current1, current_advance_f(R, R->smom0[e], R->smom1[e], 0.0 * R->p.O0 / R->p.O0, 1.0 * R->p.O0 / R->p.O0,
                                             R->p.sources[e].n_smooth, 0.5 * dt), 3 * M);
    efield_update(R, R->E, R->B, R->charge1, R->current1);
    pass_grid(R, R->E, 3);
    return ok;
}

/* ------------------------------------------------------------------------------------------------
 * Domain_PC (Domain_PC.cc:84-205)
 */
static void pc_average(orc_run *R, double *a, double const *b)
{
    for (long i = 0; i < 3 * R->M; ++i)
        a[i] = (a[i] + b[i]) * .5;
}
static int pc_particles(orc_run *R, Bucket *b, int s, double *mom0, double *mom1, double const *B1, double const *E1, uint64_t counter)
{
    h1d_kinetic_desc const *d  = &R->p.kinetic[s];
    double const            dt = R->p.dt;
    int                     ok = 1;
    if (!update_pos(R, b, 0.5 * dt, 0.5))
        ok = 0;
    particle_bc(R, b, s, counter);
    half_grid(R, mom1, B1);
    update_velocity(R, b, d, mom1, (double *)E1, dt);
    if (!update_pos(R, b, 0.5 * dt, 0.5))
        ok = 0;
    particle_bc(R, b, s, counter + 1);
    collect_part(R, b, d, mom0, mom1);
    addto(R->charge, collect_smooth_rho(R, mom0, d->Oc, d->op, d->n_smooth), R->M);
    addto(R->current, collect_smooth_J(R, mom1, d->Oc, d->op, d->n_smooth), 3 * R->M);
    return ok;
}
static int pc_cycle(orc_run *R)
{
    long const   M  = R->M;
    double const dt = R->p.dt;
    int          ok = 1;
    /* predictor */
    memcpy(R->B1, R->B, sizeof(double) * 3 * M);
    bfield_update(R, R->B1, R->E, dt);
    pass_grid(R, R->B1, 3);
    efield_update(R, R->E1, R->B1, R->charge, R->current);
    pass_grid(R, R->E1, 3);
    pc_average(R, R->B1, R->B);
    pc_average(R, R->E1, R->E);
    memset(R->charge, 0, sizeof(double) * M);
    memset(R->current, 0, sizeof(double) * 3 * M);
    for (int s = 0; s < R->p.n_kinetic; ++s) {
        bucket_copy(&R->pred, &R->part[s]);
        ok &= pc_particles(R, &R->pred, s, R->pmom0, R->pmom1, R->B1, R->E1, (uint64_t)R->step * 8 + 0);
    }
    for (int ci = 0; ci < R->p.n_cold; ++ci) {
        h1d_cold_desc const *d = &R->p.cold[ci];
        memcpy(R->pc_n_full, R->cn_full[ci], sizeof(double) * M);
        memcpy(R->pc_nV_full, R->cnV_full[ci], sizeof(double) * 3 * M);
        double *sn = R->cn_full[ci], *snV = R->cnV_full[ci];
        R->cn_full[ci] = R->pc_n_full, R->cnV_full[ci] = R->pc_nV_full;
        cold_update_vel(R, ci, R->E1, dt);
        cold_collect_part(R, R->cn_full[ci], R->cnV_full[ci], R->pmom0, R->pmom1);
        R->cn_full[ci] = sn, R->cnV_full[ci] = snV;
        addto(R->charge, collect_smooth_rho(R, R->pmom0, d->Oc, d->op, d->n_smooth), M);
        addto(R->current, collect_smooth_J(R, R->pmom1, d->Oc, d->op, d->n_smooth), 3 * M);
    }
    for (int e = 0; e < R->p.n_sources; ++e) { /* a predictor copy's update(dt): at the full-time step */
        src_collect(R, e, (double)R->step * dt + dt);
        src_add(R, e, R->charge, R->current);
    }
    /* corrector */
    memcpy(R->B1, R->B, sizeof(double) * 3 * M);
    bfield_update(R, R->B1, R->E1, dt);
    pass_grid(R, R->B1, 3);
    efield_update(R, R->E1, R->B1, R->charge, R->current);
    pass_grid(R, R->E1, 3);
    pc_average(R, R->B1, R->B);
    pc_average(R, R->E1, R->E);
    memset(R->charge, 0, sizeof(double) * M);
    memset(R->current, 0, sizeof(double) * 3 * M);
    for (int s = 0; s < R->p.n_kinetic; ++s)
        ok &= pc_particles(R, &R->part[s], s, R->mom0[s], R->mom1[s], R->B1, R->E1, (uint64_t)R->step * 8 + 2);
    for (int ci = 0; ci < R->p.n_cold; ++ci) {
        h1d_cold_desc const *d = &R->p.cold[ci];
        cold_update_vel(R, ci, R->E1, dt);
        cold_collect_part(R, R->cn_full[ci], R->cnV_full[ci], R->cmom0[ci], R->cmom1[ci]);
        addto(R->charge, collect_smooth_rho(R, R->cmom0[ci], d->Oc, d->op, d->n_smooth), M);
        addto(R->current, collect_smooth_J(R, R->cmom1[ci], d->Oc, d->op, d->n_smooth), 3 * M);
    }
    for (int e = 0; e < R->p.n_sources; ++e) { /* update(dt) of the source itself */
        src_collect(R, e, (double)R->step * dt + dt);
        src_add(R, e, R->charge, R->current);
    }
    bfield_update(R, R->B, R->E1, dt);
    pass_grid(R, R->B, 3);
    efield_update(R, R->E, R->B, R->charge, R->current);
    pass_grid(R, R->E, 3);
    return ok;
}

/* ------------------------------------------------------------------------------------------------
 * public entry points (same shape as the CUDA library's C-ABI)
 */
static int check_params(h1d_params const *p, char *msg, size_t cap)
{
#define BAD(...) return snprintf(msg, cap, __VA_ARGS__), H1D_ERR_INVALID_ARG
    if (!p)
        BAD("null params");
    if (p->Nx < 2 * P)
        BAD("Nx must be at least %d", 2 * P);
    if (!(p->Dx > 0) || !(p->c > 0) || !(p->O0 > 0) || !(p->dt > 0) || p->xi < 0)
        BAD("Dx, c, O0, dt must be positive and xi non-negative");
    if (p->n_subcycles < 2)
        BAD("n_subcycles should be at least 2");
    if (p->algorithm != H1D_ALGO_PC && p->algorithm != H1D_ALGO_CAMCL)
        BAD("unknown algorithm");
    if (p->particle_bc < 0 || p->particle_bc > 2)
        BAD("unknown particle boundary condition");
    if (p->n_kinetic < 0 || p->n_kinetic > H1D_MAX_KINETIC || p->n_cold < 0 || p->n_cold > H1D_MAX_COLD)
        BAD("too many species");
    if (p->phase_retardation_inset < 0 || p->phase_retardation_inset > p->Nx / 2 || p->amplitude_damping_inset < 0
        || p->amplitude_damping_inset > p->Nx / 2)
        BAD("masking inset is greater than half the domain length");
    if (p->phase_retardation_factor < 0 || p->phase_retardation_factor > 1 || p->amplitude_damping_factor < 0
        || p->amplitude_damping_factor > 1)
        BAD("masking factor outside [0, 1]");
    if (!(p->efluid.Oc < 0) || !(p->efluid.op > 0) || p->efluid.beta < 0)
        BAD("invalid electron fluid descriptor");
    for (int s = 0; s < p->n_kinetic; ++s) {
        h1d_kinetic_desc const *d = &p->kinetic[s];
        if (d->Oc == 0 || !(d->op > 0))
            BAD("kinetic species %d: Oc should not be zero and op should be positive", s);
        if (d->shape_order < 1 || d->shape_order > 3)
            BAD("kinetic species %d: shape order must be 1, 2 or 3", s);
        if (!(d->moment_norm > 0))
            BAD("kinetic species %d: moment_norm must be positive", s);
        if (d->n_smooth < 0)
            BAD("kinetic species %d: negative smoothing count", s);
        if ((d->scheme != H1D_FULL_F && d->scheme != H1D_DELTA_F) || !(d->psd_refresh_frequency >= 0))
            BAD("kinetic species %d: unknown particle scheme or negative psd_refresh_frequency", s);
        if (d->vdf < H1D_VDF_BIMAXWELLIAN || d->vdf > H1D_VDF_COUNTER_BEAM)
            BAD("kinetic species %d: unknown equilibrium distribution", s);
        if ((d->scheme == H1D_DELTA_F || d->psd_refresh_frequency != 0)
            && (!(d->vth1 > 0) || ((d->vdf == H1D_VDF_BIMAXWELLIAN || d->vdf == H1D_VDF_LOSSCONE) && !(d->T2_T1 > 0))
                || (d->vdf == H1D_VDF_COUNTER_BEAM && !(d->vdf_param[0] > 0))))
            BAD("kinetic species %d: evolving weights need the equilibrium vth1 > 0 (and T2_T1 > 0, nu > 0)", s);
    }
    for (int s = 0; s < p->n_cold; ++s)
        if (p->cold[s].Oc == 0 || !(p->cold[s].op > 0) || p->cold[s].n_smooth < 0)
            BAD("cold species %d: invalid descriptor", s);
    if (p->n_sources < 0 || p->n_sources > H1D_MAX_SOURCES)
        BAD("too many external sources");
    for (int e = 0; e < p->n_sources; ++e) { /* ExternalSourceBase (PlasmaDesc.h:383-403) */
        h1d_source_desc const *d = &p->sources[e];
        if (!(d->ease_in >= 0) || !(d->ease_out >= 0))
            BAD("external source %d: ease-in/-out should be non-negative", e);
        if (d->n_points < 0 || d->n_points > H1D_MAX_SOURCE_POINTS || d->n_smooth < 0)
            BAD("external source %d: invalid descriptor", e);
    }
    if (p->xi > 0) { /* ParamSet.cc:25-29 */
        double const lim = M_PI_2, xd = p->xi * p->Dx;
        double const e[4] = { -0.5 * p->Nx, -0.5 * p->Nx + p->Nx, -0.5 * p->Nx + 0.5, -0.5 * p->Nx + 0.5 + p->Nx };
        for (int k = 0; k < 4; ++k)
            if (!(fabs(xd * e[k]) < lim))
                BAD("invalid domain extent: |xi*D1*q1| >= pi/2");
    }
    return H1D_OK;
#undef BAD
}

int orc_create(h1d_params const *p, orc_run **out)
{
    char msg[512] = { 0 };
    int  st       = check_params(p, msg, sizeof msg);
    if (st) {
        fprintf(stderr, "oracle: %s\n", msg);
        return st;
    }
    orc_run *R = xcalloc(1, sizeof(orc_run));
    R->p       = *p;
    if (!(R->p.moment_weighting > 0))
        R->p.moment_weighting = 1;
    R->Nx       = p->Nx;
    R->M        = p->Nx + 2 * P;
    R->full_min = -0.5 * (double)p->Nx;
    R->full_len = (double)p->Nx;
    R->half_min = R->full_min + 0.5;
    R->xi = p->xi, R->xi2 = p->xi * p->xi, R->D1 = p->Dx, R->D2 = 1, R->D3 = 1;
    R->inv_D1 = 1 / R->D1, R->inv_D2 = 1 / R->D2, R->inv_D3 = 1 / R->D3;
    R->sqrt_g      = R->D1 * R->D2 * R->D3;
    R->homogeneous = p->xi < 1e-10;
    long const M   = R->M;
    R->B = xcalloc(3 * M, 8), R->B1 = xcalloc(3 * M, 8), R->E = xcalloc(3 * M, 8), R->E1 = xcalloc(3 * M, 8);
    R->charge = xcalloc(M, 8), R->charge1 = xcalloc(M, 8), R->rho = xcalloc(M, 8), R->lambda = xcalloc(M, 8);
    R->current = xcalloc(3 * M, 8), R->current1 = xcalloc(3 * M, 8), R->J = xcalloc(3 * M, 8), R->gamma = xcalloc(3 * M, 8);
    R->smooth_buf = xcalloc(3 * M, 8), R->Bprev = xcalloc(3 * M, 8), R->Ecovar = xcalloc(3 * M, 8);
    R->Pe = xcalloc(M, 8), R->dPe = xcalloc(3 * M, 8), R->Je = xcalloc(3 * M, 8), R->covar = xcalloc(3 * M, 8), R->contr = xcalloc(3 * M, 8);
    for (int s = 0; s < p->n_kinetic; ++s)
        R->mom0[s] = xcalloc(M, 8), R->mom1[s] = xcalloc(3 * M, 8), R->mom2[s] = xcalloc(6 * M, 8);
    for (int s = 0; s < p->n_kinetic; ++s) {
        R->eq0[s] = xcalloc(M, 8), R->eq2[s] = xcalloc(6 * M, 8);
        if (evolves_psd(&p->kinetic[s]) || p->kinetic[s].scheme == H1D_DELTA_F)
            cache_equilibrium(R, s);
    }
    R->pmom0 = xcalloc(M, 8), R->pmom1 = xcalloc(3 * M, 8);
    for (int s = 0; s < p->n_cold; ++s) {
        R->cn_full[s] = xcalloc(M, 8), R->cnV_full[s] = xcalloc(3 * M, 8);
        R->cmom0[s] = xcalloc(M, 8), R->cmom1[s] = xcalloc(3 * M, 8), R->cmom2[s] = xcalloc(6 * M, 8);
    }
    R->pc_n_full = xcalloc(M, 8), R->pc_nV_full = xcalloc(3 * M, 8);
    for (int e = 0; e < R->p.n_sources; ++e)
        R->smom0[e] = xcalloc(M, 8), R->smom1[e] = xcalloc(3 * M, 8);
    *out = R;
    return H1D_OK;
}

int orc_destroy(orc_run *R)
{
    if (!R)
        return H1D_OK;
    double *all[] = { R->B, R->B1, R->E, R->E1, R->charge, R->charge1, R->rho, R->lambda, R->current, R->current1, R->J,
                      R->gamma, R->smooth_buf, R->Bprev, R->Ecovar, R->Pe, R->dPe, R->Je, R->covar, R->contr, R->pmom0,
                      R->pmom1, R->pc_n_full, R->pc_nV_full };
    for (size_t k = 0; k < sizeof all / sizeof *all; ++k)
        free(all[k]);
    for (int s = 0; s < R->p.n_kinetic; ++s)
        free(R->mom0[s]), free(R->mom1[s]), free(R->mom2[s]), bucket_free(&R->part[s]);
    for (int s = 0; s < R->p.n_kinetic; ++s)
        free(R->eq0[s]), free(R->eq2[s]);
    for (int s = 0; s < R->p.n_cold; ++s)
        free(R->cn_full[s]), free(R->cnV_full[s]), free(R->cmom0[s]), free(R->cmom1[s]), free(R->cmom2[s]);
    for (int e = 0; e < R->p.n_sources; ++e)
        free(R->smom0[e]), free(R->smom1[e]);
    bucket_free(&R->pred), bucket_free(&R->bufL), bucket_free(&R->bufR);
    free(R);
    return H1D_OK;
}

int orc_upload_particles(orc_run *R, int s, int64_t n, double const *q1, double const *vx, double const *vy,
                         double const *vz, double const *w)
{
    if (!R || s < 0 || s >= R->p.n_kinetic || n < 0)
        return H1D_ERR_INVALID_ARG;
    Bucket *b = &R->part[s];
    bucket_reserve(b, n);
    b->n = n;
    memcpy(b->q1, q1, 8 * n), memcpy(b->vx, vx, 8 * n), memcpy(b->vy, vy, 8 * n), memcpy(b->vz, vz, 8 * n),
        memcpy(b->w, w, 8 * n);
    for (int64_t k = 0; k < n; ++k)
        b->pid[k] = k, b->real_f[k] = w[k], b->marker[k] = 1.0;
    return H1D_OK;
}
int orc_upload_psd(orc_run *R, int s, int64_t n, double const *real_f, double const *marker)
{
    if (!R || s < 0 || s >= R->p.n_kinetic || n != R->part[s].n || (n && (!real_f || !marker)))
        return H1D_ERR_INVALID_ARG;
    memcpy(R->part[s].real_f, real_f, 8 * n), memcpy(R->part[s].marker, marker, 8 * n);
    return H1D_OK;
}
int orc_download_psd(orc_run *R, int s, double *real_f, double *marker)
{
    if (!R || s < 0 || s >= R->p.n_kinetic)
        return H1D_ERR_INVALID_ARG;
    Bucket const *b = &R->part[s];
    if (real_f) memcpy(real_f, b->real_f, 8 * b->n);
    if (marker) memcpy(marker, b->marker, 8 * b->n);
    return H1D_OK;
}
int orc_upload_fields(orc_run *R, double const *B, double const *E)
{
    if (!R)
        return H1D_ERR_INVALID_ARG;
    if (B)
        memcpy(R->B, B, sizeof(double) * 3 * R->M);
    if (E)
        memcpy(R->E, E, sizeof(double) * 3 * R->M);
    return H1D_OK;
}
int orc_upload_cold(orc_run *R, int i, double const *n_full, double const *nV_full)
{
    if (!R || i < 0 || i >= R->p.n_cold)
        return H1D_ERR_INVALID_ARG;
    memcpy(R->cn_full[i], n_full, sizeof(double) * R->M);
    memcpy(R->cnV_full[i], nV_full, sizeof(double) * 3 * R->M);
    return H1D_OK;
}

/* Domain_CAMCL::advance_by (Domain_CAMCL.cc:21-56) / Domain_PC::advance_by (Domain_PC.cc:21-78) */
int orc_advance(orc_run *R, uint32_t n_steps)
{
    if (!R)
        return H1D_ERR_INVALID_ARG;
    int ok = 1;
    if (!R->recurring) {
        R->recurring = 1;
        pass_grid(R, R->E, 3);
        pass_grid(R, R->B, 3);
        if (R->p.algorithm == H1D_ALGO_PC) {
            long const M = R->M;
            memset(R->charge, 0, sizeof(double) * M);
            memset(R->current, 0, sizeof(double) * 3 * M);
            for (int s = 0; s < R->p.n_kinetic; ++s) {
                h1d_kinetic_desc const *d = &R->p.kinetic[s];
                collect_part(R, &R->part[s], d, R->mom0[s], R->mom1[s]);
                addto(R->charge, collect_smooth_rho(R, R->mom0[s], d->Oc, d->op, d->n_smooth), M);
                addto(R->current, collect_smooth_J(R, R->mom1[s], d->Oc, d->op, d->n_smooth), 3 * M);
            }
            for (int ci = 0; ci < R->p.n_cold; ++ci) {
                h1d_cold_desc const *d = &R->p.cold[ci];
                pass_grid(R, R->cn_full[ci], 1);
                pass_grid(R, R->cnV_full[ci], 3);
                cold_collect_part(R, R->cn_full[ci], R->cnV_full[ci], R->cmom0[ci], R->cmom1[ci]);
                addto(R->charge, collect_smooth_rho(R, R->cmom0[ci], d->Oc, d->op, d->n_smooth), M);
                addto(R->current, collect_smooth_J(R, R->cmom1[ci], d->Oc, d->op, d->n_smooth), 3 * M);
            }
            for (int e = 0; e < R->p.n_sources; ++e) { /* a predictor copy's update(0) */
                src_collect(R, e, (double)R->step * R->p.dt + 0);
                src_add(R, e, R->charge, R->current);
            }
        }
    }
    for (uint32_t i = 0; i < n_steps; ++i) {
        int const step_ok = R->p.algorithm == H1D_ALGO_CAMCL ? camcl_cycle(R) : pc_cycle(R);
        R->step++;
        if (!step_ok) {
            ok = 0;
            break; /* the reference throws from inside cycle() */
        }
    }
    /* post-process: collect all moments */
    for (int s = 0; s < R->p.n_kinetic; ++s) {
        collect_all(R, &R->part[s], &R->p.kinetic[s], R->mom0[s], R->mom1[s], R->mom2[s]);
        gather_grid(R, R->mom0[s], 1);
        gather_grid(R, R->mom1[s], 3);
        gather_grid(R, R->mom2[s], 6);
    }
    for (int ci = 0; ci < R->p.n_cold; ++ci) {
        cold_collect_part(R, R->cn_full[ci], R->cnV_full[ci], R->cmom0[ci], R->cmom1[ci]);
        double *nvv = R->cmom2[ci], *n = R->cmom0[ci], *nV = R->cmom1[ci];
        for (long i = 0; i < R->Nx; ++i) {
            double const  ni = n[i + P];
            double const *v  = nV + 3 * (i + P);
            double       *t  = nvv + 6 * (i + P);
            t[0] = t[3] = v[0] / ni;
            t[1] = t[4] = v[1] / ni;
            t[2] = t[5] = v[2] / ni;
            t[0] *= v[0], t[1] *= v[1], t[2] *= v[2];
            t[3] *= v[1], t[4] *= v[2], t[5] *= v[0];
        }
        gather_grid(R, R->cmom0[ci], 1);
        gather_grid(R, R->cmom1[ci], 3);
        gather_grid(R, R->cmom2[ci], 6);
    }
    if (!ok) {
        snprintf(R->msg, sizeof R->msg, "update_pos - particle(s) moved too far");
        return H1D_ERR_MOVED_TOO_FAR;
    }
    return H1D_OK;
}

int orc_particle_count(orc_run *R, int s, int64_t *n)
{
    if (!R || s < 0 || s >= R->p.n_kinetic || !n)
        return H1D_ERR_INVALID_ARG;
    *n = R->part[s].n;
    return H1D_OK;
}
int orc_download_particles(orc_run *R, int s, double *q1, double *vx, double *vy, double *vz, double *w, int64_t *pid)
{
    if (!R || s < 0 || s >= R->p.n_kinetic)
        return H1D_ERR_INVALID_ARG;
    Bucket const *b = &R->part[s];
    if (q1) memcpy(q1, b->q1, 8 * b->n);
    if (vx) memcpy(vx, b->vx, 8 * b->n);
    if (vy) memcpy(vy, b->vy, 8 * b->n);
    if (vz) memcpy(vz, b->vz, 8 * b->n);
    if (w) memcpy(w, b->w, 8 * b->n);
    if (pid) memcpy(pid, b->pid, 8 * b->n);
    return H1D_OK;
}
int orc_download_fields(orc_run *R, double *B, double *E)
{
    if (!R)
        return H1D_ERR_INVALID_ARG;
    if (B) memcpy(B, R->B, sizeof(double) * 3 * R->M);
    if (E) memcpy(E, R->E, sizeof(double) * 3 * R->M);
    return H1D_OK;
}
int orc_download_sources(orc_run *R, double *charge, double *current)
{
    if (!R)
        return H1D_ERR_INVALID_ARG;
    if (charge) memcpy(charge, R->charge, sizeof(double) * R->M);
    if (current) memcpy(current, R->current, sizeof(double) * 3 * R->M);
    return H1D_OK;
}
int orc_download_moments(orc_run *R, int s, double *n, double *nV, double *nvv)
{
    if (!R || s < 0 || s >= R->p.n_kinetic)
        return H1D_ERR_INVALID_ARG;
    if (n) memcpy(n, R->mom0[s], sizeof(double) * R->M);
    if (nV) memcpy(nV, R->mom1[s], sizeof(double) * 3 * R->M);
    if (nvv) memcpy(nvv, R->mom2[s], sizeof(double) * 6 * R->M);
    return H1D_OK;
}
int orc_download_cold(orc_run *R, int i, double *n, double *nV, double *nvv, double *n_full, double *nV_full)
{
    if (!R || i < 0 || i >= R->p.n_cold)
        return H1D_ERR_INVALID_ARG;
    if (n) memcpy(n, R->cmom0[i], sizeof(double) * R->M);
    if (nV) memcpy(nV, R->cmom1[i], sizeof(double) * 3 * R->M);
    if (nvv) memcpy(nvv, R->cmom2[i], sizeof(double) * 6 * R->M);
    if (n_full) memcpy(n_full, R->cn_full[i], sizeof(double) * R->M);
    if (nV_full) memcpy(nV_full, R->cnV_full[i], sizeof(double) * 3 * R->M);
    return H1D_OK;
}

/* VHistogramRecorder::histogram / local_counting (Recorder/VHistogramRecorder.cc:222-306) on one
 * process: particles with q1 in [ext_loc, ext_loc + ext_len) (Range::is_member), velocity relative
 * to the local bulk velocity nV/n interpolated with Shape<1> from the recorded moments (zero where
 * n < 1e-15), gyro-averaged (v1 = v_par, v2 = |v_perp|; the field-aligned basis is Cartesian on the
 * field line), binned by floor((v - min) * dim / len); per bin {marker count, weight sum,
 * real_f/marker sum} divided by the number of particles in the extent (without a phase-space
 * density upload real_f = w and marker = 1, so real_f/marker = w). */
int orc_vhistogram(orc_run *R, int s, double ext_loc, double ext_len, double v1min, double v1len, int64_t v1dim,
                   double v2min, double v2len, int64_t v2dim, double *out, int64_t *total)
{
    if (!R || s < 0 || s >= R->p.n_kinetic || v1dim <= 0 || v2dim <= 0 || !(v1len > 0) || !(v2len > 0) || !out)
        return H1D_ERR_INVALID_ARG;
    memset(out, 0, sizeof(double) * 3 * (size_t)(v1dim * v2dim));
    Bucket const *b     = &R->part[s];
    int64_t       count = 0;
    for (int64_t k = 0; k < b->n; ++k) {
        double const q1 = b->q1[k];
        if (!(q1 >= ext_loc && q1 < ext_loc + ext_len))
            continue;
        ++count;
        Shp sh;
        shape1(&sh, q1 - R->half_min);
        double n = 0;
        for (int j = 0; j <= 1; ++j)
            n += *at1(R->mom0[s], sh.i[j]) * sh.w[j];
        V3 V = interp3(R->mom1[s], &sh, 1);
        if (n < 1e-15)
            V.x = V.y = V.z = 0;
        else
            V.x /= n, V.y /= n, V.z /= n;
        double const v1 = b->vx[k] - V.x, vy = b->vy[k] - V.y, vz = b->vz[k] - V.z;
        double const v2 = sqrt(vy * vy + vz * vz);
        double const f1 = floor((v1 - v1min) * (double)v1dim / v1len);
        double const f2 = floor((v2 - v2min) * (double)v2dim / v2len);
        if (f1 >= 0 && f1 < (double)v1dim && f2 >= 0 && f2 < (double)v2dim) {
            double *o = out + 3 * ((int64_t)f1 * v2dim + (int64_t)f2);
            o[0] += 1, o[1] += b->w[k], o[2] += b->real_f[k] / b->marker[k];
        }
    }
    if (count > 0)
        for (int64_t i = 0; i < 3 * v1dim * v2dim; ++i)
            out[i] /= (double)count;
    if (total)
        *total = count;
    return H1D_OK;
}

/* EnergyRecorder::dump (EnergyRecorder.cc:98-140); MFA <-> Cartesian is a pass-through */
int orc_energy(orc_run *R, double *dB2O2, double *dE2O2, double *KE_lab, double *KE_pla)
{
    if (!R)
        return H1D_ERR_INVALID_ARG;
    long const   N     = R->Nx;
    double const denom = 2 * (double)N;
    double       b[3] = { 0, 0, 0 }, e[3] = { 0, 0, 0 };
    for (long i = 0; i < N; ++i)
        for (int c = 0; c < 3; ++c) {
            double const x = R->B[3 * (i + P) + c];
            b[c] += x * x;
            double const y = R->E[3 * (i + P) + c];
            e[c] += y * y;
        }
    for (int c = 0; c < 3; ++c)
        dB2O2[c] = b[c] / denom, dE2O2[c] = e[c] / denom;
    int const ns = R->p.n_kinetic + R->p.n_cold;
    for (int s = 0; s < ns; ++s) {
        double *n, *nV, *nvv, Oc, op;
        if (s < R->p.n_kinetic)
            n = R->mom0[s], nV = R->mom1[s], nvv = R->mom2[s], Oc = R->p.kinetic[s].Oc, op = R->p.kinetic[s].op;
        else
            n = R->cmom0[s - R->p.n_kinetic], nV = R->cmom1[s - R->p.n_kinetic], nvv = R->cmom2[s - R->p.n_kinetic],
            Oc = R->p.cold[s - R->p.n_kinetic].Oc, op = R->p.cold[s - R->p.n_kinetic].op;
        double lab[3] = { 0, 0, 0 }, pla[3] = { 0, 0, 0 };
        for (long i = 0; i < N; ++i) {
            double const ni = n[i + P];
            if (ni < 1e-15)
                continue;
            double const *t = nvv + 6 * (i + P), *v = nV + 3 * (i + P);
            for (int c = 0; c < 3; ++c) {
                lab[c] += t[c];
                pla[c] += t[c] - v[c] * v[c] / ni;
            }
        }
        double const tmp = R->p.O0 / Oc * op / R->p.c; /* Species.h:50-54 */
        double const f   = tmp * tmp / (2 * (double)N);
        for (int c = 0; c < 3; ++c)
            KE_lab[3 * s + c] = lab[c] * f, KE_pla[3 * s + c] = pla[c] * f;
    }
    return H1D_OK;
}

char const *orc_status_string(orc_run *R) { return R ? R->msg : "null run"; }
int         orc_step_count(orc_run *R) { return R ? (int)R->step : -1; }

/* ------------------------------------------------------------------------------------------------
 * primitive probes for the known-answer tests of the LibPIC unit tests
 * (src/LibPIC/test/test-Shape.cc, test-BorisPush.cc, test-Geometry.cc, test-MaskingFunction.cc,
 *  test-GridArray.cc)
 */
void orc_shape(int order, double x, int64_t *idx, double *w)
{
    Shp s;
    shape(&s, order, x);
    for (int j = 0; j <= order; ++j)
        idx[j] = s.i[j], w[j] = s.w[j];
}
void orc_boris(double dt, double c, double O0, double Oc, double *v, double const *B, double const *E)
{
    Boris const b  = boris_make(dt, c, O0, Oc);
    V3          vv = { v[0], v[1], v[2] };
    V3 const    BB = { B[0], B[1], B[2] }, EE = { E[0], E[1], E[2] };
    boris_push(&b, &vv, BB, EE);
    v[0] = vv.x, v[1] = vv.y, v[2] = vv.z;
}
double orc_mask(int64_t inset, double factor, double offset) { return mask_fn((long)inset, factor, offset); }
/* out: [0] curvi q1 of Cartesian x (MirrorGeometry.cc:24-33), [1] x back from q1,
 *      [2..4] Bcart_div_B0(q1, y, z), [5] Bmag_div_B0(q1), [6] contravariant q1-velocity of v=(1,0,0) */
void orc_geometry(double xi, double D1, double x, double y, double z, double *out)
{
    orc_run R;
    memset(&R, 0, sizeof R);
    R.xi = xi, R.xi2 = xi * xi, R.D1 = D1, R.D2 = R.D3 = 1, R.inv_D1 = 1 / D1, R.inv_D2 = R.inv_D3 = 1;
    R.homogeneous = xi < 1e-10;
    R.p.O0        = 1;
    double q1;
    if (R.homogeneous) {
        double const sqrt_3 = 1.732050807568877193176604123436845839024;
        double const tmp    = xi * x / sqrt_3;
        q1                  = (1 - tmp) * (1 + tmp) * x / D1;
    } else {
        q1 = atan(xi * x) / (xi * D1);
    }
    out[0]     = q1;
    out[1]     = g_curvi_to_cart(&R, q1);
    V3 const b = g_Bcart_yz(&R, q1, y, z);
    out[2] = b.x, out[3] = b.y, out[4] = b.z;
    out[5]      = g_BOB0(&R, q1);
    V3 const v  = { 1, 0, 0 };
    out[6]      = g_cart_to_contr(&R, v, q1).x;
}
/* GridArray::smooth_assign / deposit / interp on a scalar grid of N interior cells */
void orc_grid_smooth(int64_t N, double const *src, double *dst)
{
    for (int64_t i = 0; i < N; ++i)
        dst[i + P] = (src[i - 1 + P] + 2 * src[i + P] + src[i + 1 + P]) * .25;
}
void orc_grid_deposit(int order, double x, double weight, double *g)
{
    Shp s;
    shape(&s, order, x);
    for (int j = 0; j <= order; ++j)
        g[s.i[j] + P] += weight * s.w[j];
}
double orc_grid_interp(int order, double x, double const *g)
{
    Shp s;
    shape(&s, order, x);
    double y = 0;
    for (int j = 0; j <= order; ++j)
        y += g[s.i[j] + P] * s.w[j];
    return y;
}
