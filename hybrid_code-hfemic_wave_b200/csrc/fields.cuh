// Grid phase of the hybrid_1d hot path (FP64): everything of one cycle that is not a particle
// loop, in one kernel launch.
//
// CAM-CL (src/hybrid_1d/Core/Domain_CAMCL.cc:57-193):
//   per species collect_smooth of n/nV at x^N and x^{N+1} (Domain.hh:35-74): 1/Nc scale,
//   charge/current conversion factors (Species.h:42-49), ghost fold (SubdomainDelegate.cc:122-181),
//   3-point smoothing (GridArray.h:134-142); cold fluid push and moments (ColdSpecies.cc:31-65);
//   averaging; the B subcycle with Ohm's-law E (BField.cc:24-74, EField.cc:41-126);
//   E*, current advance with Lambda/Gamma (Domain_CAMCL.cc:131-151, Current.cc:45-52); final E;
//   B on the half grid for the next push (PartSpecies.cc:27-34).
// Predictor-corrector (src/hybrid_1d/Core/Domain_PC.cc:84-205) uses the same building blocks in
// three phases around its two particle passes.
//
// Layout and parallelisation.  Every grid quantity of the reference, ghost cells included, is
// the periodic image of the interior after each boundary_pass (ghosts are filled periodically
// whatever the particle boundary; only the moment fold and the masking depend on position).  So
// each CTA owns `seg` interior cells and recomputes, redundantly, a halo of `H` cells on each side
// from the step's inputs; H is larger than the total stencil reach of one cycle, so CTAs never
// exchange data inside a step and there is no inter-CTA synchronisation.  One thread per local
// cell; all arrays of the cycle live in shared memory.  Per-cell geometry (cos of the mirror
// field at full and half grid points, masking factors) is tabulated once on the host.
//
// This file is compiled without FMA contraction so that, given the same moments, the field
// cycle evaluates the reference's expressions operation for operation.
#pragma once

#include "device_common.cuh"

namespace h1d {

constexpr int MAXK = 8;
constexpr int MAXC = 4;
constexpr int MAXE = 2; // external current sources

// per-cell geometry table, SoA over the Nx interior cells (index = interior cell)
enum GeoIdx {
    G_FCOV_X, G_FCOV_Y, G_FCOV_Z, // covariant basis at full-grid points  (CurviBasis.h:52-56)
    G_FCON_X, G_FCON_Y, G_FCON_Z, // contravariant basis at full-grid points (CurviBasis.h:65-69)
    G_HCOV_X, G_HCOV_Y, G_HCOV_Z, // same at half-grid points
    G_HCON_X, G_HCON_Y, G_HCON_Z,
    G_HBX,                        // Bcart(half point).x = O0/cos^2 (MFABasis.h:47)
    G_MP1, G_MP2, G_MA1, G_MA2,   // phase-retardation / amplitude-damping factors, in the order
                                  // the reference applies them (BField.cc:40-48)
    G_COUNT
};

struct KinSrc {
    double const *raw[2][4]; // unscaled deposits at x^N and x^{N+1}: n, nVx, nVy, nVz (cell 0)
    double const *eq;        // delta-f: equilibrium n0 added to the density moment (cell 0), or null
    double       *zero[2][4]; // the deposit set of the next cycle, cleared here
    double        s1;         // 1/Nc (PartSpecies.cc:222-223)
    double        cdcf, ccf;  // charge / current density conversion factors
    double        lamf, gamf; // Lambda / Gamma factors (Charge.cc:31-36, Current.cc:34-39)
    int           nsm;
};
struct ColdSrc {
    double const *n;    // mom0_full (cell 0)
    double const *nV_in;
    double       *nV_out;
    BorisK        boris;
    double        cdcf, ccf, lamf, gamf, w;
    int           nsm;
};

struct FieldArgs {
    int           Nx, H, seg, bc;
    double const *geo; // G_COUNT x Nx
    double const *B_in, *E_in; // AoS, cell 0
    double       *B_out, *E_out, *EB_out, *charge_out, *current_out; // EB: {E, B on the half grid} per cell
    float        *EBf_out; // FP32 copy of EB for the mixed-precision particle pass, or null
    int           nk, nc;
    KinSrc        k[MAXK];
    ColdSrc       c[MAXC];
    // external sources (Core/ExternalSource.cc:12-66) as species whose raw[0] = raw[1] is the
    // source's moment<1> (n zero), s1 = 1, charge / current factors 0 / 1, Lambda / Gamma 0 / 1
    int           ne;
    KinSrc        e[MAXE];
    double        dt, sub_dt, c_light, sqrt_g, O0, inv_D1;
    int           m;  // n_subcycles
    int           fb; // CAM-CL: sources smoothed together per group of barrier phases (<= FB_MAX)
    // electron fluid (EField.cc:63-87)
    double        mOeOO0oe2, gamma, O02beO2, cO2, cOsqrtg;
    // predictor-corrector (Domain_PC.cc:84-205): phase 0 initial sources, 1 predicted fields,
    // 2 after the predictor deposit, 3 after the corrector deposit
    int           phase;
    double const *charge_in, *current_in; // sources of the previous corrector (cell 0)
    double const *E1_in;                  // averaged E of the previous phase (cell 0)
    double       *E1_out;                 // averaged E for the next particle pass (cell 0)
};

// block -> (run, segment) of a batched field launch
struct FieldBlock {
    int run, seg;
};

struct Cell {
    int    t, L, g, gm;
    bool   owner;
    double fcx, fcy, fcz, fnx, fny, fnz, hcx, hcy, hcz, hnx, hny, hnz, hbx, mp1, mp2, ma1, ma2;
};

// fold of one raw deposit array onto interior cell gm, times 1/Nc (plus the delta-f equilibrium
// eq, zero in the ghost cells; PartSpecies.cc:115-128) and a conversion factor
__device__ __forceinline__ double fold(double const *r, int gm, int Nx, int bc, double s1, double f,
                                       double const *eq = nullptr)
{
    double m = r[gm] * s1;
    if (eq)
        m = m + eq[gm] * 1.0;
    double v = m * f;
    if (bc == 0) {
        if (gm < PAD)
            v = v + (r[Nx + gm] * s1) * f;
        if (gm >= Nx - PAD)
            v = v + (r[gm - Nx] * s1) * f;
    } else {
        if (gm == 0)
            v = v + ((r[-1] * s1) * f + ((r[-2] * s1) * f + (r[-3] * s1) * f));
        if (gm == Nx - 1)
            v = v + ((r[Nx] * s1) * f + ((r[Nx + 1] * s1) * f + (r[Nx + 2] * s1) * f));
    }
    return v;
}

__device__ __forceinline__ d3 sld3(double const *a, int t) { return { a[3 * t], a[3 * t + 1], a[3 * t + 2] }; }
__device__ __forceinline__ void sst3(double *a, int t, d3 v) { a[3 * t] = v.x, a[3 * t + 1] = v.y, a[3 * t + 2] = v.z; }

// n smoothings of a scalar and a vector array together (Charge::smooth / Current::smooth,
// GridArray.h:134-142); ping-pongs between (a, v) and (ta, tv) and returns where the result is
struct SV {
    double *a, *v;
};
static __device__ SV smooth_n(Cell const &C, int n, double *a, double *v, double *ta, double *tv)
{
    int const tl = max(C.t - 1, 0), tr = min(C.t + 1, C.L - 1);
    for (int it = 0; it < n; ++it) {
        __syncthreads();
        ta[C.t] = (a[tl] + 2 * a[C.t] + a[tr]) * .25;
        for (int k = 0; k < 3; ++k)
            tv[3 * C.t + k] = (v[3 * tl + k] + 2 * v[3 * C.t + k] + v[3 * tr + k]) * .25;
        double *x = a;
        a         = ta;
        ta        = x;
        x         = v;
        v         = tv;
        tv        = x;
    }
    __syncthreads();
    return { a, v };
}

__device__ __forceinline__ d3 covar_full(Cell const &C, d3 b) { return { C.fcx * b.x, C.fcy * b.y, C.fcz * b.z }; }
__device__ __forceinline__ d3 contr_full(Cell const &C, d3 b) { return { C.fnx * b.x, C.fny * b.y, C.fnz * b.z }; }
template <class G>
__device__ __forceinline__ d3 covar_half(G const &C, d3 b) { return { C.hcx * b.x, C.hcy * b.y, C.hcz * b.z }; }
template <class G>
__device__ __forceinline__ d3 contr_half(G const &C, d3 b) { return { C.hnx * b.x, C.hny * b.y, C.hnz * b.z }; }
template <class G>
__device__ __forceinline__ d3 mask_p(G const &C, d3 v) { return (v * C.mp1) * C.mp2; }
template <class G>
__device__ __forceinline__ d3 mask_a(G const &C, d3 v) { return (v * C.ma1) * C.ma2; }

// electron pressure gradient, masked (EField.cc:63-87, 44): needs Pe of the neighbours
__device__ __forceinline__ double dPe_at(FieldArgs const &a, Cell const &C, double const *Pe)
{
    int const tl = max(C.t - 1, 0), tr = min(C.t + 1, C.L - 1);
    return ((Pe[tr] - Pe[tl]) * a.cO2 * C.mp1) * C.mp2;
}
// pow(x, 1) is x exactly (the isothermal closure), so that case skips the library pow
__device__ __forceinline__ double Pe_of(FieldArgs const &a, double rho)
{
    double const x = a.mOeOO0oe2 * rho;
    return (a.gamma == 1.0 ? x : pow(x, a.gamma)) * a.O02beO2;
}

// Ohm's law at local cell t with half-grid geometry C (EField.cc:88-126) from Bcov/Bcon of the
// current B (with the neighbour at t+1), contravariant current jc, masked dPe and rho; returns
// the masked E
template <class G>
__device__ __forceinline__ d3 E_at_g(FieldArgs const &a, G const &C, int t, int L, double const *Bcov, double const *Bcon,
                                     d3 jc, double dPe, double rho)
{
    int const tr = min(t + 1, L - 1);
    d3 const  B1 = sld3(Bcov, tr), B0 = sld3(Bcov, t);
    d3        Je = { 0 - jc.x, (-B1.z + B0.z) * a.cOsqrtg - jc.y, (+B1.y - B0.y) * a.cOsqrtg - jc.z };
    Je           = mask_p(C, Je);
    d3 const  d1 = sld3(Bcon, tr), d0 = sld3(Bcon, t);
    d3 const  Bc = { a.inv_D1 * a.O0 + (d1.x + d0.x) * 0.5, 0 * a.O0 + (d1.y + d0.y) * 0.5, 0 * a.O0 + (d1.z + d0.z) * 0.5 };
    d3 const  lz = cross(Je, Bc) * a.sqrt_g;
    d3 const  Ec = { (lz.x - dPe) / rho, (lz.y - 0.0) / rho, (lz.z - 0.0) / rho };
    return mask_a(C, contr_half(C, Ec));
}
// E_at_g inside the B subcycle: only the y and z components (the ones Faraday's law reads; x is
// returned as 0), and the division by the density, which the sub-steps share, as a multiplication
// by its reciprocal (within one rounding of the quotient)
__device__ __forceinline__ d3 E_sub(FieldArgs const &a, Cell const &C, int t, int L, double const *Bcov, double const *Bcon,
                                    d3 jc, double inv_rho)
{
    int const    tr  = min(t + 1, L - 1);
    double const B1y = Bcov[3 * tr + 1], B1z = Bcov[3 * tr + 2], B0y = Bcov[3 * t + 1], B0z = Bcov[3 * t + 2];
    d3           Je  = { 0 - jc.x, (-B1z + B0z) * a.cOsqrtg - jc.y, (+B1y - B0y) * a.cOsqrtg - jc.z };
    Je               = mask_p(C, Je);
    d3 const     d1  = sld3(Bcon, tr), d0 = sld3(Bcon, t);
    d3 const     Bc  = { a.inv_D1 * a.O0 + (d1.x + d0.x) * 0.5, 0 * a.O0 + (d1.y + d0.y) * 0.5, 0 * a.O0 + (d1.z + d0.z) * 0.5 };
    double const ly  = (Je.z * Bc.x - Je.x * Bc.z) * a.sqrt_g;
    double const lz  = (Je.x * Bc.y - Je.y * Bc.x) * a.sqrt_g;
    double const ey  = (ly - 0.0) * inv_rho, ez = (lz - 0.0) * inv_rho;
    return { 0.0, ((C.hny * ey) * C.ma1) * C.ma2, ((C.hnz * ez) * C.ma1) * C.ma2 }; // mask_a(contr_half(Ec))
}
__device__ __forceinline__ d3 E_at(FieldArgs const &a, Cell const &C, double const *Bcov, double const *Bcon, d3 jc,
                                   double dPe, double rho)
{
    return E_at_g(a, C, C.t, C.L, Bcov, Bcon, jc, dPe, rho);
}

// Faraday at this cell (BField.cc:50-64) from the covariant E at this cell (E1) and at the one
// before (E0); returns the new masked B
__device__ __forceinline__ d3 B_at_e(FieldArgs const &a, Cell const &C, d3 E1, d3 E0, d3 Bprev, double dtp)
{
    double const k = dtp * a.c_light / a.sqrt_g;
    d3 const     Bc = { 0, (-E1.z + E0.z) * k, (+E1.y - E0.y) * k };
    d3 const     Bk = covar_full(C, Bc); // contr_to_cart uses the covariant basis
    d3           B  = { 0 - Bk.x, 0 - Bk.y, 0 - Bk.z };
    B               = mask_p(C, B);
    B               = B + Bprev;
    return mask_a(C, B);
}
// the same with Ecov from shared memory (at t and t-1)
__device__ __forceinline__ d3 B_at(FieldArgs const &a, Cell const &C, double const *Ecov, d3 Bprev, double dtp)
{
    int const t = C.t, tl = max(t - 1, 0);
    return B_at_e(a, C, sld3(Ecov, t), sld3(Ecov, tl), Bprev, dtp);
}

__device__ __forceinline__ void load_cell(FieldArgs const &a, Cell &C, int blk)
{
    C.t     = threadIdx.x;
    C.L     = blockDim.x;
    int const g0 = blk * a.seg;
    C.g     = g0 - a.H + C.t;
    C.gm    = ((C.g % a.Nx) + a.Nx) % a.Nx;
    C.owner = C.t >= a.H && C.t < a.H + a.seg && C.g < a.Nx;
    double const *G = a.geo;
    long const    N = a.Nx, i = C.gm;
    C.fcx = G[G_FCOV_X * N + i], C.fcy = G[G_FCOV_Y * N + i], C.fcz = G[G_FCOV_Z * N + i];
    C.fnx = G[G_FCON_X * N + i], C.fny = G[G_FCON_Y * N + i], C.fnz = G[G_FCON_Z * N + i];
    C.hcx = G[G_HCOV_X * N + i], C.hcy = G[G_HCOV_Y * N + i], C.hcz = G[G_HCOV_Z * N + i];
    C.hnx = G[G_HCON_X * N + i], C.hny = G[G_HCON_Y * N + i], C.hnz = G[G_HCON_Z * N + i];
    C.hbx = G[G_HBX * N + i];
    C.mp1 = G[G_MP1 * N + i], C.mp2 = G[G_MP2 * N + i], C.ma1 = G[G_MA1 * N + i], C.ma2 = G[G_MA2 * N + i];
}

// owner writes of an interior value and of its ghost images (periodic fill, Delegate.cc:76-87)
__device__ __forceinline__ void put3(double *g, Cell const &C, int Nx, d3 v)
{
    st3(g, C.gm, v);
    if (C.gm < PAD)
        st3(g, Nx + C.gm, v);
    if (C.gm >= Nx - PAD)
        st3(g, C.gm - Nx, v);
}
__device__ __forceinline__ void put1(double *g, Cell const &C, int Nx, double v)
{
    g[C.gm] = v;
    if (C.gm < PAD)
        g[Nx + C.gm] = v;
    if (C.gm >= Nx - PAD)
        g[C.gm - Nx] = v;
}

// owner write of the interleaved push record {E, B averaged onto the half grid} and its ghost
// images; the half-grid B of the last ghost cell stays NaN (PartSpecies.cc:32)
__device__ __forceinline__ void put_eb(double *eb, float *ebf, Cell const &C, int Nx, d3 E, d3 Bh)
{
    auto put = [&](int i, bool withB) {
        double *p = eb + 6 * i;
        p[0] = E.x, p[1] = E.y, p[2] = E.z;
        if (withB)
            p[3] = Bh.x, p[4] = Bh.y, p[5] = Bh.z;
        if (ebf) {
            float *f = ebf + EBF_STRIDE * i;
            f[0] = static_cast<float>(E.x), f[1] = static_cast<float>(E.y), f[2] = static_cast<float>(E.z);
            if (withB)
                f[3] = static_cast<float>(Bh.x), f[4] = static_cast<float>(Bh.y), f[5] = static_cast<float>(Bh.z);
        }
    };
    put(C.gm, true);
    if (C.gm < PAD)
        put(Nx + C.gm, C.gm < PAD - 1);
    if (C.gm >= Nx - PAD)
        put(C.gm - Nx, true);
}

// shared-memory carve-up: 9 scalar and 14 vector arrays of L doubles
struct Smem {
    double *rho0, *rho1, *tr, *ts, *Pe, *Pe1, *lam, *t2, *rho_avg;
    double *J0, *J1, *tJ, *tJs, *B0, *B1, *E, *Bcov, *Bcon, *Ecov, *gam, *Jsum, *Javg, *aux;
};
constexpr int SMEM_SCALARS = 9, SMEM_VECTORS = 14;
__device__ __forceinline__ Smem carve(double *sm, int L)
{
    Smem s;
    double *p = sm;
    s.rho0 = p, p += L;
    s.rho1 = p, p += L;
    s.tr = p, p += L;
    s.ts = p, p += L;
    s.Pe = p, p += L;
    s.Pe1 = p, p += L;
    s.lam = p, p += L;
    s.t2 = p, p += L;
    s.rho_avg = p, p += L;
    s.J0 = p, p += 3 * L;
    s.J1 = p, p += 3 * L;
    s.tJ = p, p += 3 * L;
    s.tJs = p, p += 3 * L;
    s.B0 = p, p += 3 * L;
    s.B1 = p, p += 3 * L;
    s.E = p, p += 3 * L;
    s.Bcov = p, p += 3 * L;
    s.Bcon = p, p += 3 * L;
    s.Ecov = p, p += 3 * L;
    s.gam = p, p += 3 * L;
    s.Jsum = p, p += 3 * L;
    s.Javg = p, p += 3 * L;
    s.aux = p, p += 3 * L;
    return s;
}

// collect_smooth of one kinetic species' deposit d; ends synchronised
static __device__ SV collect_kinetic(FieldArgs const &a, Cell const &C, Smem const &S, KinSrc const &K, int d)
{
    int const gm = C.gm;
    S.tr[C.t]    = fold(K.raw[d][0], gm, a.Nx, a.bc, K.s1, K.cdcf, K.eq);
    for (int q = 0; q < 3; ++q)
        S.tJ[3 * C.t + q] = fold(K.raw[d][1 + q], gm, a.Nx, a.bc, K.s1, K.ccf);
    return smooth_n(C, K.nsm, S.tr, S.tJ, S.ts, S.tJs);
}

// cold species (ColdSpecies.cc:31-65): push nV with E and the background field, moments x w
static __device__ d3 cold_push(FieldArgs const &a, Cell const &C, ColdSrc const &K, double const *E_cell0)
{
    d3 const     E  = ld3(E_cell0, C.gm);
    double const n  = K.n[C.gm];
    d3 const     Bc = { C.hbx, 0 * a.O0, 0 * a.O0 };
    return boris_push(K.boris, ld3(K.nV_in, C.gm), Bc, E * n);
}

// shared memory of the CAM-CL field body with smoothing groups of fb items (see below)
constexpr int FB_MAX     = 8;  // items per smoothing group
constexpr int FS_FIXED_L = 16; // arrays of L doubles outside the groups
constexpr int FS_ITEM_L  = 8;  // per item: a, ta (L each), v, tv (3L each)
constexpr int FS_GHOST   = 24; // per item: 4 quantities x 6 ghost-fold partners
__host__ __device__ constexpr size_t camcl_smem_bytes(int L, int fb)
{
    return sizeof(double) * (static_cast<size_t>(L) * (FS_FIXED_L + FS_ITEM_L * fb) + static_cast<size_t>(FS_GHOST) * fb);
}

#ifdef H1D_FIELD_TU
// ------------------------------------------------------------------------------------------------
// CAM-CL cycle: shared-memory layout and the sources' smoothing in groups.
//
// The sources of every species (kinetic deposits at x^N and x^{N+1}, cold fluid, external
// sources) and the current-advance terms are smoothed in groups of up to `fb` items that share
// their barrier phases: an item is a (scalar, vector) pair of arrays with its own smoothing
// count, and a group takes max(count) + 1 barriers however many items it holds.  The raw deposits
// of a group are staged in shared memory first, every thread loading its cell and threads 0..23
// the ghost-fold partners, so the group pays one round of L2 latency.  Each value is computed
// with the same operations, in the same order, as per-species collect_smooth.
// ------------------------------------------------------------------------------------------------
struct CamclSmem {
    double *Pe1;                       // L
    double *Bcov[2], *Bcon[2], *Bavg;  // 3L each; Bcov / Bcon ping-pong across the subcycles
    double *items;                     // per item j at items + 8 L j: a (L), ta (L), v (3L), tv (3L)
    double *gh;                        // ghost-fold partners: [item][quantity][6]
    int     L;
    __device__ __forceinline__ double *a(int j) const { return items + FS_ITEM_L * L * j; }
    __device__ __forceinline__ double *ta(int j) const { return items + FS_ITEM_L * L * j + L; }
    __device__ __forceinline__ double *v(int j) const { return items + FS_ITEM_L * L * j + 2 * L; }
    __device__ __forceinline__ double *tv(int j) const { return items + FS_ITEM_L * L * j + 5 * L; }
};
__device__ __forceinline__ CamclSmem carve_camcl(double *p, int L, int fb)
{
    CamclSmem s;
    s.L   = L;
    s.Pe1 = p, p += L;
    for (int k = 0; k < 2; ++k) {
        s.Bcov[k] = p, p += 3 * L;
        s.Bcon[k] = p, p += 3 * L;
    }
    s.Bavg = p, p += 3 * L;
    s.items = p, p += FS_ITEM_L * L * fb;
    s.gh = p;
    return s;
}

// stage the raw deposit arrays r[0..3] of item j: this cell into ta (n) / tv (nV), and the six
// ghost-fold partners r[-3..-1], r[Nx..Nx+2] of every quantity into gh (threads 0..23)
__device__ __forceinline__ void stage_raw(FieldArgs const &a, Cell const &C, CamclSmem const &S, int j,
                                          double const *const (&r)[4])
{
    int const t = C.t;
    S.ta(j)[t]  = __ldg(r[0] + C.gm);
#pragma unroll
    for (int q = 1; q < 4; ++q)
        S.tv(j)[3 * t + q - 1] = __ldg(r[q] + C.gm);
    if (t < 24) {
        int const q = t / 6, k = t % 6;
        S.gh[(j * 4 + q) * 6 + k] = __ldg(r[q] + (k < 3 ? k - 3 : a.Nx + k - 3));
    }
}
// fold of staged quantity q of item j onto interior cell gm, as fold() computes it from the raw array
__device__ __forceinline__ double fold_staged(FieldArgs const &a, Cell const &C, CamclSmem const &S, int j, int q,
                                              double s1, double f, double const *eq)
{
    int const     gm = C.gm, Nx = a.Nx;
    double const *g  = S.gh + (j * 4 + q) * 6; // g[0..2] = r[-3..-1], g[3..5] = r[Nx..Nx+2]
    double        m  = (q == 0 ? S.ta(j)[C.t] : S.tv(j)[3 * C.t + q - 1]) * s1;
    if (eq)
        m = m + eq[gm] * 1.0;
    double v = m * f;
    if (a.bc == 0) {
        if (gm < PAD)
            v = v + (g[3 + gm] * s1) * f;
        if (gm >= Nx - PAD)
            v = v + (g[gm - Nx + 3] * s1) * f;
    } else {
        if (gm == 0)
            v = v + ((g[2] * s1) * f + ((g[1] * s1) * f + (g[0] * s1) * f));
        if (gm == Nx - 1)
            v = v + ((g[3] * s1) * f + ((g[4] * s1) * f + (g[5] * s1) * f));
    }
    return v;
}

// nsm_of(j) smoothings of item j's arrays (a, v) for every j < n together (most = the largest
// count), ping-ponging with (ta, tv); with_scalar = false smooths the vectors only.  Item j's result
// is in (a, v) when its count is even and in (ta, tv) when it is odd.  The items are visited by a
// loop, not unrolled: the kernel is latency-bound and its code must stay small.  Ends synchronised.
template <class NsmOf>
__device__ __forceinline__ void smooth_group(Cell const &C, CamclSmem const &S, int n, NsmOf const &nsm_of, int most,
                                             bool with_scalar)
{
    int const tl = max(C.t - 1, 0), tr = min(C.t + 1, C.L - 1), t = C.t;
    for (int it = 0; it < most; ++it) {
        __syncthreads();
        bool const odd = it & 1;
#pragma unroll 1
        for (int j = 0; j < n; ++j) {
            if (it >= nsm_of(j))
                continue;
            double const *a  = odd ? S.ta(j) : S.a(j);
            double       *ta = odd ? S.a(j) : S.ta(j);
            double const *v  = odd ? S.tv(j) : S.v(j);
            double       *tv = odd ? S.v(j) : S.tv(j);
            if (with_scalar)
                ta[t] = (a[tl] + 2 * a[t] + a[tr]) * .25;
#pragma unroll
            for (int k = 0; k < 3; ++k)
                tv[3 * t + k] = (v[3 * tl + k] + 2 * v[3 * t + k] + v[3 * tr + k]) * .25;
        }
    }
    __syncthreads();
}
__device__ __forceinline__ double const *smoothed_a(CamclSmem const &S, int j, int nsm) { return nsm & 1 ? S.ta(j) : S.a(j); }
__device__ __forceinline__ double const *smoothed_v(CamclSmem const &S, int j, int nsm) { return nsm & 1 ? S.tv(j) : S.v(j); }

// one source item of the CAM-CL cycle: kinetic species s at deposit d, cold species c, or
// external source e (their order is the reference's accumulation order)
struct SrcItem {
    int kind, idx, d; // kind 0 kinetic, 1 cold, 2 external
};
__device__ __forceinline__ SrcItem src_item(FieldArgs const &a, int i)
{
    if (i < 2 * a.nk)
        return { 0, i >> 1, i & 1 };
    i -= 2 * a.nk;
    if (i < a.nc)
        return { 1, i, 0 };
    return { 2, i - a.nc, 0 };
}
__device__ __forceinline__ int src_nsm(FieldArgs const &a, SrcItem const &it)
{
    return it.kind == 0 ? a.k[it.idx].nsm : it.kind == 1 ? a.c[it.idx].nsm : a.e[it.idx].nsm;
}
// the smoothing count of item s of the current advance (kinetic species, cold species, external sources)
__device__ __forceinline__ int adv_nsm(FieldArgs const &a, int s)
{
    return s < a.nk ? a.k[s].nsm : s < a.nk + a.nc ? a.c[s - a.nk].nsm : a.e[s - a.nk - a.nc].nsm;
}

// ------------------------------------------------------------------------------------------------
// CAM-CL cycle (Domain_CAMCL.cc:57-193)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void camcl_field_body(FieldArgs const &a, int blk)
{
    extern __shared__ double sm[];
    Cell C;
    load_cell(a, C, blk);
    CamclSmem const S = carve_camcl(sm, C.L, a.fb);
    int const       t = C.t, Nx = a.Nx, L = C.L;

    // the deposits of a group of source items into shared memory (kinetic and external ones; the
    // loop is unrolled by four so that their loads are in flight together)
    int const  n_src     = 2 * a.nk + a.nc + a.ne;
    auto const stage_src = [&](int i0) {
        int const n = min(a.fb, n_src - i0);
#pragma unroll 4
        for (int j = 0; j < n; ++j) {
            SrcItem const it = src_item(a, i0 + j);
            if (it.kind == 0)
                stage_raw(a, C, S, j, a.k[it.idx].raw[it.d]);
            else if (it.kind == 2)
                stage_raw(a, C, S, j, a.e[it.idx].raw[0]);
        }
    };
    stage_src(0); // before the cold push, so that the two rounds of loads overlap

    d3 const Bn = ld3(a.B_in, C.gm);
    d3       cold_nV[MAXC];
    double   cold_n[MAXC]; // mom0_full of each cold species at this cell, read once
    for (int ci = 0; ci < a.nc; ++ci) {
        cold_n[ci]  = a.c[ci].n[C.gm];
        cold_nV[ci] = cold_push(a, C, a.c[ci], a.E_in);
    }

    // 1-2. sources at x^N and x^{N+1}, every species' collect_smooth in groups
    double rho0 = 0, rho1 = 0;
    d3     J0 = { 0, 0, 0 }, J1 = { 0, 0, 0 };
    for (int i0 = 0; i0 < n_src; i0 += a.fb) {
        int const  n      = min(a.fb, n_src - i0);
        auto const nsm_of = [&](int j) { return src_nsm(a, src_item(a, i0 + j)); };
        int        most   = 0;
        if (i0 > 0) // the first group was staged above
            stage_src(i0);
#pragma unroll 1
        for (int j = 0; j < n; ++j) { // a cold species' sources need no neighbour: formed directly
            SrcItem const it = src_item(a, i0 + j);
            most             = max(most, src_nsm(a, it));
            if (it.kind == 1) {
                ColdSrc const &K = a.c[it.idx];
                S.a(j)[t]        = (cold_n[it.idx] * K.w) * K.cdcf;
                sst3(S.v(j), t, (cold_nV[it.idx] * K.w) * K.ccf);
            }
        }
        __syncthreads();
#pragma unroll 1
        for (int j = 0; j < n; ++j) {
            SrcItem const it = src_item(a, i0 + j);
            if (it.kind != 1) {
                KinSrc const &K = it.kind == 0 ? a.k[it.idx] : a.e[it.idx];
                S.a(j)[t]       = fold_staged(a, C, S, j, 0, K.s1, K.cdcf, K.eq);
#pragma unroll
                for (int q = 0; q < 3; ++q)
                    S.v(j)[3 * t + q] = fold_staged(a, C, S, j, 1 + q, K.s1, K.ccf, nullptr);
            }
        }
        smooth_group(C, S, n, nsm_of, most, true);
#pragma unroll 1
        for (int j = 0; j < n; ++j) {
            SrcItem const it  = src_item(a, i0 + j);
            int const     nsm = src_nsm(a, it);
            double const  r   = smoothed_a(S, j, nsm)[t];
            d3 const      v   = sld3(smoothed_v(S, j, nsm), t);
            if (it.kind == 0 && it.d == 1) {
                J1 = J1 + v;
                rho1 += r;
            } else if (it.kind == 0) {
                J0 = J0 + v;
                rho0 += r;
            } else { // cold and external sources enter both
                J0 = J0 + v;
                rho0 += r;
                J1 = J1 + v;
                rho1 += r;
            }
        }
    }
    // the first group of the current advance (step 5) is staged now, so that its loads complete
    // during the subcycle (a thread's staging writes only its own cell of the items, which it
    // has read above, and the ghost partners, which no one reads any more)
    int const  n_adv     = a.nk + a.nc + a.ne;
    auto const stage_adv = [&](int i0) {
        int const n = min(a.fb, n_adv - i0);
#pragma unroll 4
        for (int j = 0; j < n; ++j) {
            int const s = i0 + j;
            if (s < a.nk || s >= a.nk + a.nc)
                stage_raw(a, C, S, j, (s < a.nk ? a.k[s] : a.e[s - a.nk - a.nc]).raw[1]);
        }
    };
    stage_adv(0);

    // 3. averages
    // (the pressure gradient at rho_avg enters only the x component of the subcycle's E, which
    // Faraday's law does not read, so only the one at rho^{N+1} is formed)
    double const rho_avg = (rho0 + rho1) * .5;
    d3 const     J_avg   = (J0 + J1) * .5;
    S.Pe1[t]             = Pe_of(a, rho1);
    sst3(S.Bcov[0], t, covar_full(C, Bn));
    sst3(S.Bcon[0], t, contr_full(C, Bn));
    __syncthreads();
    double const dPe1 = dPe_at(a, C, S.Pe1);
    d3 const     jc   = contr_half(C, J_avg);

    // 4. subcycle: E at every cell (its covariant y and z components are exchanged through Bavg,
    // free until the average), then Faraday's law from E at this cell and the one before; Ohm's
    // law reads only the y and z components of the covariant B
    double const inv_rho = 1.0 / rho_avg;
    int const    tm      = max(t - 1, 0);
    d3 X = Bn, Y = Bn; // X is updated, Y holds the newest B
    for (int i = 0; i <= a.m; ++i) {
        int const    p    = i & 1;
        d3 const     Ec   = covar_half(C, E_sub(a, C, t, L, S.Bcov[p], S.Bcon[p], jc, inv_rho));
        S.Bavg[2 * t]     = Ec.y;
        S.Bavg[2 * t + 1] = Ec.z;
        __syncthreads();
        d3 const     Em   = { 0.0, S.Bavg[2 * tm], S.Bavg[2 * tm + 1] };
        double const dtp  = (i == 0 || i == a.m) ? a.sub_dt : 2.0 * a.sub_dt;
        d3 const     Bnew = B_at_e(a, C, Ec, Em, X, dtp);
        X                 = Bnew;
        S.Bcov[1 - p][3 * t + 1] = C.fcy * Bnew.y;
        S.Bcov[1 - p][3 * t + 2] = C.fcz * Bnew.z;
        sst3(S.Bcon[1 - p], t, contr_full(C, Bnew));
        __syncthreads();
        d3 const tmp = X; // the older one is updated next
        X            = Y;
        Y            = tmp;
    }
    // after the loop Y is b0 (updated last) and X is b1; average into B
    int const pb   = (a.m + 1) & 1; // the buffer nobody reads any more
    d3 const  Bavg = (Y + X) * .5;
    sst3(S.Bavg, t, Bavg);
    sst3(S.Bcov[pb], t, covar_full(C, Bavg));
    sst3(S.Bcon[pb], t, contr_full(C, Bavg));
    __syncthreads();

    // 5. E* from (B, rho^{N+1}, J^{N+1/2})
    d3 const Es = E_at_g(a, C, t, L, S.Bcov[pb], S.Bcon[pb], jc, dPe1, rho1);
    // current advance (Domain_CAMCL.cc:131-151, Current.cc:45-52)
    d3 const  Bnext = sld3(S.Bavg, min(t + 1, L - 1));
    d3 const  Bi    = { C.hbx + (Bnext.x + Bavg.x) * 0.5, 0 * a.O0 + (Bnext.y + Bavg.y) * 0.5,
                        0 * a.O0 + (Bnext.z + Bavg.z) * 0.5 };
    for (int i0 = 0; i0 < n_adv; i0 += a.fb) {
        int const  n      = min(a.fb, n_adv - i0);
        auto const nsm_of = [&](int j) { return adv_nsm(a, i0 + j); };
        int        most   = 0;
#pragma unroll 1
        for (int j = 0; j < n; ++j)
            most = max(most, adv_nsm(a, i0 + j));
        if (i0 > 0) { // the first group was staged before the subcycle
            stage_adv(i0);
            __syncthreads();
        }
#pragma unroll 1
        for (int j = 0; j < n; ++j) {
            int const s = i0 + j;
            double    lam;
            d3        gam;
            if (s < a.nk || s >= a.nk + a.nc) {
                KinSrc const &K = s < a.nk ? a.k[s] : a.e[s - a.nk - a.nc];
                lam             = fold_staged(a, C, S, j, 0, K.s1, K.lamf, K.eq);
                gam             = { fold_staged(a, C, S, j, 1, K.s1, K.gamf, nullptr),
                                    fold_staged(a, C, S, j, 2, K.s1, K.gamf, nullptr),
                                    fold_staged(a, C, S, j, 3, K.s1, K.gamf, nullptr) };
            } else {
                ColdSrc const &K = a.c[s - a.nk];
                lam              = (cold_n[s - a.nk] * K.w) * K.lamf;
                gam              = (cold_nV[s - a.nk] * K.w) * K.gamf;
            }
            d3 const Jadv = (Es * lam + cross(gam, Bi)) * (0.5 * a.dt);
            sst3(S.v(j), t, { 0 + Jadv.x, 0 + Jadv.y, 0 + Jadv.z });
        }
        smooth_group(C, S, n, nsm_of, most, false);
#pragma unroll 1
        for (int j = 0; j < n; ++j)
            J1 = J1 + sld3(smoothed_v(S, j, adv_nsm(a, i0 + j)), t);
    }
    // 6. E from (B, rho^{N+1}, J^+ advanced)
    d3 const Ef = E_at_g(a, C, t, L, S.Bcov[pb], S.Bcon[pb], contr_half(C, J1), dPe1, rho1);

    if (C.owner) {
        put3(a.B_out, C, Nx, Bavg);
        put3(a.E_out, C, Nx, Ef);
        put1(a.charge_out, C, Nx, rho_avg);
        put3(a.current_out, C, Nx, J_avg);
        d3 const Bh = (Bnext + Bavg) * 0.5;
        put_eb(a.EB_out, a.EBf_out, C, Nx, Ef, Bh);
        for (int ci = 0; ci < a.nc; ++ci)
            st3(a.c[ci].nV_out, C.gm, cold_nV[ci]);
        // clear the deposit set of the next cycle (interior + ghost images)
        for (int s = 0; s < a.nk; ++s)
            for (int d = 0; d < 2; ++d)
                for (int q = 0; q < 4; ++q)
                    put1(a.k[s].zero[d][q], C, Nx, 0.0);
    }
}


// ------------------------------------------------------------------------------------------------
// predictor-corrector phases (Domain_PC.cc:21-205)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void pc_field_body(FieldArgs const &a, int blk)
{
    extern __shared__ double sm[];
    Cell C;
    load_cell(a, C, blk);
    Smem const S = carve(sm, C.L);
    int const  t = C.t, Nx = a.Nx, ph = a.phase;

    // sources: kinetic species (deposit at the end position), then cold species
    double rho = 0;
    d3     J   = { 0, 0, 0 };
    if (ph != 1) {
        for (int s = 0; s < a.nk; ++s) {
            SV const r = collect_kinetic(a, C, S, a.k[s], 1);
            rho += r.a[t];
            J = J + sld3(r.v, t);
        }
        for (int ci = 0; ci < a.nc; ++ci) {
            ColdSrc const &K = a.c[ci];
            d3             v;
            if (ph == 0)
                v = ld3(K.nV_in, C.gm);
            else if (ph == 2) // predictor copy pushed with the predicted fields (Domain_PC.cc:125-133)
                v = boris_push(K.boris, ld3(K.nV_in, C.gm), d3{ C.hbx, 0 * a.O0, 0 * a.O0 }, ld3(a.E1_in, C.gm) * K.n[C.gm]);
            else // corrector: the state pushed in phase 2
                v = ld3(K.nV_out, C.gm);
            S.tr[t] = (K.n[C.gm] * K.w) * K.cdcf;
            sst3(S.tJ, t, (v * K.w) * K.ccf);
            SV const r = smooth_n(C, K.nsm, S.tr, S.tJ, S.ts, S.tJs);
            rho += r.a[t];
            J = J + sld3(r.v, t);
        }
        for (int s = 0; s < a.ne; ++s) { // external sources (Domain_PC.cc:51-56, 134-140, 189-193)
            SV const r = collect_kinetic(a, C, S, a.e[s], 1);
            rho += r.a[t];
            J = J + sld3(r.v, t);
        }
    }
    if (ph == 0) {
        if (C.owner) {
            put1(a.charge_out, C, Nx, rho);
            put3(a.current_out, C, Nx, J);
            for (int s = 0; s < a.nk; ++s)
                for (int d = 0; d < 2; ++d)
                    for (int q = 0; q < 4; ++q)
                        put1(a.k[s].zero[d][q], C, Nx, 0.0);
        }
        return;
    }
    double const rho_src = ph == 1 ? a.charge_in[C.gm] : rho;
    d3 const     J_src   = ph == 1 ? ld3(a.current_in, C.gm) : J;
    d3 const     E0      = ld3(a.E_in, C.gm);
    d3 const     B0      = ld3(a.B_in, C.gm);
    d3 const     Eb      = ph == 1 ? E0 : ld3(a.E1_in, C.gm); // E driving Faraday's law
    sst3(S.Ecov, t, covar_half(C, Eb));
    S.Pe[t] = Pe_of(a, rho_src);
    __syncthreads();
    d3 const     Bn  = B_at(a, C, S.Ecov, B0, a.dt);
    double const dPe = dPe_at(a, C, S.Pe);
    sst3(S.Bcov, t, covar_full(C, Bn));
    sst3(S.Bcon, t, contr_full(C, Bn));
    __syncthreads();
    d3 const En = E_at(a, C, S.Bcov, S.Bcon, contr_half(C, J_src), dPe, rho_src);
    if (ph == 3) {
        if (C.owner) {
            put3(a.B_out, C, Nx, Bn);
            put3(a.E_out, C, Nx, En);
            put1(a.charge_out, C, Nx, rho_src);
            put3(a.current_out, C, Nx, J_src);
            for (int s = 0; s < a.nk; ++s)
                for (int d = 0; d < 2; ++d)
                    for (int q = 0; q < 4; ++q)
                        put1(a.k[s].zero[d][q], C, Nx, 0.0);
        }
        return;
    }
    d3 const B1a = (Bn + B0) * .5;
    d3 const E1a = (En + E0) * .5;
    sst3(S.B0, t, B1a);
    __syncthreads();
    d3 const Bh = (sld3(S.B0, min(t + 1, C.L - 1)) + B1a) * 0.5;
    if (C.owner) {
        put3(a.E1_out, C, Nx, E1a);
        put_eb(a.EB_out, a.EBf_out, C, Nx, E1a, Bh);
        if (ph == 2) {
            for (int ci = 0; ci < a.nc; ++ci) { // corrector push of the cold fluid (Domain_PC.cc:182-188)
                ColdSrc const &K = a.c[ci];
                st3(K.nV_out, C.gm, boris_push(K.boris, ld3(K.nV_in, C.gm), d3{ C.hbx, 0 * a.O0, 0 * a.O0 }, E1a * K.n[C.gm]));
            }
            for (int s = 0; s < a.nk; ++s)
                for (int d = 0; d < 2; ++d)
                    for (int q = 0; q < 4; ++q)
                        put1(a.k[s].zero[d][q], C, Nx, 0.0);
        }
    }
}

// one run: the arguments are kernel constants, block b covers segment b
__global__ void __launch_bounds__(512) camcl_field_kernel(FieldArgs const __grid_constant__ a) { camcl_field_body(a, blockIdx.x); }
__global__ void __launch_bounds__(512) pc_field_kernel(FieldArgs const __grid_constant__ a) { pc_field_body(a, blockIdx.x); }

// an ensemble: block b covers segment map[b].seg of run map[b].run, whose arguments it copies
// from the device table into shared memory
__device__ __forceinline__ void load_args(FieldArgs &dst, FieldArgs const *src)
{
    static_assert(sizeof(FieldArgs) % 8 == 0, "FieldArgs is copied in 8-byte words");
    auto const *s = reinterpret_cast<unsigned long long const *>(src);
    auto       *d = reinterpret_cast<unsigned long long *>(&dst);
    for (int i = threadIdx.x; i < static_cast<int>(sizeof(FieldArgs) / 8); i += blockDim.x)
        d[i] = s[i];
    __syncthreads();
}
__global__ void __launch_bounds__(512) camcl_field_batch_kernel(FieldArgs const *table, FieldBlock const *map)
{
    __shared__ FieldArgs a;
    FieldBlock const     b = map[blockIdx.x];
    load_args(a, table + b.run);
    camcl_field_body(a, b.seg);
}
__global__ void __launch_bounds__(512) pc_field_batch_kernel(FieldArgs const *table, FieldBlock const *map)
{
    __shared__ FieldArgs a;
    FieldBlock const     b = map[blockIdx.x];
    load_args(a, table + b.run);
    pc_field_body(a, b.seg);
}

#endif // H1D_FIELD_TU

} // namespace h1d
