/*
 * snow_oracle.c -- CPU restatement of the SnowSimulation substep (TEST INFRASTRUCTURE).
 *
 * Checker only: tests/, __graft_entry__.smoke() and bench.py's CPU baseline load
 * it; the CUDA library never does.  Every function cites the reference lines it
 * restates (cuda_simulation.cu unless another file is named).
 *
 * Arithmetic contract shared with the CUDA kernels (so FP32 parity is bit-exact):
 *   - every expression is evaluated as the reference writes it, left to right, each
 *     operation rounded separately (dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z as in
 *     helper_math.h, length(v) = sqrt(dot(v,v))); no fused multiply-add anywhere
 *     (build with -ffp-contract=off, never -ffast-math);
 *   - sqrt and division are IEEE correctly rounded;
 *   - every neighbor sum is accumulated per cell (cells in z,y,x order, particles
 *     in ascending sorted index) and the cell partial is added to the running total,
 *     exactly the structure of the reference's per-cell helper functions;
 *   - float -> int conversions saturate as CUDA's cvt.rzi does (NaN -> 0).
 *
 * Where the reference is racy, this file fixes one canonical order (the CUDA path
 * produces the same result):
 *   - XSPH (Q5, :3504-3660) is Jacobi: every read sees the pre-kernel velocities;
 *   - freezing/melting (Q8, :4387-4449) assign target slots in ascending source index;
 *   - link formation (Q10, :4127-4284) runs sequentially in "colour order": hash cells
 *     are grouped in 2x2x2 super-cells, super-cells get one of 8 colours from the
 *     parity of their coordinates, colours are processed 0..7 and inside a colour the
 *     particles in ascending sorted index.  Same-coloured super-cells are >= 3 cells
 *     apart, so their link edits never touch the same particle and any interleaving of
 *     them gives this result;
 *   - adjust_connections (:4768-4808) runs sequentially in ascending index;
 *   - interlink breaking (Q4, :4624-4765) needs no rule: both ends of a link see the
 *     same length and distance, so the result does not depend on the order.
 */
#include "snow_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORACLE_DOUBLE
#define RFMA fma
#define RSQRT sqrt
#define RFLOOR floor
#define RFABS fabs
#define RFMIN fmin
#else
#define RFMA fmaf
#define RSQRT sqrtf
#define RFLOOR floorf
#define RFABS fabsf
#define RFMIN fminf
#endif

#define EMPTY 0xFFFFFFFFu
#define UMAX 0xFFFFFFFFu
#define R(x) ((real)(x))

int or_real_size(void) { return (int)sizeof(real); }

static float g_dom[5] = {-1.f, 1.f, -1.f, 1.f, 0.f};   /* walls x, z and floor y (the reference: +-1, 0) */
void or_set_domain(float x_min, float x_max, float z_min, float z_max, float floor_y)
{
    g_dom[0] = x_min; g_dom[1] = x_max; g_dom[2] = z_min; g_dom[3] = z_max; g_dom[4] = floor_y;
}
void or_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------ vectors */
static inline r3 v3(real x, real y, real z) { r3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline r3 vadd(r3 a, r3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline r3 vsub(r3 a, r3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline r3 vsc(real s, r3 a) { return v3(s * a.x, s * a.y, s * a.z); }
static inline r3 vdivs(r3 a, real s) { return v3(a.x / s, a.y / s, a.z / s); }
static inline real vdot(r3 a, r3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline real vlen(r3 a) { return RSQRT(vdot(a, a)); }
static inline int vnan(r3 a) { return isnan(a.x) || isnan(a.y) || isnan(a.z); }
static inline int vinf(r3 a) { return isinf(a.x) || isinf(a.y) || isinf(a.z); }
static const r3 ZERO3 = {0, 0, 0};

/* --------------------------------------------------------------- constants */
typedef struct {
    real h, r, two_r, poly6, poly6_G, spiky, spiky_G, visc_lap;
    real keps, pbd_eps, rho0, inv_rho0, eps, scorr_coeff, scorr_div;
    real g[3], damping, max_speed, min_speed, b_damping, mu_s, mu_k, k_stretch;
    real k_water, k_snow, C_water, C_snow, Tf, blending, sor, sph_visc, dem_visc;
    real Th, k_ref, brk;
    real origin[3], cell[3];
    uint32_t gs[3], ncells, maxc;
} K;

static K mk(const or_params* P)
{
    K k;
    k.h = R(P->effective_radius); k.r = R(P->particle_radius);
    k.two_r = R(2.0f) * k.r;
    k.poly6 = R(P->poly6); k.poly6_G = R(P->poly6_G); k.spiky = R(P->spiky);
    k.spiky_G = R(P->spiky_G); k.visc_lap = R(P->viscosity_laplacian);
    k.keps = R(P->kernel_epsilon); k.pbd_eps = R(P->pbd_epsilon);
    k.rho0 = R(P->rest_density); k.inv_rho0 = R(1.0f) / k.rho0; k.eps = R(P->epsilon);
    k.scorr_coeff = R(P->scorr_coeff); k.scorr_div = R(P->scorr_divisor);
    for (int i = 0; i < 3; i++) {
        k.g[i] = R(P->gravity[i]); k.origin[i] = R(P->world_origin[i]);
        k.cell[i] = R(P->cell_size[i]); k.gs[i] = P->grid_size[i];
    }
    k.damping = R(P->global_damping); k.max_speed = R(P->maximum_speed);
    k.min_speed = R(P->minimum_speed); k.b_damping = R(P->boundary_damping);
    k.mu_s = R(P->static_friction); k.mu_k = R(P->kinematic_friction);
    k.k_stretch = R(P->k_stretch); k.k_water = R(P->k_water); k.k_snow = R(P->k_snow);
    k.C_water = R(P->C_water); k.C_snow = R(P->C_snow); k.Tf = R(P->freezing_point);
    k.blending = R(P->blending_speed); k.sor = R(P->sor_coeff);
    k.sph_visc = R(P->sph_viscosity); k.dem_visc = R(P->dem_viscosity);
    k.Th = R(P->T_homogeneous); k.k_ref = R(P->k_refreezing); k.brk = R(P->break_threshold);
    k.ncells = P->num_cells; k.maxc = P->maximum_connection;
    return k;
}

/* ----------------------------------------------------------- SPH kernels :30-137 */
static inline real W_poly6(const K* k, real d)
{
    if (d >= 0 && d < k->h) {
        real h2 = k->h * k->h, d2 = d * d, q = h2 - d2;
        real q3 = q * q * q;
        return k->poly6 * q3;
    }
    return 0;
}
static inline r3 G_poly6(const K* k, r3 diff, real d)
{
    if (d >= 0 && d < k->h) {
        real h2 = k->h * k->h, d2 = d * d, q = h2 - d2, q2 = q * q;
        real s = k->poly6_G * q2;
        return vsc(s, diff);
    }
    return ZERO3;
}
static inline r3 G_spiky(const K* k, r3 diff, real d)
{
    if (d >= 0 && d < k->h) {
        real q = k->h - d, q2 = q * q;
        real s = k->spiky_G * (q2 / (d + k->keps));
        return vsc(s, diff);
    }
    return ZERO3;
}
static inline real L_visc(const K* k, real d)
{
    if (d >= 0 && d < k->h) return k->visc_lap * (k->h - d);
    return 0;
}

/* ------------------------------------------------------------ grid :141-157 */
static inline int32_t cvt_s32(real x)
{
    if (x != x) return 0;
    if (x >= R(2147483648.0)) return INT32_MAX;
    if (x < R(-2147483648.0)) return INT32_MIN;
    return (int32_t)x;
}
static inline uint32_t cvt_u32(real x)
{
    if (x != x) return 0;
    if (x <= R(0)) return 0;
    if (x >= R(4294967296.0)) return UMAX;
    return (uint32_t)x;
}
typedef struct { int32_t x, y, z; } i3;
static inline i3 gpos(const K* k, r3 p)
{
    i3 g;
    g.x = cvt_s32(RFLOOR((p.x - k->origin[0]) / k->cell[0]));
    g.y = cvt_s32(RFLOOR((p.y - k->origin[1]) / k->cell[1]));
    g.z = cvt_s32(RFLOOR((p.z - k->origin[2]) / k->cell[2]));
    return g;
}
/* hash of grid cell g + (dx,dy,dz), wrapped per axis (int add wraps like CUDA) */
static inline uint32_t ghash(const K* k, i3 g, int dx, int dy, int dz)
{
    uint32_t x = ((uint32_t)g.x + (uint32_t)dx) & (k->gs[0] - 1u);
    uint32_t y = ((uint32_t)g.y + (uint32_t)dy) & (k->gs[1] - 1u);
    uint32_t z = ((uint32_t)g.z + (uint32_t)dz) & (k->gs[2] - 1u);
    return (z * k->gs[1]) * k->gs[0] + y * k->gs[0] + x;
}
/* cell range [s,e) of a neighbor cell; 0 when the cell is marked empty */
static inline int crange(const K* k, const or_cells* cd, i3 g, int dx, int dy, int dz,
                         uint32_t* s, uint32_t* e)
{
    uint32_t h = ghash(k, g, dx, dy, dz);
    uint32_t st = cd->cell_start[h];
    if (st == EMPTY) return 0;
    *s = st; *e = cd->cell_end[h];
    return 1;
}
#define FOR27 for (int oz = -1; oz <= 1; oz++) for (int oy = -1; oy <= 1; oy++) for (int ox = -1; ox <= 1; ox++)

/* launch coverage of compute_grid_size(n, 512) (:348-357) */
static inline uint32_t coverage(uint32_t n)
{
    if (n == 0) return 0;
    uint32_t t = n < 512u ? n : 512u;
    uint32_t b = (n % t) ? n / t + 1 : n / t;
    return b * t;
}
static inline uint32_t umin(uint32_t a, uint32_t b) { return a < b ? a : b; }

/* ------------------------------------------------ hash / sort / reorder :194-420 */
void or_calculate_hash(const or_params* P, or_cells cd, const r3* pos, uint32_t n)
{
    K k = mk(P);
    for (uint32_t i = 0; i < n; i++) {
        i3 g = gpos(&k, pos[i]);
        cd.grid_hash[i] = ghash(&k, g, 0, 0, 0);
        cd.grid_index[i] = i;
    }
}

/* thrust::sort_by_key is stable: LSD radix on 32-bit keys (:1455-1468) */
void or_sort_particles(or_cells cd, uint32_t n)
{
    if (n < 2) return;
    uint32_t* k2 = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* v2 = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t* ka = cd.grid_hash; uint32_t* va = cd.grid_index;
    uint32_t* kb = k2; uint32_t* vb = v2;
    for (int pass = 0; pass < 4; pass++) {
        uint32_t cnt[257];
        memset(cnt, 0, sizeof(cnt));
        int sh = 8 * pass;
        for (uint32_t i = 0; i < n; i++) cnt[((ka[i] >> sh) & 255u) + 1]++;
        for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
        for (uint32_t i = 0; i < n; i++) {
            uint32_t b = (ka[i] >> sh) & 255u;
            kb[cnt[b]] = ka[i]; vb[cnt[b]] = va[i]; cnt[b]++;
        }
        uint32_t* t;
        t = ka; ka = kb; kb = t;
        t = va; va = vb; vb = t;
    }
    /* after 4 passes the data is back in the caller's arrays */
    free(k2); free(v2);
}

void or_reorder_data(or_cells cd, const r3* pos, uint32_t n, uint32_t num_cells)
{
    for (uint32_t c = 0; c < num_cells; c++) cd.cell_start[c] = EMPTY;
    for (uint32_t i = 0; i < n; i++) {
        uint32_t h = cd.grid_hash[i];
        if (i == 0 || h != cd.grid_hash[i - 1]) {
            cd.cell_start[h] = i;
            if (i > 0) cd.cell_end[cd.grid_hash[i - 1]] = i;
        }
        if (i == n - 1) cd.cell_end[h] = i + 1;
        cd.sorted_pos[i] = pos[cd.grid_index[i]];
    }
}

/* sort_and_reorder (:398-420); Q1: the reference clears only num_particles cells */
static void sort_and_reorder(const or_params* P, const K* k, r3* pos, or_cells cd, uint32_t n, int quirks)
{
    if (n == 0) return;
    or_calculate_hash(P, cd, pos, n);
    or_sort_particles(cd, n);
    uint32_t nc = quirks == OR_QUIRKS_FIXED ? k->ncells : umin(n, k->ncells);
    or_reorder_data(cd, pos, n, nc);
}

/* ------------------------------------------------ boundary volume :159-192, :303-346 */
void or_compute_boundary_volume(const or_params* P, or_cells cd, const real* mass, real* volume, uint32_t n)
{
    K k = mk(P);
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)n; ii++) {
        uint32_t i = (uint32_t)ii;
        uint32_t o = cd.grid_index[i];
        r3 p = cd.sorted_pos[i];
        real rho = mass[o] * W_poly6(&k, 0);
        i3 g = gpos(&k, p);
        FOR27 {
            uint32_t s, e; real cs = 0;
            if (crange(&k, &cd, g, ox, oy, oz, &s, &e))
                for (uint32_t j = s; j < e; j++)
                    if (j != i) cs += mass[cd.grid_index[j]] * W_poly6(&k, vlen(vsub(p, cd.sorted_pos[j])));
            rho += cs;
        }
        volume[o] = mass[o] / rho;
    }
}

/* ------------------------------------------------------------ per-cell sums */
/* sum over 27 cells of mass_j * W(d)   (pbf_density_0 :543-582 with skip,
   pbf_boundary_density_coupling :668-707 without) */
static real acc_massW(const K* k, real acc, const or_cells* cd, const real* mass,
                      r3 p, i3 g, uint32_t skip)
{
    FOR27 {
        uint32_t s, e; real cs = 0;
        if (crange(k, cd, g, ox, oy, oz, &s, &e))
            for (uint32_t j = s; j < e; j++) {
                if (j == skip) continue;
                cs += mass[cd->grid_index[j]] * W_poly6(k, vlen(vsub(p, cd->sorted_pos[j])));
            }
        acc += cs;
    }
    return acc;
}
/* sum of (rho0*V_j) * W(d)   (pbf_density_1 :585-625 with skip,
   pbf_density_coupling_vol :628-665 without) */
static real acc_volW(const K* k, real acc, const or_cells* cd, const real* vol,
                     r3 p, i3 g, uint32_t skip)
{
    FOR27 {
        uint32_t s, e; real cs = 0;
        if (crange(k, cd, g, ox, oy, oz, &s, &e))
            for (uint32_t j = s; j < e; j++) {
                if (j == skip) continue;
                cs += (k->rho0 * vol[cd->grid_index[j]]) * W_poly6(k, vlen(vsub(p, cd->sorted_pos[j])));
            }
        acc += cs;
    }
    return acc;
}
/* lambda denominators (pbf_lambda_0 :711-751, pbf_boundary_lambda :846-881,
   pbf_lambda_boundary :804-843, pbf_lambda_1 :754-801).
   mode 0: s = 1/rho0; mode 1: s = (1/rho0)*((rho0*V_j)/m_self);
   mode 2: s = (1/rho0)*((rho0*V_j)/m_j) */
static real acc_gradsq(const K* k, real acc, const or_cells* cd, r3 p, i3 g, uint32_t skip,
                       int mode, const real* vol, const real* mass_j, real m_self)
{
    FOR27 {
        uint32_t s, e; real cs = 0;
        if (crange(k, cd, g, ox, oy, oz, &s, &e))
            for (uint32_t j = s; j < e; j++) {
                if (j == skip) continue;
                r3 v = vsub(p, cd->sorted_pos[j]);
                real d = vlen(v);
                real sc;
                if (mode == 0) sc = k->inv_rho0;
                else {
                    uint32_t oj = cd->grid_index[j];
                    real m = mode == 1 ? m_self : mass_j[oj];
                    sc = k->inv_rho0 * ((k->rho0 * vol[oj]) / m);
                }
                r3 gc = vsc(sc, G_spiky(k, v, d));
                cs += vdot(gc, gc);
            }
        acc += cs;
    }
    return acc;
}

static inline real scorr_of(const K* k, real d, float dt)
{
    real x = W_poly6(k, d) / k->scorr_div;
    real x4 = (x * x) * (x * x);
    return ((-k->scorr_coeff * x4) * R(dt)) * R(dt);
}

/* pbf_correction :883-929 -- same-set term with contrib_j, spiky gradient */
static r3 acc_pbf_own(const K* k, r3 acc, const or_cells* cd, r3 p, i3 g, uint32_t skip,
                      real lam_i, const real* lam, const real* contrib, float dt)
{
    FOR27 {
        uint32_t s, e; r3 cs = ZERO3;
        if (crange(k, cd, g, ox, oy, oz, &s, &e))
            for (uint32_t j = s; j < e; j++) {
                if (j == skip) continue;
                uint32_t oj = cd->grid_index[j];
                r3 v = vsub(p, cd->sorted_pos[j]);
                real d = vlen(v);
                r3 gr = G_spiky(k, v, d);
                real sc = scorr_of(k, d, dt);
                cs = vadd(cs, vsc(contrib[oj] * ((lam_i + lam[oj]) + sc), gr));
            }
        acc = vadd(acc, cs);
    }
    return acc;
}
/* pbf_correction_boundary :932-979 */
static r3 acc_pbf_bnd(const K* k, r3 acc, const or_cells* cd, r3 p, i3 g,
                      real lam_i, const real* lam, float dt)
{
    FOR27 {
        uint32_t s, e; r3 cs = ZERO3;
        if (crange(k, cd, g, ox, oy, oz, &s, &e))
            for (uint32_t j = s; j < e; j++) {
                uint32_t oj = cd->grid_index[j];
                r3 v = vsub(p, cd->sorted_pos[j]);
                real d = vlen(v);
                r3 gr = G_spiky(k, v, d);
                real sc = scorr_of(k, d, dt);
                cs = vadd(cs, vsc((lam_i + lam[oj]) + sc, gr));
            }
        acc = vadd(acc, cs);
    }
    return acc;
}
/* pbf_correction_coupling :982-1034.  Reference quirks: the self-skip compares a
   sorted index of the other set with this set's index, and s_corr reads an
   uninitialised variable (Q2) that is multiplied by scorr_coeff = 0; it is taken
   as 0.  quirks=fixed: no skip, s_corr as in the other terms. */
static r3 acc_pbf_cpl(const K* k, r3 acc, const or_cells* cd, r3 p, i3 g, uint32_t skip,
                      real lam_i, const real* lam, float dt, int quirks)
{
    FOR27 {
        uint32_t s, e; r3 cs = ZERO3;
        if (crange(k, cd, g, ox, oy, oz, &s, &e))
            for (uint32_t j = s; j < e; j++) {
                if (quirks == OR_QUIRKS_REFERENCE && j == skip) continue;
                uint32_t oj = cd->grid_index[j];
                r3 v = vsub(p, cd->sorted_pos[j]);
                real d = vlen(v);
                if (d <= k->two_r) {
                    r3 gr = G_poly6(k, v, d);
                    real x = W_poly6(k, d) / k->scorr_div;
                    real x4 = (x * x) * (x * x);
                    real sc = quirks == OR_QUIRKS_REFERENCE
                                  ? ((((-k->scorr_coeff) * R(0)) * x4) * R(dt)) * R(dt)
                                  : ((-k->scorr_coeff * x4) * R(dt)) * R(dt);
                    cs = vadd(cs, vsc((lam_i + lam[oj]) + sc, gr));
                }
            }
        acc = vadd(acc, cs);
    }
    return acc;
}
/* non-penetration (pbd_distance_correction_contrib :1470-1527 with skip,
   pbd_distance_correction_coupling_contrib :1648-1705 without) */
static r3 acc_contact(const K* k, r3 acc, const or_cells* cd, r3 p, i3 g, uint32_t skip,
                      real w0, const real* invm)
{
    FOR27 {
        uint32_t s, e; r3 cs = ZERO3;
        if (crange(k, cd, g, ox, oy, oz, &s, &e))
            for (uint32_t j = s; j < e; j++) {
                if (j == skip) continue;
                r3 v = vsub(p, cd->sorted_pos[j]);
                real d = vlen(v);
                if (d < k->two_r) {
                    real w1 = invm[cd->grid_index[j]];
                    real ws = w0 + w1;
                    real C = d - k->two_r;
                    r3 n = vdivs(v, d + k->pbd_eps);
                    cs = vadd(cs, vsc(((-w0) * (R(1) / ws)) * C, n));
                }
            }
        acc = vadd(acc, cs);
    }
    return acc;
}
/* pbd_sph_sph_distance_correction :1586-1646 (gated by contrib_i <= 0.99) */
static r3 acc_contact_sph(const K* k, r3 acc, const or_cells* cd, r3 p, i3 g, uint32_t skip,
                          real w0, real contrib_i, const real* invm)
{
    FOR27 {
        uint32_t s, e; r3 cs = ZERO3;
        if (crange(k, cd, g, ox, oy, oz, &s, &e))
            for (uint32_t j = s; j < e; j++) {
                if (j == skip) continue;
                if (!(contrib_i <= R(0.99f))) continue;
                r3 v = vsub(p, cd->sorted_pos[j]);
                real d = vlen(v);
                if (d < k->two_r) {
                    real w1 = invm[cd->grid_index[j]];
                    real ws = w0 + w1;
                    real C = d - k->two_r;
                    r3 n = vdivs(v, d + k->pbd_eps);
                    cs = vadd(cs, vsc(((-w0) * (R(1) / ws)) * C, n));
                }
            }
        acc = vadd(acc, cs);
    }
    return acc;
}
/* friction (pbd_friction_correction :1836-1918 own set, and
   pbd_friction_correction_boundary :1920-1987) */
static inline r3 friction_term(const K* k, r3 pp0, r3 op0, r3 pp1, r3 dx_extra, int own, real w0, real w1, real d, r3 v)
{
    real ws = w0 + w1;
    r3 n = vdivs(v, d + k->pbd_eps);
    real pen = k->two_r - d;
    r3 dx = vsub(pp0, op0);
    if (own) dx = vadd(dx, dx_extra);
    r3 dxt = vsub(dx, vsc(vdot(dx, n), n));
    real thr = k->mu_s * pen;
    real len = vlen(dxt);
    if (vlen(dxt) > thr) {
        real c = RFMIN((k->mu_k * pen) / (len + R(0.000001f)), R(1.f));
        dxt = vsc(c, dxt);
    }
    (void)pp1;
    return vsc(-(w0 / ws), dxt);
}

/* ------------------------------------------------------- stage: density :2219-2596 */
static void stage_density(const K* k, or_particles* sph, uint32_t ns, or_particles* dem, uint32_t nd,
                          or_particles* b, uint32_t nb, const or_cells* scd, const or_cells* dcd,
                          const or_cells* bcd)
{
    const real W0 = W_poly6(k, 0);
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)ns; ii++) {
        uint32_t i = (uint32_t)ii, o = scd->grid_index[i];
        r3 p = scd->sorted_pos[i]; i3 g = gpos(k, p);
        real rho = sph->mass[o] * W0;
        rho = acc_massW(k, rho, scd, sph->mass, p, g, i);
        rho = acc_massW(k, rho, dcd, dem->mass, p, g, UMAX);
        rho = acc_volW(k, rho, bcd, b->volume, p, g, UMAX);
        sph->density[o] = rho;
        sph->C[o] = (rho / k->rho0) - R(1) > 0 ? (rho / k->rho0) - R(1) : R(0);
    }
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)nd; ii++) {
        uint32_t i = (uint32_t)ii, o = dcd->grid_index[i];
        r3 p = dcd->sorted_pos[i]; i3 g = gpos(k, p);
        real rho = dem->mass[o] * W0;
        rho = acc_massW(k, rho, dcd, dem->mass, p, g, i);
        rho = acc_massW(k, rho, scd, sph->mass, p, g, UMAX);
        rho = acc_volW(k, rho, bcd, b->volume, p, g, UMAX);
        dem->density[o] = rho;
        dem->C[o] = (rho / k->rho0) - R(1) > 0 ? (rho / k->rho0) - R(1) : R(0);
    }
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)nb; ii++) {
        uint32_t i = (uint32_t)ii, o = bcd->grid_index[i];
        r3 p = bcd->sorted_pos[i]; i3 g = gpos(k, p);
        real rho = (k->rho0 * b->volume[o]) * W0;
        rho = acc_volW(k, rho, bcd, b->volume, p, g, i);
        rho = acc_massW(k, rho, dcd, dem->mass, p, g, UMAX);
        rho = acc_massW(k, rho, scd, sph->mass, p, g, UMAX);
        b->density[o] = rho;
        b->C[o] = (rho / k->rho0) - R(1) > 0 ? (rho / k->rho0) - R(1) : R(0);
    }
}

/* ------------------------------------------------------- stage: lambdas :2598-2960 */
static void stage_lambda(const K* k, or_particles* sph, uint32_t ns, or_particles* dem, uint32_t nd,
                         or_particles* b, uint32_t nb, const or_cells* scd, const or_cells* dcd,
                         const or_cells* bcd)
{
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)ns; ii++) {
        uint32_t i = (uint32_t)ii, o = scd->grid_index[i];
        r3 p = scd->sorted_pos[i]; i3 g = gpos(k, p);
        real lam = -sph->C[o];
        real gs = vdot(ZERO3, ZERO3);
        gs = acc_gradsq(k, gs, scd, p, g, i, 0, NULL, NULL, 0);
        gs = acc_gradsq(k, gs, dcd, p, g, UMAX, 0, NULL, NULL, 0);
        gs = acc_gradsq(k, gs, bcd, p, g, UMAX, 1, b->volume, NULL, sph->mass[o]);
        sph->lambda[o] = lam / (gs + k->eps);
    }
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)nd; ii++) {
        uint32_t i = (uint32_t)ii, o = dcd->grid_index[i];
        r3 p = dcd->sorted_pos[i]; i3 g = gpos(k, p);
        real lam = -dem->C[o];
        real gs = vdot(ZERO3, ZERO3);
        gs = acc_gradsq(k, gs, dcd, p, g, i, 0, NULL, NULL, 0);
        gs = acc_gradsq(k, gs, scd, p, g, UMAX, 0, NULL, NULL, 0);
        gs = acc_gradsq(k, gs, bcd, p, g, UMAX, 1, b->volume, NULL, dem->mass[o]);
        dem->lambda[o] = lam / (gs + k->eps);
    }
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)nb; ii++) {
        uint32_t i = (uint32_t)ii, o = bcd->grid_index[i];
        r3 p = bcd->sorted_pos[i]; i3 g = gpos(k, p);
        real lam = -b->C[o];
        real gs = vdot(ZERO3, ZERO3);
        gs = acc_gradsq(k, gs, bcd, p, g, i, 2, b->volume, b->mass, 0);
        gs = acc_gradsq(k, gs, scd, p, g, UMAX, 0, NULL, NULL, 0);
        gs = acc_gradsq(k, gs, dcd, p, g, UMAX, 0, NULL, NULL, 0);
        b->lambda[o] = lam / (gs + k->eps);
    }
}

/* ------------------------------------------- stage: PBF corrections :3070-3351 */
static void stage_pbf(const K* k, or_particles* sph, uint32_t ns, or_particles* dem, uint32_t nd,
                      or_particles* b, const or_cells* scd, const or_cells* dcd, const or_cells* bcd,
                      float dt, int quirks)
{
    /* compute_pbf_sph_correction :3070-3184 */
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)ns; ii++) {
        uint32_t i = (uint32_t)ii, o = scd->grid_index[i];
        r3 p = scd->sorted_pos[i]; i3 g = gpos(k, p);
        real li = sph->lambda[o];
        r3 c = ZERO3;
        c = acc_pbf_own(k, c, scd, p, g, i, li, sph->lambda, sph->contrib, dt);
        c = acc_pbf_cpl(k, c, dcd, p, g, i, li, dem->lambda, dt, quirks);
        c = acc_pbf_bnd(k, c, bcd, p, g, li, b->lambda, dt);
        c = vsc(k->inv_rho0, c);
        c = vsc(sph->contrib[o], c);
        if (vnan(c)) c = ZERO3;
        sph->correction[o] = vadd(sph->correction[o], c);
    }
    /* compute_pbf_new_dem_correction :3187-3304.  Q3: the reference takes the
       original index from the SPH cell data; its += targets may repeat, so this
       loop runs in ascending thread index. */
    for (uint32_t i = 0; i < nd; i++) {
        uint32_t o = quirks == OR_QUIRKS_REFERENCE ? scd->grid_index[i] : dcd->grid_index[i];
        r3 p = dcd->sorted_pos[i]; i3 g = gpos(k, p);
        real li = dem->lambda[o];
        r3 c = ZERO3;
        c = acc_pbf_cpl(k, c, scd, p, g, i, li, sph->lambda, dt, quirks);
        if (vnan(c)) c = ZERO3;
        c = acc_pbf_own(k, c, dcd, p, g, i, li, dem->lambda, dem->contrib, dt);
        if (vnan(c)) c = ZERO3;
        c = acc_pbf_bnd(k, c, bcd, p, g, li, b->lambda, dt);
        if (vnan(c)) c = ZERO3;
        c = vsc(k->inv_rho0, c);
        c = vsc(R(1) - dem->contrib[o], c);
        if (vnan(c)) c = ZERO3;
        dem->correction[o] = vadd(dem->correction[o], c);
    }
}

/* --------------------------------------- stage: distance corrections :2061-2217, :3353-3417 */
static void stage_distance(const K* k, or_particles* sph, uint32_t ns, or_particles* dem, uint32_t nd,
                           or_particles* b, const or_cells* scd, const or_cells* dcd, const or_cells* bcd,
                           int correct_dem, int sph_sph)
{
    if (correct_dem) {
        /* compute_sph_dem_distance_correction :2061-2110 */
        #pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)ns; ii++) {
            uint32_t i = (uint32_t)ii, o = scd->grid_index[i];
            r3 p = scd->sorted_pos[i]; i3 g = gpos(k, p);
            r3 c = acc_contact(k, ZERO3, dcd, p, g, UMAX, sph->massInv[o], dem->massInv);
            c = vsc(R(1) - sph->contrib[o], c);
            if (vnan(c)) c = ZERO3;
            sph->correction[o] = vadd(sph->correction[o], vsc(k->k_stretch, c));
        }
        /* compute_dem_sph_distance_correction :2112-2162 */
        #pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)nd; ii++) {
            uint32_t i = (uint32_t)ii, o = dcd->grid_index[i];
            r3 p = dcd->sorted_pos[i]; i3 g = gpos(k, p);
            r3 c = acc_contact(k, ZERO3, scd, p, g, UMAX, dem->massInv[o], sph->massInv);
            c = vsc(k->k_stretch * dem->contrib[o], c);
            if (vnan(c)) c = ZERO3;
            dem->correction[o] = vadd(dem->correction[o], c);
        }
    }
    if (sph_sph) {
        /* compute_sph_sph_distance_correction :2164-2217 */
        #pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)ns; ii++) {
            uint32_t i = (uint32_t)ii, o = scd->grid_index[i];
            r3 p = scd->sorted_pos[i]; i3 g = gpos(k, p);
            r3 c = acc_contact_sph(k, ZERO3, scd, p, g, i, sph->massInv[o], sph->contrib[o], sph->massInv);
            c = vsc(R(1) - sph->contrib[o], c);
            if (vnan(c)) c = ZERO3;
            sph->correction[o] = vadd(sph->correction[o], c);
        }
    }
    /* compute_dem_distance_correction :1765-1834 */
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)nd; ii++) {
        uint32_t i = (uint32_t)ii, o = dcd->grid_index[i];
        r3 p = dcd->sorted_pos[i]; i3 g = gpos(k, p);
        real w0 = dem->massInv[o];
        r3 c = acc_contact(k, ZERO3, dcd, p, g, i, w0, dem->massInv);
        c = acc_contact(k, c, bcd, p, g, UMAX, w0, b->massInv);
        c = vsc(dem->contrib[o], c);
        if (vnan(c)) c = ZERO3;
        dem->correction[o] = vadd(dem->correction[o], c);
    }
}

/* ------------------------------------------------ stage: interlink :4624-4765 */
static void delete_record(const K* k, or_particles* d, uint32_t i0, uint32_t i1)
{
    for (uint32_t s = i0 * k->maxc; s < (i0 + 1) * k->maxc; s++)
        if (d->connect_record[s] == i1) { d->connect_record[s] = UMAX; d->connect_length[s] = 0; break; }
    for (uint32_t s = i1 * k->maxc; s < (i1 + 1) * k->maxc; s++)
        if (d->connect_record[s] == i0) { d->connect_record[s] = UMAX; d->connect_length[s] = 0; break; }
}
static r3 link_corr(const K* k, or_particles* d, uint32_t i0, uint32_t i1, real L, uint32_t n)
{
    if (i0 == i1 || i0 >= n || i1 >= n || L == 0) return ZERO3;
    r3 p0 = d->predict_positions[i0], p1 = d->predict_positions[i1];
    r3 v = vsub(p0, p1);
    real dist = vlen(v);
    if (dist > k->brk * L) { delete_record(k, d, i0, i1); return ZERO3; }
    if (dist > k->h) { delete_record(k, d, i0, i1); return ZERO3; }
    real w0 = d->massInv[i0], w1 = d->massInv[i1];
    real ws = w0 + w1, C = dist - L;
    r3 n3 = vdivs(v, dist + k->pbd_eps);
    r3 res = vsc(((k->k_ref * -w0) * (R(1) / ws)) * C, n3);
    if (vlen(res) > R(1)) return ZERO3;
    if (vnan(res)) return ZERO3;
    if (vinf(res)) return ZERO3;
    return res;
}
static void stage_interlink(const K* k, or_particles* dem, uint32_t nd)
{
    for (uint32_t i = 0; i < nd; i++) {
        r3 c = ZERO3;
        for (uint32_t s = k->maxc * i; s < k->maxc * (i + 1); s++) {
            uint32_t j = dem->connect_record[s];
            if (j != UMAX) c = vadd(c, link_corr(k, dem, i, j, dem->connect_length[s], nd));
        }
        if (vnan(c)) c = ZERO3;
        dem->correction[i] = vadd(dem->correction[i], c);
    }
}

/* ------------------------------------------------------ apply / finalize :1342-1408 */
static void stage_apply(const K* k, or_particles* d, const or_cells* cd, uint32_t nthreads)
{
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)nthreads; ii++) {
        uint32_t i = (uint32_t)ii, o = cd->grid_index[i];
        r3 np = vadd(cd->sorted_pos[i], vsc(k->sor, d->correction[o]));
        d->new_positions[o] = np;
        d->predict_positions[o] = np;
        d->correction[o] = ZERO3;
    }
}
static void stage_finalize(const K* k, or_particles* d, uint32_t nthreads, float dt)
{
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)nthreads; ii++) {
        uint32_t i = (uint32_t)ii;
        r3 diff = vsub(d->new_positions[i], d->positions[i]);
        r3 tp = d->new_positions[i];
        r3 tv = vlen(diff) >= k->min_speed ? vdivs(diff, R(dt)) : ZERO3;
        d->velocity[i] = tv;
        d->positions[i] = tp;
    }
}

/* ------------------------------------------------------- friction :1989-2059 */
static void stage_friction(const K* k, or_particles* dem, or_particles* b, const or_cells* dcd,
                           const or_cells* bcd, uint32_t nthreads)
{
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)nthreads; ii++) {
        uint32_t i = (uint32_t)ii, o = dcd->grid_index[i];
        r3 p = dcd->sorted_pos[i];
        r3 op0 = dem->positions[o];
        real w0 = dem->massInv[o];
        i3 g = gpos(k, p);
        r3 c = ZERO3;
        FOR27 {
            uint32_t s, e; r3 cs = ZERO3;
            if (crange(k, dcd, g, ox, oy, oz, &s, &e))
                for (uint32_t j = s; j < e; j++) {
                    if (j == i) continue;
                    uint32_t oj = dcd->grid_index[j];
                    r3 op1 = dem->positions[oj];
                    r3 pp1 = dcd->sorted_pos[j];
                    r3 v = vsub(p, pp1);
                    real d = vlen(v);
                    if (d <= k->two_r)
                        cs = vadd(cs, friction_term(k, p, op0, pp1, vsub(pp1, op1), 1, w0, dem->massInv[oj], d, v));
                }
            c = vadd(c, cs);
        }
        FOR27 {
            uint32_t s, e; r3 cs = ZERO3;
            if (crange(k, bcd, g, ox, oy, oz, &s, &e))
                for (uint32_t j = s; j < e; j++) {
                    uint32_t oj = bcd->grid_index[j];
                    r3 pb = bcd->sorted_pos[j];
                    r3 v = vsub(p, pb);
                    real d = vlen(v);
                    if (d <= k->two_r)
                        cs = vadd(cs, friction_term(k, p, op0, pb, ZERO3, 0, w0, b->massInv[oj], d, v));
                }
            c = vadd(c, cs);
        }
        if (vnan(c)) c = ZERO3;
        dem->correction[o] = c;
    }
}

/* ------------------------------------------------- integrate :447-540, :1422-1453 */
static void stage_integrate(const K* k, or_particles* d, uint32_t nthreads, float dt, int cd_on)
{
    const real DT = R(dt);
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)nthreads; ii++) {
        uint32_t i = (uint32_t)ii;
        r3 gdt = v3(DT * k->g[0], DT * k->g[1], DT * k->g[2]);
        r3 tv = vadd(d->velocity[i], gdt);
        tv = v3(tv.x * k->damping, tv.y * k->damping, tv.z * k->damping);
        if (!cd_on) {
            r3 pp = vadd(d->positions[i], vsc(DT, tv));
            d->predict_positions[i] = pp;
            d->velocity[i] = tv;
            d->new_positions[i] = pp;
            continue;
        }
        r3 tp = vadd(d->positions[i], vsc(DT, tv));
        if (tp.x + k->r >= R(g_dom[1])) { tv.x = -RFABS(tv.x); tv = vsc(k->b_damping, tv); }
        if (tp.x - k->r <= R(g_dom[0])) { tv.x = RFABS(tv.x); tv = vsc(k->b_damping, tv); }
        if (tp.z + k->r >= R(g_dom[3])) { tv.z = -RFABS(tv.z); tv = vsc(k->b_damping, tv); }
        if (tp.z - k->r <= R(g_dom[2])) { tv.z = RFABS(tv.z); tv = vsc(k->b_damping, tv); }
        if (d->positions[i].y - k->r <= R(g_dom[4])) {
            d->positions[i].y = R(g_dom[4]) + k->r;
            tv.y = RFABS(tv.y);
            tv = vsc(k->b_damping, tv);
        }
        if (vlen(tv) > k->max_speed) tv = vsc(k->max_speed / vlen(tv), tv);
        r3 pp = vadd(d->positions[i], vsc(DT, tv));
        d->predict_positions[i] = pp;
        d->velocity[i] = tv;
        d->new_positions[i] = pp;
        if (d->contrib[i] < R(0.99f)) d->contrib[i] += k->blending;
        if (d->contrib[i] >= R(0.99f)) d->contrib[i] = R(1.f);
    }
}

/* ------------------------------------------------------------ heat :3764-3970 */
static real heat_cell(const K* k, const or_cells* cd, const or_particles* other, i3 g,
                      int ox, int oy, int oz, uint32_t skip, r3 p, real Ti, real ki, real kj)
{
    uint32_t s, e; real res = 0;
    if (crange(k, cd, g, ox, oy, oz, &s, &e))
        for (uint32_t j = s; j < e; j++) {
            if (j == skip) continue;
            uint32_t oj = cd->grid_index[j];
            real d = vlen(vsub(p, cd->sorted_pos[j]));
            res += (((other->mass[oj] / other->density[oj]) * (((R(4.f) * ki) * kj) / (ki + kj)))
                    * (other->T[oj] - Ti)) * L_visc(k, d);
        }
    return res;
}
static void stage_heat(const K* k, or_particles* sph, uint32_t ns, or_particles* dem, uint32_t nd,
                       const or_cells* scd, const or_cells* dcd, float dt, int quirks)
{
    /* transfer_heat_sph :3812-3878 (Q7: the own cell, 27 times) */
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)ns; ii++) {
        uint32_t i = (uint32_t)ii, o = scd->grid_index[i];
        r3 p = scd->sorted_pos[i]; i3 g = gpos(k, p);
        real Ti = sph->T[o], dT = 0;
        FOR27 {
            int a = quirks == OR_QUIRKS_REFERENCE ? 0 : ox, b = quirks == OR_QUIRKS_REFERENCE ? 0 : oy,
                c = quirks == OR_QUIRKS_REFERENCE ? 0 : oz;
            dT += heat_cell(k, scd, sph, g, a, b, c, i, p, Ti, k->k_water, k->k_water);
        }
        FOR27 {
            int a = quirks == OR_QUIRKS_REFERENCE ? 0 : ox, b = quirks == OR_QUIRKS_REFERENCE ? 0 : oy,
                c = quirks == OR_QUIRKS_REFERENCE ? 0 : oz;
            dT += heat_cell(k, dcd, dem, g, a, b, c, UMAX, p, Ti, k->k_water, k->k_snow);
        }
        dT = dT / (k->C_water * sph->density[o]);
        sph->new_T[o] = Ti + dT * R(dt);
    }
    /* transfer_heat_dem :3880-3937 */
    #pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)nd; ii++) {
        uint32_t i = (uint32_t)ii, o = dcd->grid_index[i];
        r3 p = dcd->sorted_pos[i]; i3 g = gpos(k, p);
        real Ti = dem->T[o], dT = 0;
        FOR27 {
            int a = quirks == OR_QUIRKS_REFERENCE ? 0 : ox, b = quirks == OR_QUIRKS_REFERENCE ? 0 : oy,
                c = quirks == OR_QUIRKS_REFERENCE ? 0 : oz;
            dT += heat_cell(k, dcd, dem, g, a, b, c, i, p, Ti, k->k_snow, k->k_snow);
        }
        FOR27 {
            int a = quirks == OR_QUIRKS_REFERENCE ? 0 : ox, b = quirks == OR_QUIRKS_REFERENCE ? 0 : oy,
                c = quirks == OR_QUIRKS_REFERENCE ? 0 : oz;
            dT += heat_cell(k, scd, sph, g, a, b, c, UMAX, p, Ti, k->k_snow, k->k_water);
        }
        dT = dT / (k->C_snow * dem->density[o]);
        dem->new_T[o] = Ti + dT * R(dt);
    }
    /* thrust::copy new_T -> T (:3968-3969) */
    for (uint32_t i = 0; i < ns; i++) sph->T[i] = sph->new_T[i];
    for (uint32_t i = 0; i < nd; i++) dem->T[i] = dem->new_T[i];
}

/* -------------------------------------------------- phase change :3974-4125, :4387-4622 */
static void copy_info(const K* k, const or_particles* s, or_particles* d, uint32_t i, uint32_t t)
{
    d->positions[t] = s->positions[i];
    d->predict_positions[t] = s->predict_positions[i];
    d->new_positions[t] = s->new_positions[i];
    d->velocity[t] = s->velocity[i];
    d->force[t] = s->force[i];
    d->correction[t] = s->correction[i];
    d->mass[t] = s->mass[i];
    d->massInv[t] = s->massInv[i];
    d->contrib[t] = s->contrib[i];
    d->density[t] = s->density[i];
    d->C[t] = s->C[i];
    d->lambda[t] = s->lambda[i];
    d->T[t] = s->T[i];
    d->new_T[t] = s->new_T[i];
    d->trackId[t] = s->trackId[i];
    for (uint32_t c = 0; c < k->maxc; c++) {
        d->connect_record[t * k->maxc + c] = s->connect_record[i * k->maxc + c];
        d->connect_length[t * k->maxc + c] = s->connect_length[i * k->maxc + c];
    }
    d->iter_end[t] = s->iter_end[i];
}
static void reset_records(const K* k, or_particles* d, uint32_t t)
{
    for (uint32_t c = 0; c < k->maxc; c++) {
        d->connect_record[t * k->maxc + c] = UMAX;
        d->connect_length[t * k->maxc + c] = 0;
    }
    d->iter_end[t] = k->maxc * t;
}
/* rebase = 1 (quirks=fixed, snow set): a moved particle keeps its link count, iter_end =
   t*maxc + count; the reference copies iter_end verbatim (Q13). */
static void compact_set(const K* k, or_particles* d, or_particles* buf, uint32_t full, int rebase)
{
    for (uint32_t i = 0; i < full; i++) copy_info(k, d, buf, i, i);
    for (uint32_t i = 0; i < full; i++) {
        if (d->predicate[i] == 1) {
            uint32_t t = d->scan_index[i];
            copy_info(k, buf, d, i, t);
            if (rebase) d->iter_end[t] = k->maxc * t + (buf->iter_end[i] - k->maxc * i);
            d->new_index[i] = t;
        } else d->new_index[i] = UMAX;
    }
}
static void stage_phase(const K* k, or_particles* sph, uint32_t* ns, or_particles* dem, uint32_t* nd,
                        or_particles* buf, uint32_t full, int freeze, int melt, int fixed)
{
    /* freezing :4416-4449 */
    if (freeze)
        for (uint32_t i = 0; i < *ns; i++)
            if (sph->T[i] <= k->Tf && sph->contrib[i] >= R(0.99f)) {
                uint32_t t = (*dem->new_end)++;
                sph->contrib[i] = 0;
                copy_info(k, sph, dem, i, t);
                sph->predicate[i] = 0;
                sph->trackId[i] = 0;
                dem->predicate[t] = 1;
                reset_records(k, dem, t);
            }
    /* melting :4387-4414 */
    if (melt)
        for (uint32_t i = 0; i < *nd; i++)
            if (dem->T[i] > k->Tf && dem->contrib[i] >= R(0.99f)) {
                uint32_t t = (*sph->new_end)++;
                dem->contrib[i] = 0;
                copy_info(k, dem, sph, i, t);
                dem->predicate[i] = 0;
                dem->trackId[i] = 0;
                sph->predicate[t] = 1;
            }
    /* compact_and_clean :4495-4589 */
    /* thrust::count of predicate == 1, thrust::exclusive_scan of the predicates */
    uint32_t sn = 0, dn = 0, a = 0, b = 0;
    for (uint32_t i = 0; i < full; i++) { sn += sph->predicate[i] == 1; sph->scan_index[i] = a; a += sph->predicate[i]; }
    for (uint32_t i = 0; i < full; i++) { dn += dem->predicate[i] == 1; dem->scan_index[i] = b; b += dem->predicate[i]; }
    /* shuffle_useless_record :4068-4111 */
    for (uint32_t i = 0; i < *nd; i++)
        for (uint32_t s = k->maxc * i; s < (i + 1) * k->maxc; s++) {
            uint32_t r = dem->connect_record[s];
            if (r < *nd && dem->predicate[r] == 0) {
                dem->connect_record[s] = UMAX;
                dem->connect_length[s] = 0;
                dem->iter_end[i]--;
            }
        }
    compact_set(k, sph, buf, full, 0);
    compact_set(k, dem, buf, full, fixed);
    *ns = sn; *nd = dn;
    *sph->new_end = sn; *dem->new_end = dn;
    for (uint32_t i = 0; i < sn; i++) sph->predicate[i] = 1;
    for (uint32_t i = 0; i < dn; i++) dem->predicate[i] = 1;
    /* clean_tail :4482-4493 / clean_particle_info :4004-4034 */
    for (uint32_t t = sn; t < full; t++) {
        sph->predicate[t] = 0; sph->trackId[t] = 0; sph->scan_index[t] = 0; reset_records(k, sph, t);
    }
    for (uint32_t t = dn; t < full; t++) {
        dem->predicate[t] = 0; dem->trackId[t] = 0; dem->scan_index[t] = 0; reset_records(k, dem, t);
    }
    /* update_record_index :4114-4125 */
    for (uint32_t s = 0; s < k->maxc * dn; s++)
        if (dem->connect_record[s] != UMAX) dem->connect_record[s] = dem->new_index[dem->connect_record[s]];
}

/* ------------------------------------------ link formation :4127-4292 (canonical order) */
static inline uint32_t hash_colour(const K* k, uint32_t h)
{
    uint32_t x = h % k->gs[0], y = (h / k->gs[0]) % k->gs[1], z = h / (k->gs[0] * k->gs[1]);
    return ((x >> 1) & 1u) | (((y >> 1) & 1u) << 1) | (((z >> 1) & 1u) << 2);
}
static uint32_t link_tolerance(const K* k, real T, int dynamic)
{
    uint32_t tol = dynamic ? cvt_u32(((T - k->Tf) / (k->Th - k->Tf)) * R((float)k->maxc)) : k->maxc;
    return tol < k->maxc ? tol : k->maxc;
}
static void connect_particle(const K* k, or_particles* d, const or_cells* cd, uint32_t i, int dynamic)
{
    r3 p = cd->sorted_pos[i];
    uint32_t o = cd->grid_index[i];
    i3 g = gpos(k, p);
    real T = d->T[o];
    const uint32_t M = k->maxc;
    FOR27 {
        uint32_t s, e;
        if (!crange(k, cd, g, ox, oy, oz, &s, &e)) continue;
        for (uint32_t j = s; j < e; j++) {
            if (j == i) continue;
            uint32_t o1 = cd->grid_index[j];
            real dist = vlen(vsub(p, cd->sorted_pos[j]));
            uint32_t count = d->iter_end[o] - o * M;
            uint32_t tol = link_tolerance(k, T, dynamic);
            if (dist < k->h && count < tol) {
                int dup = 0;
                for (uint32_t idx = M * o; idx < M * (o + 1); idx++)
                    if (d->connect_record[idx] == o1) { dup = 1; break; }
                if (dup) goto next_cell;   /* the reference returns from the cell helper */
                for (uint32_t idx = M * o; idx < M * (o + 1); idx++) {
                    if (d->connect_record[idx] == UMAX) {
                        d->connect_record[idx] = o1;
                        int valid = 0;
                        if (d->iter_end[o1] < (o1 + 1) * M)
                            for (uint32_t q = o1 * M; q < (o1 + 1) * M; q++)
                                if (d->connect_record[q] == UMAX) {
                                    d->connect_record[q] = o;
                                    d->connect_length[q] = dist;
                                    d->iter_end[o1]++;
                                    valid = 1;
                                    break;
                                }
                        if (valid) { d->connect_length[idx] = dist; d->iter_end[o]++; }
                        else d->connect_record[idx] = UMAX;
                        break;
                    }
                }
            }
        }
    next_cell:;
    }
}
void or_connect_and_record(const or_params* P, or_particles* dem, uint32_t n, or_cells cd, int dynamic)
{
    K k = mk(P);
    for (uint32_t c = 0; c < 8; c++)
        for (uint32_t i = 0; i < n; i++)
            if (hash_colour(&k, cd.grid_hash[i]) == c) connect_particle(&k, dem, &cd, i, dynamic);
}
/* adjust_connections_d :4768-4808, sequential; the reference indexes the partner's
   slots with an empty record (UINT_MAX) once count exceeds the cap -- that read is
   out of bounds there and is skipped here. */
static void stage_adjust(const K* k, or_particles* d, uint32_t n, uint32_t full)
{
    const uint32_t M = k->maxc;
    for (uint32_t i = 0; i < n; i++) {
        real T = d->T[i];
        uint32_t cm = cvt_u32(((T - k->Tf) / (k->Th - k->Tf)) * R((float)M));
        if (cm > M) cm = M;
        uint32_t count = 0;
        for (uint32_t s = M * i; s < M * (i + 1); s++) {
            count = d->connect_record[s] != UMAX ? count + 1 : count;
            if (count > cm) {
                uint32_t j = d->connect_record[s];
                d->connect_record[s] = UMAX;
                d->connect_length[s] = 0;
                d->iter_end[i]--;
                if (j == UMAX || j >= full) continue;
                for (uint32_t q = M * j; q < M * (j + 1); q++)
                    if (d->connect_record[q] == i) {
                        d->connect_record[q] = UMAX; d->connect_length[q] = 0; d->iter_end[j]--;
                    }
            }
        }
    }
}

/* ---------------------------------------------------------------- XSPH :3419-3711 */
static r3 acc_xsph(const K* k, r3 acc, const or_cells* cd, const or_particles* o_, const r3* vel,
                   r3 p, i3 g, uint32_t skip, r3 vi)
{
    FOR27 {
        uint32_t s, e; r3 cs = ZERO3;
        if (crange(k, cd, g, ox, oy, oz, &s, &e))
            for (uint32_t j = s; j < e; j++) {
                if (j == skip) continue;
                uint32_t oj = cd->grid_index[j];
                real d = vlen(vsub(p, cd->sorted_pos[j]));
                r3 vij = vsub(vel[oj], vi);
                real a = o_->mass[oj] / o_->density[oj];
                real w = W_poly6(k, d);
                cs = vadd(cs, v3((a * vij.x) * w, (a * vij.y) * w, (a * vij.z) * w));
            }
        acc = vadd(acc, cs);
    }
    return acc;
}
static void stage_xsph(const K* k, or_particles* sph, uint32_t ns, or_particles* dem, uint32_t nd,
                       const or_cells* scd, const or_cells* dcd, int step_sph, int step_dem,
                       int dem_visc, uint32_t full, int quirks)
{
    r3* tmp = (r3*)malloc(sizeof(r3) * (full ? full : 1));
    if (step_sph && ns) {
        memcpy(tmp, sph->velocity, sizeof(r3) * full);
        #pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)ns; ii++) {
            uint32_t i = (uint32_t)ii, o = scd->grid_index[i];
            r3 p = scd->sorted_pos[i]; i3 g = gpos(k, p);
            r3 vi = tmp[o];
            r3 c = acc_xsph(k, ZERO3, scd, sph, tmp, p, g, i, vi);
            c = acc_xsph(k, c, dcd, dem, dem->velocity, p, g, UMAX, vi);
            c = vsc(k->sph_visc, c);
            sph->velocity[o] = vadd(vi, c);
        }
    }
    if (dem_visc && step_dem) {
        /* Q6: launched with the SPH grid, so only the first coverage(n_sph) DEM
           particles (in sorted order) are smoothed. */
        uint32_t nt = quirks == OR_QUIRKS_REFERENCE ? umin(coverage(ns), nd) : nd;
        memcpy(tmp, dem->velocity, sizeof(r3) * full);
        #pragma omp parallel for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)nt; ii++) {
            uint32_t i = (uint32_t)ii, o = dcd->grid_index[i];
            r3 p = dcd->sorted_pos[i]; i3 g = gpos(k, p);
            r3 vi = tmp[o];
            r3 c = acc_xsph(k, ZERO3, dcd, dem, tmp, p, g, i, vi);
            c = acc_xsph(k, c, scd, sph, sph->velocity, p, g, UMAX, vi);
            c = vsc(k->dem_visc, c);
            dem->velocity[o] = vadd(vi, c);
        }
    }
    free(tmp);
}

/* -------------------------------------------------------------- snow_simulation :4861-5157 */
#define STOP(n) do { if (stop_after == (n)) return 0; } while (0)
int or_snow_simulation(const or_params* P,
                       or_particles* sph, uint32_t* sph_size,
                       or_particles* dem, uint32_t* dem_size,
                       or_particles* bnd, uint32_t b_size,
                       uint32_t full, or_particles* buffer,
                       or_cells scd, or_cells dcd, or_cells bcd,
                       or_scene* scene, float dt, int iterations,
                       uint32_t flags, float temperature_variation,
                       int quirks, int stop_after)
{
    K k = mk(P);
    const int fixed = quirks == OR_QUIRKS_FIXED;
    int step_sph = scene->current_time >= scene->fluid_start_time;
    int step_dem = scene->current_time >= scene->solid_start_time;
    /* launch coverage computed from the sizes at entry (:4891-4894) */
    const uint32_t cov_s0 = coverage(*sph_size), cov_d0 = coverage(*dem_size);

    sort_and_reorder(P, &k, dem->predict_positions, dcd, *dem_size, quirks);
    sort_and_reorder(P, &k, sph->predict_positions, scd, *sph_size, quirks);
    STOP(1);
    stage_density(&k, sph, *sph_size, dem, *dem_size, bnd, b_size, &scd, &dcd, &bcd);
    STOP(2);
    if (flags & OR_COMPUTE_TEMPERATURE) {
        stage_heat(&k, sph, *sph_size, dem, *dem_size, &scd, &dcd, dt, quirks);
        /* environmental_heat_transfer :4847-4859 */
        const real dTe = R(temperature_variation);
        if (step_sph) for (uint32_t i = 0; i < *sph_size; i++) sph->T[i] += dTe;
        if (step_dem) for (uint32_t i = 0; i < *dem_size; i++) dem->T[i] += dTe;
    }
    STOP(3);
    if (flags & OR_CHANGE_PHASE)
        stage_phase(&k, sph, sph_size, dem, dem_size, buffer, full,
                    (flags & OR_SIMULATE_FREEZING) != 0, (flags & OR_SIMULATE_MELTING) != 0, fixed);
    STOP(4);
    sort_and_reorder(P, &k, dem->predict_positions, dcd, *dem_size, quirks);
    sort_and_reorder(P, &k, sph->predict_positions, scd, *sph_size, quirks);
    STOP(5);
    if (flags & OR_USE_INTERLINK) {
        or_connect_and_record(P, dem, *dem_size, dcd, (flags & OR_DYNAMIC_MAX_CONN) != 0);
        if (flags & OR_DYNAMIC_MAX_CONN) stage_adjust(&k, dem, *dem_size, full);
    }
    STOP(6);
    {
        const int cd_on = (flags & OR_CD_ON) != 0;
        /* integrate_pbd_cd_d has no bounds check: the whole launch coverage runs */
        if (step_sph) stage_integrate(&k, sph, fixed ? *sph_size : umin(coverage(*sph_size), full), dt, cd_on);
        if (step_dem) stage_integrate(&k, dem, fixed ? *dem_size : umin(coverage(*dem_size), full), dt, cd_on);
    }
    STOP(7);
    /* Q12: apply/finalize/friction keep the launch grid computed at entry */
    const uint32_t ap_s = fixed ? *sph_size : umin(cov_s0, *sph_size);
    const uint32_t ap_d = fixed ? *dem_size : umin(cov_d0, *dem_size);
    for (int it = 0; it < iterations; it++) {
        const int base = 10 + 10 * it;
        sort_and_reorder(P, &k, dem->predict_positions, dcd, *dem_size, quirks);
        sort_and_reorder(P, &k, sph->predict_positions, scd, *sph_size, quirks);
        STOP(base + 0);
        stage_density(&k, sph, *sph_size, dem, *dem_size, bnd, b_size, &scd, &dcd, &bcd);
        STOP(base + 1);
        stage_lambda(&k, sph, *sph_size, dem, *dem_size, bnd, b_size, &scd, &dcd, &bcd);
        STOP(base + 2);
        stage_pbf(&k, sph, *sph_size, dem, *dem_size, bnd, &scd, &dcd, &bcd, dt, quirks);
        STOP(base + 3);
        stage_distance(&k, sph, *sph_size, dem, *dem_size, bnd, &scd, &dcd, &bcd,
                       (flags & OR_SPH_DEM_CORRECTION) != 0, (flags & OR_SPH_SPH_CORRECTION) != 0);
        STOP(base + 4);
        if (flags & OR_USE_INTERLINK) stage_interlink(&k, dem, *dem_size);
        STOP(base + 5);
        if (step_sph) stage_apply(&k, sph, &scd, ap_s);
        if (step_dem) stage_apply(&k, dem, &dcd, ap_d);
        STOP(base + 6);
        if ((flags & OR_DEM_FRICTION) && step_dem) {
            sort_and_reorder(P, &k, dem->predict_positions, dcd, *dem_size, quirks);
            sort_and_reorder(P, &k, sph->predict_positions, scd, *sph_size, quirks);
            stage_friction(&k, dem, bnd, &dcd, &bcd, ap_d);
            stage_apply(&k, dem, &dcd, ap_d);
        }
        STOP(base + 7);
    }
    if (step_sph) stage_finalize(&k, sph, ap_s, dt);
    if (step_dem) stage_finalize(&k, dem, ap_d, dt);
    STOP(90);
    stage_xsph(&k, sph, *sph_size, dem, *dem_size, &scd, &dcd, step_sph, step_dem,
               (flags & OR_DEM_VISCOSITY) != 0, full, quirks);
    scene->current_time += dt;
    return 0;
}

void or_energy_momentum(const or_params* P, const or_particles* sph, uint32_t ns,
                        const or_particles* dem, uint32_t nd, double out[4])
{
    double e = 0, mx = 0, my = 0, mz = 0;
    for (uint32_t i = 0; i < ns; i++) {
        double m = (double)sph->mass[i];
        e += m * (double)P->C_water * (double)sph->T[i];
        mx += m * (double)sph->velocity[i].x; my += m * (double)sph->velocity[i].y; mz += m * (double)sph->velocity[i].z;
    }
    for (uint32_t i = 0; i < nd; i++) {
        double m = (double)dem->mass[i];
        e += m * (double)P->C_snow * (double)dem->T[i];
        mx += m * (double)dem->velocity[i].x; my += m * (double)dem->velocity[i].y; mz += m * (double)dem->velocity[i].z;
    }
    out[0] = e; out[1] = mx; out[2] = my; out[3] = mz;
}
