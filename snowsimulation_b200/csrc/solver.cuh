// solver.cuh -- constraint and integration kernels of the substep.
//
// One thread per particle in sorted order (neighbouring threads share cells, so the
// 27-cell gathers hit L1), fused across the particle sets of a stage, grid-stride over
// the set sizes held on the device.  Each neighbor sum keeps the reference's structure
// (per-cell partial sums added to the running total, cells z-y-x, particles ascending)
// and skips only terms that are exactly zero: a term is evaluated when
// d2 < cut-off, which is equivalent to the reference's distance test d < h (resp.
// d < 2r, d <= 2r) because sqrt is correctly rounded and monotone.
#pragma once
#include "common.cuh"
#include "sort.cuh"

namespace snowb {

struct Sets {
    snowb_particle_data sph, dem, bnd;
};
// compact sorted attribute copies (valid for sorted index j < n of the last sort)
struct Sorted {
    float* invm;     // massInv
    float* contrib;  // contrib
    float* lambda;   // lambda (written by the lambda stage)
    float* mass;     // boundary only: mass
};

// Neighbour lists.  The density+lambda pass records, per water or snow particle, every
// candidate that passed the support test (d < h), in traversal order, tagged with its
// set and its cell (0..26).  The PBF and contact passes of the same sort replay the list
// (their supports are d < h or smaller) instead of re-testing ~300 candidates over 81
// cells, keeping the per-cell partial sums.  A particle with more than NLIST_K entries is
// marked overflowed and its consumers traverse the cells as before.
#ifndef SNOWB_NLIST_K
#define SNOWB_NLIST_K 384
#endif
constexpr uint32_t NLIST_K = SNOWB_NLIST_K;
constexpr uint32_t NL_J_MASK = (1u << 25) - 1u;
constexpr uint32_t NL_OVF = 1u << 31;
struct NList {
    uint32_t* e;       // entry k of slot s at e[k * stride + s]: j | cell << 25 | set << 30
    uint32_t* cnt;     // per slot: own | other << 10 | boundary << 20 (| NL_OVF)
    uint32_t stride;   // 2 * capacity: water slots [0, cap), snow slots [cap, 2 cap)
    uint32_t cap;
};
struct NLWriter {
    uint32_t* e;
    uint32_t stride, slot, n;
    __device__ __forceinline__ void push(uint32_t j, int cell, int set)
    {
        if (n < NLIST_K) e[(size_t)n * stride + slot] = j | ((uint32_t)cell << 25) | ((uint32_t)set << 30);
        ++n;
    }
};
#define CELL27 ((oz + 1) * 9 + (oy + 1) * 3 + (ox + 1))

// ------------------------------------------------------------ per-cell neighbour sums
// pbf_correction (:883-929)
__device__ __forceinline__ float3 pbf_own_cell(const DevParams& P, const SetView& v, float3 p, GCell g, int ox, int oy,
                                               int oz, uint32_t skip, float li, const float* lam_s, const float* lam_o,
                                               const float* con_s, const float* con_o, float dt)
{
    float3 cs = f3(0.f, 0.f, 0.f);
    uint32_t s, e;
    if (v.range(P, g, ox, oy, oz, s, e))
        for (uint32_t j = s; j < e; ++j) {
            if (j == skip) continue;
            float3 dv = sub3(p, v.pos(j));
            float d2 = dot3(dv, dv);
            if (d2 < P.h2_lt) {
                float d = sqrtf(d2);
                float3 gr = G_spiky_in(P, dv, d);
                float lj = v.attr(lam_s, lam_o, j), cj = v.attr(con_s, con_o, j);
                cs = add3(cs, sc3(cj * lam_scorr(P, li + lj, d, dt), gr));
            }
        }
    return cs;
}
__device__ __forceinline__ float3 acc_pbf_own(const DevParams& P, float3 acc, const SetView& v, float3 p, GCell g,
                                              uint32_t skip, float li, const float* lam_s, const float* lam_o,
                                              const float* con_s, const float* con_o, float dt)
{
    FOR27 acc = add3(acc, pbf_own_cell(P, v, p, g, ox, oy, oz, skip, li, lam_s, lam_o, con_s, con_o, dt));
    return acc;
}
// pbf_correction_boundary (:932-979)
__device__ __forceinline__ float3 pbf_bnd_cell(const DevParams& P, const SetView& v, float3 p, GCell g, int ox, int oy,
                                               int oz, float li, const float* lam_s, const float* lam_o, float dt)
{
    float3 cs = f3(0.f, 0.f, 0.f);
    uint32_t s, e;
    if (v.range(P, g, ox, oy, oz, s, e))
        for (uint32_t j = s; j < e; ++j) {
            float3 dv = sub3(p, v.pos(j));
            float d2 = dot3(dv, dv);
            if (d2 < P.h2_lt) {
                float d = sqrtf(d2);
                float3 gr = G_spiky_in(P, dv, d);
                cs = add3(cs, sc3(lam_scorr(P, li + v.attr(lam_s, lam_o, j), d, dt), gr));
            }
        }
    return cs;
}
__device__ __forceinline__ float3 acc_pbf_bnd(const DevParams& P, float3 acc, const SetView& v, float3 p, GCell g,
                                              float li, const float* lam_s, const float* lam_o, float dt)
{
    FOR27 acc = add3(acc, pbf_bnd_cell(P, v, p, g, ox, oy, oz, li, lam_s, lam_o, dt));
    return acc;
}
// pbf_correction_coupling (:982-1034); reference quirks: the self-skip compares indices of
// two different sets, and s_corr is taken as 0 (it reads an uninitialised value times 0)
__device__ __forceinline__ float3 pbf_cpl_cell(const DevParams& P, const SetView& v, float3 p, GCell g, int ox, int oy,
                                               int oz, uint32_t skip, float li, const float* lam_s, const float* lam_o,
                                               float dt)
{
    const bool ref = P.quirks == SNOWB_QUIRKS_REFERENCE;
    float3 cs = f3(0.f, 0.f, 0.f);
    uint32_t s, e;
    if (v.range(P, g, ox, oy, oz, s, e))
        for (uint32_t j = s; j < e; ++j) {
            if (ref && j == skip) continue;
            float3 dv = sub3(p, v.pos(j));
            float d2 = dot3(dv, dv);
            if (d2 < P.r2_le) {
                float d = sqrtf(d2);
                float3 gr = G_poly6(P, dv, d);
                cs = add3(cs, sc3(lam_scorr_cpl(P, li + v.attr(lam_s, lam_o, j), d, dt), gr));
            }
        }
    return cs;
}
__device__ __forceinline__ float3 acc_pbf_cpl(const DevParams& P, float3 acc, const SetView& v, float3 p, GCell g,
                                              uint32_t skip, float li, const float* lam_s, const float* lam_o,
                                              float dt)
{
    FOR27 acc = add3(acc, pbf_cpl_cell(P, v, p, g, ox, oy, oz, skip, li, lam_s, lam_o, dt));
    return acc;
}
// non-penetration: pbd_distance_correction_contrib (:1470-1527, skip) and
// pbd_distance_correction_coupling_contrib (:1648-1705, no skip)
// per-cell partial of acc_contact (cell at offset ox, oy, oz)
__device__ __forceinline__ float3 contact_cell(const DevParams& P, const SetView& v, float3 p, GCell g, int ox, int oy,
                                               int oz, uint32_t skip, float w0, const float* invm_s,
                                               const float* invm_o)
{
    float3 cs = f3(0.f, 0.f, 0.f);
    uint32_t s, e;
    if (v.range_culled(P, g, ox, oy, oz, p, P.r2_cull, s, e))
        for (uint32_t j = s; j < e; ++j) {
            if (j == skip) continue;
            float3 dv = sub3(p, v.pos(j));
            float d2 = dot3(dv, dv);
            if (d2 < P.r2_lt) {
                float d = sqrtf(d2);
                float w1 = v.attr(invm_s, invm_o, j);
                float ws = w0 + w1;
                float C = d - P.two_r;
                float3 n = div3(dv, d + P.pbd_eps);
                cs = add3(cs, sc3(((-w0) * (1.f / ws)) * C, n));
            }
        }
    return cs;
}
__device__ __forceinline__ float3 acc_contact(const DevParams& P, float3 acc, const SetView& v, float3 p, GCell g,
                                              uint32_t skip, float w0, const float* invm_s, const float* invm_o)
{
    FOR27 acc = add3(acc, contact_cell(P, v, p, g, ox, oy, oz, skip, w0, invm_s, invm_o));
    return acc;
}

// Replays of a recorded neighbour segment [k0, k1) of slot `slot`, per-cell partial sums
// kept (entries of one cell are contiguous and in traversal order).
struct Seg {
    const uint32_t* e;
    uint32_t stride, slot, k0, k1;
    __device__ __forceinline__ uint32_t at(uint32_t k) const { return __ldg(e + (size_t)k * stride + slot); }
};
__device__ __forceinline__ float3 seg_pbf_own(const DevParams& P, float3 acc, const Seg& S, const SetView& v,
                                              float3 p, float li, const float* lam_s, const float* lam_o,
                                              const float* con_s, const float* con_o, float dt)
{
    float3 cs = f3(0.f, 0.f, 0.f);
    uint32_t cur = 0xFFu;
    for (uint32_t k = S.k0; k < S.k1; ++k) {
        const uint32_t en = S.at(k), j = en & NL_J_MASK, cell = (en >> 25) & 31u;
        if (cell != cur) { if (cur != 0xFFu) acc = add3(acc, cs); cs = f3(0.f, 0.f, 0.f); cur = cell; }
        float3 dv = sub3(p, v.pos(j));
        float d = sqrtf(dot3(dv, dv));   // a recorded candidate: d < h
        float3 gr = G_spiky_in(P, dv, d);
        float lj = v.attr(lam_s, lam_o, j), cj = v.attr(con_s, con_o, j);
        cs = add3(cs, sc3(cj * lam_scorr(P, li + lj, d, dt), gr));
    }
    if (cur != 0xFFu) acc = add3(acc, cs);
    return acc;
}
__device__ __forceinline__ float3 seg_pbf_bnd(const DevParams& P, float3 acc, const Seg& S, const SetView& v,
                                              float3 p, float li, const float* lam_s, const float* lam_o, float dt)
{
    float3 cs = f3(0.f, 0.f, 0.f);
    uint32_t cur = 0xFFu;
    for (uint32_t k = S.k0; k < S.k1; ++k) {
        const uint32_t en = S.at(k), j = en & NL_J_MASK, cell = (en >> 25) & 31u;
        if (cell != cur) { if (cur != 0xFFu) acc = add3(acc, cs); cs = f3(0.f, 0.f, 0.f); cur = cell; }
        float3 dv = sub3(p, v.pos(j));
        float d = sqrtf(dot3(dv, dv));   // a recorded candidate: d < h
        float3 gr = G_spiky_in(P, dv, d);
        cs = add3(cs, sc3(lam_scorr(P, li + v.attr(lam_s, lam_o, j), d, dt), gr));
    }
    if (cur != 0xFFu) acc = add3(acc, cs);
    return acc;
}
__device__ __forceinline__ float3 seg_pbf_cpl(const DevParams& P, float3 acc, const Seg& S, const SetView& v,
                                              float3 p, uint32_t skip, float li, const float* lam_s,
                                              const float* lam_o, float dt)
{
    const bool ref = P.quirks == SNOWB_QUIRKS_REFERENCE;
    float3 cs = f3(0.f, 0.f, 0.f);
    uint32_t cur = 0xFFu;
    for (uint32_t k = S.k0; k < S.k1; ++k) {
        const uint32_t en = S.at(k), j = en & NL_J_MASK, cell = (en >> 25) & 31u;
        if (cell != cur) { if (cur != 0xFFu) acc = add3(acc, cs); cs = f3(0.f, 0.f, 0.f); cur = cell; }
        if (ref && j == skip) continue;
        float3 dv = sub3(p, v.pos(j));
        float d2 = dot3(dv, dv);
        if (d2 < P.r2_le) {
            float d = sqrtf(d2);
            float3 gr = G_poly6(P, dv, d);
            cs = add3(cs, sc3(lam_scorr_cpl(P, li + v.attr(lam_s, lam_o, j), d, dt), gr));
        }
    }
    if (cur != 0xFFu) acc = add3(acc, cs);
    return acc;
}
__device__ __forceinline__ float3 seg_contact(const DevParams& P, float3 acc, const Seg& S, const SetView& v,
                                              float3 p, float w0, const float* invm_s, const float* invm_o)
{
    // entries taken four (then two) at a time: their squared distances screened with packed
    // arithmetic against the slightly larger r2_cull, the exact test and the term for those
    // that pass; per-cell partials closed where the cell changes, entry by entry in order
    const P2 pp = bcast2(p);
    float3 cs = f3(0.f, 0.f, 0.f);
    uint32_t cur = 0xFFu;
    auto one = [&](uint32_t j, uint32_t cell, float3 q, bool pass) {
        if (cell != cur) { if (cur != 0xFFu) acc = add3(acc, cs); cs = f3(0.f, 0.f, 0.f); cur = cell; }
        if (!pass) return;
        float3 dv = sub3(p, q);
        float d2 = dot3(dv, dv);
        if (d2 < P.r2_lt) {
            float d = sqrtf(d2);
            float w1 = v.attr(invm_s, invm_o, j);
            float ws = w0 + w1;
            float C = d - P.two_r;
            float3 n = div3(dv, d + P.pbd_eps);
            cs = add3(cs, sc3(((-w0) * (1.f / ws)) * C, n));
        }
    };
    uint32_t k = S.k0;
    for (; k + 3 < S.k1; k += 4) {
        const uint32_t e0 = S.at(k), e1 = S.at(k + 1), e2 = S.at(k + 2), e3 = S.at(k + 3);
        const uint32_t j0 = e0 & NL_J_MASK, j1 = e1 & NL_J_MASK, j2 = e2 & NL_J_MASK, j3 = e3 & NL_J_MASK;
        const float3 q0 = v.pos(j0), q1 = v.pos(j1), q2 = v.pos(j2), q3 = v.pos(j3);
        const float2 da = d2_pair(pp, make_float4(q0.x, q0.y, q0.z, 0.f), make_float4(q1.x, q1.y, q1.z, 0.f));
        const float2 db = d2_pair(pp, make_float4(q2.x, q2.y, q2.z, 0.f), make_float4(q3.x, q3.y, q3.z, 0.f));
        one(j0, (e0 >> 25) & 31u, q0, da.x < P.r2_cull);
        one(j1, (e1 >> 25) & 31u, q1, da.y < P.r2_cull);
        one(j2, (e2 >> 25) & 31u, q2, db.x < P.r2_cull);
        one(j3, (e3 >> 25) & 31u, q3, db.y < P.r2_cull);
    }
    for (; k + 1 < S.k1; k += 2) {
        const uint32_t e0 = S.at(k), e1 = S.at(k + 1);
        const uint32_t j0 = e0 & NL_J_MASK, j1 = e1 & NL_J_MASK;
        const float3 q0 = v.pos(j0), q1 = v.pos(j1);
        const float2 dd = d2_pair(pp, make_float4(q0.x, q0.y, q0.z, 0.f), make_float4(q1.x, q1.y, q1.z, 0.f));
        one(j0, (e0 >> 25) & 31u, q0, dd.x < P.r2_cull);
        one(j1, (e1 >> 25) & 31u, q1, dd.y < P.r2_cull);
    }
    if (k < S.k1) {
        const uint32_t e0 = S.at(k), j0 = e0 & NL_J_MASK;
        one(j0, (e0 >> 25) & 31u, v.pos(j0), true);
    }
    if (cur != 0xFFu) acc = add3(acc, cs);
    return acc;
}
// segments of slot `slot`; false when the list overflowed (fall back to traversal)
__device__ __forceinline__ bool segments(const NList& L, uint32_t slot, Seg& own, Seg& oth, Seg& bnd)
{
    const uint32_t c = L.cnt[slot];
    if (c & NL_OVF) return false;
    const uint32_t a = c & 1023u, b = (c >> 10) & 1023u, d = (c >> 20) & 1023u;
    own = Seg{L.e, L.stride, slot, 0u, a};
    oth = Seg{L.e, L.stride, slot, a, a + b};
    bnd = Seg{L.e, L.stride, slot, a + b, a + b + d};
    return true;
}

// ======================================================================== density
// Density and W-weighted sums with an optional lambda gradient sum in the same pass.
// compute_snow_{sph,dem_sph,boundary}_density_d (:2219-2528) and, when LAMBDA is set,
// compute_snow_{sph,dem_sph,boundary}_lambdas_d (:2598-2898): lambda needs the particle's
// own C and neighbour positions only, so both come out of one traversal.  Each quantity
// keeps its own per-cell accumulation in the reference's loop order.
// one candidate of acc_WG
template <bool LAMBDA>
__device__ __forceinline__ void wg_term(const DevParams& P, float& cs, float& cg, float4 q, float3 p, uint32_t j,
                                        bool vol, int mode, float m_self, float m_j, NLWriter* wr, int cell, int set)
{
    float3 dv = sub3(p, xyz(q));
    float d2 = dot3(dv, dv);
    if (d2 < P.h2_lt) {
        if (wr) wr->push(j, cell, set);
        float d = sqrtf(d2);   // d < h: d2 passed the exact support test
        float w = vol ? P.rho0 * q.w : q.w;
        cs += w * W_poly6_in(P, d);
        if (LAMBDA) {
            float sc;
            if (mode == 0) sc = P.inv_rho0;
            else {
                float m = mode == 1 ? m_self : m_j;
                sc = P.inv_rho0 * ((P.rho0 * q.w) / m);
            }
            float3 gc = sc3(sc, G_spiky_in(P, dv, d));
            cg += dot3(gc, gc);
        }
    }
}
template <bool LAMBDA>
__device__ __forceinline__ void acc_WG(const DevParams& P, float& rho, float& gs, const SetView& v, float3 p,
                                       const Nbhd& nb, uint32_t skip, bool vol, int mode, float m_self,
                                       const float* mass_s, const float* mass_o, NLWriter* wr = nullptr, int set = 0,
                                       float* dpart = nullptr, uint32_t* dmask = nullptr)
{
    const P2 pp = bcast2(p);
    FOR27 {
        float cs = 0.f, cg = 0.f;
        uint32_t s, e;
        if (v.range_nb(nb, ox, oy, oz, s, e)) {
            const int cell = CELL27;
            if (e <= v.n) {
                // current entries only: the compact sorted copies.  Candidates are screened
                // two at a time with packed arithmetic; ptxas may contract its multiply-adds,
                // so the screen is a superset test against the slightly larger h2_cull, and
                // every candidate that passes goes through the exact scalar test and terms.
                uint32_t j = s;
                for (; j + 1 < e; j += 2) {
                    const float4 q0 = __ldg(v.p4 + j), q1 = __ldg(v.p4 + j + 1);
                    const float2 dd = d2_pair(pp, q0, q1);
                    if (dd.x < P.h2_cull && j != skip) {
                        const float mj = (LAMBDA && mode == 2) ? __ldg(mass_s + j) : 0.f;
                        wg_term<LAMBDA>(P, cs, cg, q0, p, j, vol, mode, m_self, mj, wr, cell, set);
                    }
                    if (dd.y < P.h2_cull && j + 1 != skip) {
                        const float mj = (LAMBDA && mode == 2) ? __ldg(mass_s + j + 1) : 0.f;
                        wg_term<LAMBDA>(P, cs, cg, q1, p, j + 1, vol, mode, m_self, mj, wr, cell, set);
                    }
                }
                if (j < e && j != skip) {
                    const float mj = (LAMBDA && mode == 2) ? __ldg(mass_s + j) : 0.f;
                    wg_term<LAMBDA>(P, cs, cg, __ldg(v.p4 + j), p, j, vol, mode, m_self, mj, wr, cell, set);
                }
            } else {
                for (uint32_t j = s; j < e; ++j) {
                    if (j == skip) continue;
                    const float mj = (LAMBDA && mode == 2) ? v.attr(mass_s, mass_o, j) : 0.f;
                    wg_term<LAMBDA>(P, cs, cg, v.pw(j), p, j, vol, mode, m_self, mj, wr, cell, set);
                }
            }
        }
        // dpart: keep the cell's density partial aside instead of adding it now (a partial
        // of +0, which adds nothing, is not kept)
        if (dpart) {
            if (cs != 0.f) { dpart[CELL27] = cs; *dmask |= 1u << CELL27; }
        } else {
            rho += cs;
        }
        if (LAMBDA) gs += cg;
    }
}
template <bool LAMBDA>
// with_bnd = 0: water and snow only (the boundary particles' density, C and lambda are then
// left as they were; a later density+lambda pass of the substep rewrites them).  The water
// and snow sums take the boundary's terms either way, through its compact sorted copies.
__global__ void __launch_bounds__(256) k_density(DevParams P, DevState* __restrict__ S, SetView vs, SetView vd,
                                                 SetView vb, Sets X, Sorted ss, Sorted sd, Sorted sb, NList L,
                                                 int with_bnd)
{
    const uint32_t ns = S->n_sph, nd = S->n_dem, nb = S->n_b, nbt = with_bnd ? nb : 0u;
    vs.n = ns; vd.n = nd; vb.n = nb;
    const float3 z = f3(0.f, 0.f, 0.f);
    if (LAMBDA && blockIdx.x == 0 && threadIdx.x == 0) S->far_move = 0u;   // the lists are new
    GRID_LOOP(t, ns + nd + nbt) {
        float rho, gs = dot3(z, z);
        const snowb_particle_data* D;
        float* lam_s;
        uint32_t o, i;
        if (t < ns + nd) {
            const bool w = t < ns;
            i = w ? t : t - ns;
            const SetView& own = w ? vs : vd;
            const SetView& oth = w ? vd : vs;
            D = w ? &X.sph : &X.dem;
            lam_s = w ? ss.lambda : sd.lambda;
            o = own.gi[i];
            float3 p = xyz(own.p4[i]); GCell g = grid_pos(P, p, own.scene(i));
            const Nbhd nb = make_nbhd(P, g, p, P.h2_cull);
            rho = D->mass[o] * P.W0;
            NLWriter wr{L.e, L.stride, (w ? 0u : L.cap) + i, 0u};
            // the density+lambda pass lists all three sets for the PBF and contact passes; the
            // substep's first density pass lists the snow-snow candidates for link formation
            NLWriter* pw = (LAMBDA || !w) ? &wr : nullptr;
            acc_WG<LAMBDA>(P, rho, gs, own, p, nb, i, false, 0, 0.f, nullptr, nullptr, pw, 0);
            const uint32_t n_own = wr.n;
            if (!LAMBDA) pw = nullptr;
            acc_WG<LAMBDA>(P, rho, gs, oth, p, nb, SNOWB_UMAX, false, 0, 0.f, nullptr, nullptr, pw, 1);
            const uint32_t n_oth = wr.n - n_own;
            acc_WG<LAMBDA>(P, rho, gs, vb, p, nb, SNOWB_UMAX, true, 1, D->mass[o], nullptr, nullptr, pw, 2);
            if (LAMBDA) {
                const uint32_t n_bnd = wr.n - n_own - n_oth;
                L.cnt[wr.slot] = wr.n > NLIST_K ? NL_OVF : (n_own | (n_oth << 10) | (n_bnd << 20));
                if (wr.n > NLIST_K) atomicAdd(&S->n_nl_ovf, 1u);
            } else if (!w) {
                L.cnt[wr.slot] = n_own > NLIST_K ? NL_OVF : n_own;
            }
        } else {
            // boundary: density sums the sets in the order (b, snow, water), lambda (b, water, snow)
            i = t - ns - nd; o = vb.gi[i];
            float3 p = xyz(vb.p4[i]); GCell g = grid_pos(P, p, vb.scene(i));
            const Nbhd nb = make_nbhd(P, g, p, P.h2_cull);
            rho = (P.rho0 * X.bnd.volume[o]) * P.W0;
            acc_WG<LAMBDA>(P, rho, gs, vb, p, nb, i, true, 2, 0.f, sb.mass, X.bnd.mass);
            if (LAMBDA) {
                // one traversal per set for both sums: water first (its lambda terms come
                // before the snow's), its density partials kept aside and added after the
                // snow's, cell by cell in order -- the two orders of the separate passes
                float wpart[27];
                uint32_t wmask = 0;
                acc_WG<true>(P, rho, gs, vs, p, nb, SNOWB_UMAX, false, 0, 0.f, nullptr, nullptr, nullptr, 0, wpart,
                             &wmask);
                acc_WG<true>(P, rho, gs, vd, p, nb, SNOWB_UMAX, false, 0, 0.f, nullptr, nullptr);
                while (wmask) {
                    const int c = __ffs(wmask) - 1;
                    wmask &= wmask - 1u;
                    rho += wpart[c];
                }
            } else {
                float unused = 0.f;
                acc_WG<false>(P, rho, unused, vd, p, nb, SNOWB_UMAX, false, 0, 0.f, nullptr, nullptr);
                acc_WG<false>(P, rho, unused, vs, p, nb, SNOWB_UMAX, false, 0, 0.f, nullptr, nullptr);
            }
            D = &X.bnd; lam_s = sb.lambda;
        }
        D->density[o] = rho;
        float c = (rho / P.rho0) - 1.f;
        c = c > 0.f ? c : 0.f;
        D->C[o] = c;
        if (LAMBDA) {
            float lam = (-c) / (gs + P.eps);
            D->lambda[o] = lam;
            lam_s[i] = lam;
        }
    }
}

// ======================================================== applying a correction
// apply_correction (:1342-1380) for one particle: new and predicted position q + sor * corr,
// the correction cleared, the set marked when the particle left its cell.  Passes that
// finish a particle's correction apply it themselves where k_apply would come next; limits
// carry the reference's launch sizes (Q12).
__device__ __forceinline__ uint32_t launch_limit(const DevParams& P, uint32_t n0, uint32_t n)
{
    return P.quirks == SNOWB_QUIRKS_REFERENCE ? umin32(coverage(n0), n) : n;
}
__device__ __forceinline__ float3 apply_one(const DevParams& P, const snowb_particle_data& D, const SortTrack& T,
                                            uint32_t o, float3 q, float3 corr, uint32_t scene)
{
    const float3 np = add3(q, sc3(P.sor, corr));
    st3(D.new_positions, o, np);
    st3(D.predict_positions, o, np);
    st3(D.correction, o, f3(0.f, 0.f, 0.f));
    if (T.key) track_move(P, T, o, np, scene);
    return np;
}

// ==================================================== PBF + water-side contact corrections
// compute_pbf_sph_correction (:3070-3184) fused with compute_sph_dem_distance_correction
// (:2061-2110) and compute_sph_sph_distance_correction (:2164-2217) for water, and
// compute_pbf_new_dem_correction (:3187-3304) for snow.  Each water particle adds its
// terms to its correction in the reference's kernel order.
struct StageFlags {
    int correct_dem, sph_sph, interlink, step_sph, step_dem;
};
// Water sets up to this size run the water terms one warp per particle (k_pbf_water_warp):
// with few particles one thread each leaves the GPU idle while each thread walks its
// neighbours; above it, threads fill the GPU and the warp form's extra work would cost more.
constexpr uint32_t PBF_WARP_MAX_WATER = 65536;
// apply: as in k_pbf_water_warp, for the water particles this pass takes
__global__ void __launch_bounds__(256) k_pbf(DevParams P, DevState* __restrict__ S, SetView vs, SetView vd,
                                             SetView vb, Sets X, Sorted ss, Sorted sd, Sorted sb, float dt,
                                             StageFlags F, NList L, int apply, SortTrack ts)
{
    const uint32_t ns = S->n_sph, nd = S->n_dem, nb = S->n_b;
    vs.n = ns; vd.n = nd; vb.n = nb;
    const bool ref = P.quirks == SNOWB_QUIRKS_REFERENCE;
    // up to PBF_WARP_MAX_WATER water particles the water terms come from k_pbf_water_warp;
    // the snow particles keep the thread mapping t = ns + i of the reference's launch (its
    // float atomics, Q3, follow it)
    GRID_LOOP(t, ns + nd) {
        if (t < ns) {
            if (ns <= PBF_WARP_MAX_WATER) continue;   // k_pbf_water_warp has them
            const uint32_t i = t, o = vs.gi[i];
            float3 p = xyz(vs.p4[i]); GCell g = grid_pos(P, p, vs.scene(i));
            const float li = ss.lambda[i];
            float3 c = f3(0.f, 0.f, 0.f);
            Seg so, sx, sbn;
            const bool lst = segments(L, i, so, sx, sbn);
            if (lst) {
                c = seg_pbf_own(P, c, so, vs, p, li, ss.lambda, X.sph.lambda, ss.contrib, X.sph.contrib, dt);
                c = seg_pbf_cpl(P, c, sx, vd, p, i, li, sd.lambda, X.dem.lambda, dt);
                c = seg_pbf_bnd(P, c, sbn, vb, p, li, sb.lambda, X.bnd.lambda, dt);
            } else {
                c = acc_pbf_own(P, c, vs, p, g, i, li, ss.lambda, X.sph.lambda, ss.contrib, X.sph.contrib, dt);
                c = acc_pbf_cpl(P, c, vd, p, g, i, li, sd.lambda, X.dem.lambda, dt);
                c = acc_pbf_bnd(P, c, vb, p, g, li, sb.lambda, X.bnd.lambda, dt);
            }
            c = sc3(P.inv_rho0, c);
            const float ci = X.sph.contrib[o];
            c = sc3(ci, c);
            if (nan3(c)) c = f3(0.f, 0.f, 0.f);
            float3 acc = add3(ldv3(X.sph.correction, o), c);
            const float3 z = f3(0.f, 0.f, 0.f);
            const float w0 = X.sph.massInv[o];
            // the contact terms are scaled by (1 - contrib): with contrib == 1 they add a
            // zero to a correction that is never -0 here, which leaves it unchanged
            if (F.correct_dem && ci != 1.f) {     // compute_sph_dem_distance_correction
                float3 d = lst ? seg_contact(P, z, sx, vd, p, w0, sd.invm, X.dem.massInv)
                               : acc_contact(P, z, vd, p, g, SNOWB_UMAX, w0, sd.invm, X.dem.massInv);
                d = sc3(1.f - ci, d);
                if (nan3(d)) d = z;
                acc = add3(acc, sc3(P.k_stretch, d));
            }
            if (F.sph_sph && ci != 1.f) {         // compute_sph_sph_distance_correction
                // pbd_sph_sph_distance_correction (:1586-1646) acts only for contrib <= 0.99
                float3 d = ci <= 0.99f ? acc_contact(P, z, vs, p, g, i, w0, ss.invm, X.sph.massInv) : add3(z, z);
                d = sc3(1.f - ci, d);
                if (nan3(d)) d = z;
                acc = add3(acc, d);
            }
            if (apply && i < launch_limit(P, S->n0_sph, ns)) apply_one(P, X.sph, ts, o, p, acc, vs.scene(i));
            else st3(X.sph.correction, o, acc);
        } else {
            const uint32_t i = t - ns;
            const uint32_t o = ref ? vs.gi[i] : vd.gi[i];   // Q3: SPH grid_index in the reference
            // the snow PBF correction is scaled by (1 - contrib): with contrib == 1 it adds a
            // zero (a NaN or infinity becomes zero too) to the +0 the last apply left
            if (X.dem.contrib[o] == 1.f) continue;
            float3 p = xyz(vd.p4[i]); GCell g = grid_pos(P, p, vd.scene(i));
            const float li = X.dem.lambda[o];
            float3 c = f3(0.f, 0.f, 0.f);
            Seg so, sx, sbn;
            if (segments(L, L.cap + i, so, sx, sbn)) {
                c = seg_pbf_cpl(P, c, sx, vs, p, i, li, ss.lambda, X.sph.lambda, dt);
                if (nan3(c)) c = f3(0.f, 0.f, 0.f);
                c = seg_pbf_own(P, c, so, vd, p, li, sd.lambda, X.dem.lambda, sd.contrib, X.dem.contrib, dt);
                if (nan3(c)) c = f3(0.f, 0.f, 0.f);
                c = seg_pbf_bnd(P, c, sbn, vb, p, li, sb.lambda, X.bnd.lambda, dt);
            } else {
                c = acc_pbf_cpl(P, c, vs, p, g, i, li, ss.lambda, X.sph.lambda, dt);
                if (nan3(c)) c = f3(0.f, 0.f, 0.f);
                c = acc_pbf_own(P, c, vd, p, g, i, li, sd.lambda, X.dem.lambda, sd.contrib, X.dem.contrib, dt);
                if (nan3(c)) c = f3(0.f, 0.f, 0.f);
                c = acc_pbf_bnd(P, c, vb, p, g, li, sb.lambda, X.bnd.lambda, dt);
            }
            if (nan3(c)) c = f3(0.f, 0.f, 0.f);
            c = sc3(P.inv_rho0, c);
            c = sc3(1.f - X.dem.contrib[o], c);
            if (nan3(c)) c = f3(0.f, 0.f, 0.f);
            float* q = reinterpret_cast<float*>(X.dem.correction) + 3ull * o;
            if (ref) {   // targets can repeat in the reference's indexing
                atomicAdd(q, c.x); atomicAdd(q + 1, c.y); atomicAdd(q + 2, c.z);
            } else {
                q[0] += c.x; q[1] += c.y; q[2] += c.z;
            }
        }
    }
    (void)nb;
}

// ============================================================ snow-side corrections
// delete_record (:4624-4658): remove the link from both particles' slot lists.
__device__ __forceinline__ void delete_record(const snowb_particle_data& D, uint32_t M, uint32_t i0, uint32_t i1)
{
    for (uint32_t s = i0 * M; s < (i0 + 1) * M; ++s)
        if (atomicCAS(D.connect_record + s, i1, SNOWB_UMAX) == i1) { atomicExch(D.connect_length + s, 0.f); break; }
    for (uint32_t s = i1 * M; s < (i1 + 1) * M; ++s)
        if (atomicCAS(D.connect_record + s, i0, SNOWB_UMAX) == i0) { atomicExch(D.connect_length + s, 0.f); break; }
}
// compute_dem_sph_distance_correction (:2112-2162) and compute_dem_distance_correction
// (:1765-1834) for snow particle o, added to its correction in the reference's kernel
// order (after the PBF pass; the interlink terms of k_link_sum follow).  SUMS: the two
// contact sums are kept apart instead: sums[2o] the water contact (scaled by k_stretch *
// contrib; +0 without correct_dem), sums[2o+1] the snow-then-boundary contact (scaled by
// contrib).  That pass reads no correction, so it can run beside the snow PBF pass, and
// k_link_apply adds both to the correction after the PBF term, in this order.
template <bool SUMS>
__global__ void __launch_bounds__(256) k_dem_corr(DevParams P, const DevState* __restrict__ S, SetView vs, SetView vd,
                                                  SetView vb, Sets X, Sorted ss, Sorted sd, Sorted sb, StageFlags F,
                                                  NList L, float4* __restrict__ sums)
{
    const uint32_t ns = S->n_sph, nd = S->n_dem, nb = S->n_b;
    vs.n = ns; vd.n = nd; vb.n = nb;
    const float3 z = f3(0.f, 0.f, 0.f);
    GRID_LOOP(i, nd) {
        const uint32_t o = vd.gi[i];
        float3 p = xyz(vd.p4[i]); GCell g = grid_pos(P, p, vd.scene(i));
        const float w0 = X.dem.massInv[o], ci = X.dem.contrib[o];
        float3 acc = SUMS ? z : ldv3(X.dem.correction, o);
        Seg so, sx, sbn;
        const bool lst = segments(L, L.cap + i, so, sx, sbn);
        if (F.correct_dem) {
            float3 d = lst ? seg_contact(P, z, sx, vs, p, w0, ss.invm, X.sph.massInv)
                           : acc_contact(P, z, vs, p, g, SNOWB_UMAX, w0, ss.invm, X.sph.massInv);
            d = sc3(P.k_stretch * ci, d);
            if (nan3(d)) d = z;
            if (SUMS) sums[2 * (size_t)o] = make_float4(d.x, d.y, d.z, 0.f);
            else acc = add3(acc, d);
        } else if (SUMS) {
            sums[2 * (size_t)o] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        {
            float3 d = lst ? seg_contact(P, z, so, vd, p, w0, sd.invm, X.dem.massInv)
                           : acc_contact(P, z, vd, p, g, i, w0, sd.invm, X.dem.massInv);
            d = lst ? seg_contact(P, d, sbn, vb, p, w0, sb.invm, X.bnd.massInv)
                    : acc_contact(P, d, vb, p, g, SNOWB_UMAX, w0, sb.invm, X.bnd.massInv);
            d = sc3(ci, d);
            if (nan3(d)) d = z;
            if (SUMS) sums[2 * (size_t)o + 1] = make_float4(d.x, d.y, d.z, 0.f);
            else st3(X.dem.correction, o, add3(acc, d));
        }
    }
    (void)ns; (void)nb;
}
// solve_snow_interlink_constraint_d (:4742-4765) with compute_interlink_correction
// (:4661-4739), in two passes.  Each particle's slots are summed in slot order, which one
// thread per particle walking its slots does with about 11 dependent link terms in a row
// (a record load, the partner's position, a square root and four divisions each), so the
// pass waited on memory.  Here k_link_terms evaluates every slot's term with one thread per
// slot, all independent, and k_link_sum adds each particle's terms in slot order to its
// correction, after the contact terms as in the reference.  Both ends of a link hold the
// same length and see the same distance, so whichever end breaks it first (delete_record),
// neither adds a correction; a slot whose record a partner has deleted adds nothing, and a
// zero term added to the sum leaves it unchanged (the sum of nonzero terms is never -0), so
// the result does not depend on which thread deletes first.
__device__ __forceinline__ float3 link_term(const DevParams& P, const snowb_particle_data& D, uint32_t i0, uint32_t i1,
                                           float L, uint32_t n)
{
    const float3 z = f3(0.f, 0.f, 0.f);
    if (i0 == i1 || i0 >= n || i1 >= n || L == 0.f) return z;
    const float3 v = sub3(ldv3(D.predict_positions, i0), ldv3(D.predict_positions, i1));
    const float dist = len3(v);
    if (dist > P.brk * L || dist > P.h) { delete_record(D, P.maxc, i0, i1); return z; }
    const float w0 = D.massInv[i0], w1 = D.massInv[i1];
    const float ws = w0 + w1, C = dist - L;
    const float3 n3 = div3(v, dist + P.pbd_eps);
    const float3 r = sc3(((P.k_ref * -w0) * (1.f / ws)) * C, n3);
    // len3(r) > 1 without the square root: sqrtf is monotone and correctly rounded, and the
    // smallest float whose root rounds above 1 is 1 + 2^-22, so the test is d2 > 1 + 2^-23
    if (dot3(r, r) > 0x1.000002p+0f || nan3(r) || inf3(r)) return z;
    return r;
}
// term of slot s: (x, y, z, 1) for a filled slot, w = 0 for an empty one
__global__ void __launch_bounds__(256) k_link_terms(DevParams P, const DevState* __restrict__ S,
                                                    snowb_particle_data dem, float4* __restrict__ terms)
{
    const uint32_t nd = S->n_dem, M = P.maxc;
    // Plain (cached) loads: a record that a partner deletes during the pass is one whose term
    // is zero at both ends, so whether this thread still sees it, or sees its length already
    // zeroed, the term is the same zero.
    GRID_LOOP(s, nd * M) {
        const uint32_t j = dem.connect_record[s];
        float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
        if (j != SNOWB_UMAX) {
            const float3 r = link_term(P, dem, s / M, j, dem.connect_length[s], nd);
            t = make_float4(r.x, r.y, r.z, 1.f);
        }
        terms[s] = t;
    }
}
__global__ void __launch_bounds__(256) k_link_sum(DevParams P, const DevState* __restrict__ S,
                                                  snowb_particle_data dem, const float4* __restrict__ terms)
{
    const uint32_t nd = S->n_dem, M = P.maxc;
    const float3 z = f3(0.f, 0.f, 0.f);
    GRID_LOOP(o, nd) {
        float3 d = z;
        for (uint32_t s = M * o; s < M * (o + 1); ++s) {
            const float4 t = __ldg(terms + s);
            if (t.w != 0.f) d = add3(d, xyz(t));
        }
        if (nan3(d)) d = z;
        st3(dem.correction, o, add3(ldv3(dem.correction, o), d));
    }
}

// The friction pass replays the density+lambda pass's neighbour lists when they still hold
// every contact: the friction sort point kept the snow set's sort (same cells, same order)
// and no snow particle moved more than FR_LIST_MOVE since the lists were built.  A pair
// within 2r now was then within 2r + 2 FR_LIST_MOVE = 0.028 m < h of each other (r = 0.01,
// h = 0.04; the bound is checked against the parameters on the host).
constexpr float FR_LIST_MOVE = 0.004f;

// k_link_sum and the snow part of k_apply in one pass over the sorted snow particles (the
// order k_apply takes them in; o = grid_index[i] runs over the same particles as k_link_sum's
// o): the contact sums and the interlink terms join the correction, which is applied to the
// particles within the launch limit and kept for the others, as k_apply leaves it.
__global__ void __launch_bounds__(256) k_link_apply(DevParams P, DevState* __restrict__ S, SetView vd,
                                                    snowb_particle_data dem, const float4* __restrict__ terms,
                                                    const float4* __restrict__ sums, int correct_dem, int apply,
                                                    SortTrack td)
{
    const uint32_t nd = S->n_dem, M = P.maxc;
    const uint32_t ld = apply ? launch_limit(P, S->n0_dem, nd) : 0u;
    const float3 z = f3(0.f, 0.f, 0.f);
    GRID_LOOP(i, nd) {
        const uint32_t o = vd.gi[i];
        float3 d = z;
        for (uint32_t s = M * o; s < M * (o + 1); ++s) {
            const float4 t = __ldg(terms + s);
            if (t.w != 0.f) d = add3(d, xyz(t));
        }
        if (nan3(d)) d = z;
        float3 acc = ldv3(dem.correction, o);
        if (sums) {
            if (correct_dem) acc = add3(acc, xyz(__ldg(sums + 2 * (size_t)o)));
            acc = add3(acc, xyz(__ldg(sums + 2 * (size_t)o + 1)));
        }
        acc = add3(acc, d);
        if (i < ld) {
            const float3 q = xyz(vd.p4[i]);
            const float3 np = apply_one(P, dem, td, o, q, acc, vd.scene(i));
            const float3 dp = sub3(np, q);
            if (!(dot3(dp, dp) <= FR_LIST_MOVE * FR_LIST_MOVE)) S->far_move = 1u;
        } else {
            st3(dem.correction, o, acc);
        }
    }
}


// ======================================================================= apply
// apply_correction (:1342-1380); limits carry the reference's launch sizes (Q12).
// ts, td: a particle that leaves its cell marks its set for a full sort at the next sort
// point (key null: not tracked).
__global__ void k_apply(DevParams P, DevState* __restrict__ S, SetView vs, SetView vd, Sets X, int do_sph,
                        int do_dem, SortTrack ts, SortTrack td)
{
    const uint32_t ls = do_sph ? launch_limit(P, S->n0_sph, S->n_sph) : 0u;
    const uint32_t ld = do_dem ? launch_limit(P, S->n0_dem, S->n_dem) : 0u;
    GRID_LOOP(t, ls + ld) {
        const bool w = t < ls;
        const uint32_t i = w ? t : t - ls;
        const SetView& v = w ? vs : vd;
        const snowb_particle_data& D = w ? X.sph : X.dem;
        const uint32_t o = v.gi[i];
        const float3 q = xyz(v.p4[i]);
        const float3 np = apply_one(P, D, w ? ts : td, o, q, ldv3(D.correction, o), v.scene(i));
        if (!w) {
            const float3 dp = sub3(np, q);
            if (!(dot3(dp, dp) <= FR_LIST_MOVE * FR_LIST_MOVE)) S->far_move = 1u;
        }
    }
}

// ==================================================================== friction
// compute_friction_correction (:1989-2059) with pbd_friction_correction{,_boundary}
// (:1836-1987); overwrites the correction.
__device__ __forceinline__ float3 friction_term(const DevParams& P, float3 dx, float w0, float w1, float d, float3 v)
{
    float ws = w0 + w1;
    float3 n = div3(v, d + P.pbd_eps);
    float pen = P.two_r - d;
    float3 dxt = sub3(dx, sc3(dot3(dx, n), n));
    float thr = P.mu_s * pen;
    float len = len3(dxt);
    if (len3(dxt) > thr) {
        float c = fminf((P.mu_k * pen) / (len + 0.000001f), 1.f);
        dxt = sc3(c, dxt);
    }
    return sc3(-(w0 / ws), dxt);
}
// Two phases per set: the candidate scan records the contacts (d <= 2r, a few per
// particle) with their cell in shared memory, then the friction terms are evaluated over
// the record with the per-cell partial sums closed where the cell changes (cells without
// contacts add +0 in the traversal, which leaves the sum unchanged).  The lanes of a warp
// then evaluate the costly term together instead of once per lane that found a contact.
// More than FR_K contacts fall back to the single traversal.
constexpr uint32_t FR_K = 16;
// lists: the replay of the neighbour lists is allowed (see FR_LIST_MOVE); each particle
// then takes its snow and boundary contacts from its list entries, in list order, instead
// of traversing the cells (same contacts, same order: the list holds every candidate with
// d < h in traversal order with its cell).
// APPLY: the friction correction is applied at once (the snow part of k_apply, whose
// position it reads is this pass's p: new and predicted positions, a zero correction, the
// moved mark of the set), without k_apply's far-move flag, which the next density+lambda
// pass clears before any friction pass reads it.
template <bool APPLY>
__global__ void __launch_bounds__(256) k_friction(DevParams P, const DevState* __restrict__ S, SetView vd, SetView vb,
                                                  Sets X, Sorted sd, Sorted sb, NList L, int lists, SortTrack td)
{
    __shared__ uint32_t rec_sh[FR_K * 256];
    uint32_t* const rec = rec_sh + threadIdx.x;     // entry k at rec[k * blockDim.x]
    const uint32_t bd = blockDim.x;
    vd.n = S->n_dem; vb.n = S->n_b;
    const uint32_t ld = launch_limit(P, S->n0_dem, S->n_dem);
    const bool list_ok = lists && S->resort[1] == 0u && S->far_move == 0u;
    GRID_LOOP(i, ld) {
        const uint32_t o = vd.gi[i];
        float3 p = xyz(vd.p4[i]);
        float3 op0 = ldv3(X.dem.positions, o);
        const float w0 = X.dem.massInv[o];
        Seg so, sx, sbn;
        const bool use_list = list_ok && segments(L, L.cap + i, so, sx, sbn);
        const Nbhd nb = use_list ? Nbhd{} : make_nbhd(P, grid_pos(P, p, vd.scene(i)), p, P.r2_cull);
        float3 c = f3(0.f, 0.f, 0.f);
        // snow-snow contacts (current entries screened two at a time with packed arithmetic
        // against the slightly larger r2_cull, then the exact scalar test, as in the density
        // pass)
        const P2 pp = bcast2(p);
        uint32_t n = 0;
        auto record = [&](uint32_t j, uint32_t cell) {
            if (n < FR_K) rec[n * bd] = j | (cell << 25);
            ++n;
        };
        if (use_list) {
            for (uint32_t k = so.k0; k < so.k1; ++k) {
                const uint32_t en = so.at(k), j = en & NL_J_MASK;
                const float3 v = sub3(p, vd.pos(j));
                if (dot3(v, v) < P.r2_le) record(j, (en >> 25) & 31u);
            }
        } else FOR27 {
            uint32_t s, e;
            if (vd.range_nb(nb, ox, oy, oz, s, e)) {
                const uint32_t cell = (uint32_t)CELL27;
                if (e <= vd.n) {
                    uint32_t j = s;
                    for (; j + 1 < e; j += 2) {
                        const float4 q0 = __ldg(vd.p4 + j), q1 = __ldg(vd.p4 + j + 1);
                        const float2 dd = d2_pair(pp, q0, q1);
                        if (dd.x < P.r2_cull && j != i) {
                            const float3 v = sub3(p, xyz(q0));
                            if (dot3(v, v) < P.r2_le) record(j, cell);
                        }
                        if (dd.y < P.r2_cull && j + 1 != i) {
                            const float3 v = sub3(p, xyz(q1));
                            if (dot3(v, v) < P.r2_le) record(j + 1, cell);
                        }
                    }
                    if (j < e && j != i) {
                        const float3 v = sub3(p, vd.pos(j));
                        if (dot3(v, v) < P.r2_le) record(j, cell);
                    }
                } else {
                    for (uint32_t j = s; j < e; ++j) {
                        if (j == i) continue;
                        const float3 v = sub3(p, vd.pos(j));
                        if (dot3(v, v) < P.r2_le) record(j, cell);
                    }
                }
            }
        }
        if (n <= FR_K) {
            float3 cs = f3(0.f, 0.f, 0.f);
            uint32_t cur = 0xFFu;
            for (uint32_t k = 0; k < n; ++k) {
                const uint32_t en = rec[k * bd], j = en & NL_J_MASK, cell = en >> 25;
                if (cell != cur) { if (cur != 0xFFu) c = add3(c, cs); cs = f3(0.f, 0.f, 0.f); cur = cell; }
                const float3 pp1 = vd.pos(j);
                const float3 v = sub3(p, pp1);
                const float d2 = dot3(v, v);
                const float3 op1 = ldv3(X.dem.positions, vd.gi[j]);
                const float3 dx = add3(sub3(p, op0), sub3(pp1, op1));
                cs = add3(cs, friction_term(P, dx, w0, vd.attr(sd.invm, X.dem.massInv, j), sqrtf(d2), v));
            }
            if (cur != 0xFFu) c = add3(c, cs);
        } else {   // more contacts than the record holds: the traversal evaluates them
            const Nbhd nbf = use_list ? make_nbhd(P, grid_pos(P, p, vd.scene(i)), p, P.r2_cull) : nb;
            FOR27 {
                float3 cs = f3(0.f, 0.f, 0.f);
                uint32_t s, e;
                if (vd.range_nb(nbf, ox, oy, oz, s, e))
                    for (uint32_t j = s; j < e; ++j) {
                        if (j == i) continue;
                        float3 pp1 = vd.pos(j);
                        float3 v = sub3(p, pp1);
                        float d2 = dot3(v, v);
                        if (d2 < P.r2_le) {
                            const uint32_t oj = vd.gi[j];
                            float3 op1 = ldv3(X.dem.positions, oj);
                            float3 dx = add3(sub3(p, op0), sub3(pp1, op1));
                            cs = add3(cs, friction_term(P, dx, w0, vd.attr(sd.invm, X.dem.massInv, j), sqrtf(d2), v));
                        }
                    }
                c = add3(c, cs);
            }
        }
        // snow-boundary contacts
        n = 0;
        if (use_list) {
            for (uint32_t k = sbn.k0; k < sbn.k1; ++k) {
                const uint32_t en = sbn.at(k), j = en & NL_J_MASK;
                const float3 v = sub3(p, vb.pos(j));
                if (dot3(v, v) < P.r2_le) record(j, (en >> 25) & 31u);
            }
        } else FOR27 {
            uint32_t s, e;
            if (vb.range_nb(nb, ox, oy, oz, s, e)) {
                const uint32_t cell = (uint32_t)CELL27;
                if (e <= vb.n) {
                    uint32_t j = s;
                    for (; j + 1 < e; j += 2) {
                        const float4 q0 = __ldg(vb.p4 + j), q1 = __ldg(vb.p4 + j + 1);
                        const float2 dd = d2_pair(pp, q0, q1);
                        if (dd.x < P.r2_cull) {
                            const float3 v = sub3(p, xyz(q0));
                            if (dot3(v, v) < P.r2_le) record(j, cell);
                        }
                        if (dd.y < P.r2_cull) {
                            const float3 v = sub3(p, xyz(q1));
                            if (dot3(v, v) < P.r2_le) record(j + 1, cell);
                        }
                    }
                    if (j < e) {
                        const float3 v = sub3(p, vb.pos(j));
                        if (dot3(v, v) < P.r2_le) record(j, cell);
                    }
                } else {
                    for (uint32_t j = s; j < e; ++j) {
                        const float3 v = sub3(p, vb.pos(j));
                        if (dot3(v, v) < P.r2_le) record(j, cell);
                    }
                }
            }
        }
        const float3 dx0 = sub3(p, op0);
        if (n <= FR_K) {
            float3 cs = f3(0.f, 0.f, 0.f);
            uint32_t cur = 0xFFu;
            for (uint32_t k = 0; k < n; ++k) {
                const uint32_t en = rec[k * bd], j = en & NL_J_MASK, cell = en >> 25;
                if (cell != cur) { if (cur != 0xFFu) c = add3(c, cs); cs = f3(0.f, 0.f, 0.f); cur = cell; }
                const float3 v = sub3(p, vb.pos(j));
                const float d2 = dot3(v, v);
                cs = add3(cs, friction_term(P, dx0, w0, vb.attr(sb.invm, X.bnd.massInv, j), sqrtf(d2), v));
            }
            if (cur != 0xFFu) c = add3(c, cs);
        } else {
            const Nbhd nbf = use_list ? make_nbhd(P, grid_pos(P, p, vd.scene(i)), p, P.r2_cull) : nb;
            FOR27 {
                float3 cs = f3(0.f, 0.f, 0.f);
                uint32_t s, e;
                if (vb.range_nb(nbf, ox, oy, oz, s, e))
                    for (uint32_t j = s; j < e; ++j) {
                        float3 v = sub3(p, vb.pos(j));
                        float d2 = dot3(v, v);
                        if (d2 < P.r2_le)
                            cs = add3(cs, friction_term(P, dx0, w0, vb.attr(sb.invm, X.bnd.massInv, j), sqrtf(d2), v));
                    }
                c = add3(c, cs);
            }
        }
        if (nan3(c)) c = f3(0.f, 0.f, 0.f);
        if (APPLY) {
            apply_one(P, X.dem, td, o, p, c, vd.scene(i));
        } else {
            st3(X.dem.correction, o, c);
        }
    }
}

// =================================================================== integrate
// integrate_pbd_cd_d (:467-540) / integrate_pbd_d (:447-465).  The reference kernel has no
// bounds check, so it runs over its whole launch (clamped to the allocation here).
__device__ __forceinline__ void integrate_one(const DevParams& P, const snowb_particle_data& D, uint32_t i, float dt,
                                              int cd_on)
{
    float3 tv = add3(ldv3(D.velocity, i), f3(dt * P.gx, dt * P.gy, dt * P.gz));
    tv = f3(tv.x * P.damping, tv.y * P.damping, tv.z * P.damping);
    float3 pos = ldv3(D.positions, i);
    if (!cd_on) {
        float3 pp = add3(pos, sc3(dt, tv));
        st3(D.predict_positions, i, pp);
        st3(D.velocity, i, tv);
        st3(D.new_positions, i, pp);
        return;
    }
    float3 tp = add3(pos, sc3(dt, tv));
    if (tp.x + P.r >= P.wx1) { tv.x = -fabsf(tv.x); tv = sc3(P.b_damping, tv); }
    if (tp.x - P.r <= P.wx0) { tv.x = fabsf(tv.x); tv = sc3(P.b_damping, tv); }
    if (tp.z + P.r >= P.wz1) { tv.z = -fabsf(tv.z); tv = sc3(P.b_damping, tv); }
    if (tp.z - P.r <= P.wz0) { tv.z = fabsf(tv.z); tv = sc3(P.b_damping, tv); }
    if (pos.y - P.r <= P.floor_y) {
        pos.y = P.floor_y + P.r;
        reinterpret_cast<float*>(D.positions)[3ull * i + 1] = pos.y;
        tv.y = fabsf(tv.y);
        tv = sc3(P.b_damping, tv);
    }
    if (len3(tv) > P.max_speed) tv = sc3(P.max_speed / len3(tv), tv);
    float3 pp = add3(pos, sc3(dt, tv));
    st3(D.predict_positions, i, pp);
    st3(D.velocity, i, tv);
    st3(D.new_positions, i, pp);
    float c = D.contrib[i];
    if (c < 0.99f) c += P.blending;
    if (c >= 0.99f) c = 1.f;
    D.contrib[i] = c;
}
// ts, td: a particle of the last sort (i < n) that leaves its cell marks its set for a
// full sort at the next sort point (key null: not tracked)
__global__ void k_integrate(DevParams P, const DevState* __restrict__ S, Sets X, uint32_t full, float dt, int cd_on,
                            int do_sph, int do_dem, SortTrack ts, SortTrack td)
{
    const bool ref = P.quirks == SNOWB_QUIRKS_REFERENCE;
    const uint32_t ns = S->n_sph, nd = S->n_dem;
    const uint32_t ls = do_sph ? (ref ? umin32(coverage(ns), full) : ns) : 0u;
    const uint32_t ld = do_dem ? (ref ? umin32(coverage(nd), full) : nd) : 0u;
    GRID_LOOP(t, ls + ld) {
        const bool w = t < ls;
        const uint32_t i = w ? t : t - ls;
        const snowb_particle_data& D = w ? X.sph : X.dem;
        integrate_one(P, D, i, dt, cd_on);
        const SortTrack& T = w ? ts : td;
        if (T.key && i < (w ? ns : nd))
            track_move(P, T, i, ldv3(D.predict_positions, i), T.sid ? __ldg(T.sid + i) : 0u);
    }
}

// ==================================================================== finalize
// finalize_correction (:1383-1408)
__global__ void k_finalize(DevParams P, const DevState* __restrict__ S, Sets X, float dt, int do_sph, int do_dem)
{
    const uint32_t ls = do_sph ? launch_limit(P, S->n0_sph, S->n_sph) : 0u;
    const uint32_t ld = do_dem ? launch_limit(P, S->n0_dem, S->n_dem) : 0u;
    GRID_LOOP(t, ls + ld) {
        const bool w = t < ls;
        const uint32_t i = w ? t : t - ls;
        const snowb_particle_data& D = w ? X.sph : X.dem;
        float3 np = ldv3(D.new_positions, i);
        float3 diff = sub3(np, ldv3(D.positions, i));
        float3 tv = len3(diff) >= P.min_speed ? div3(diff, dt) : f3(0.f, 0.f, 0.f);
        st3(D.velocity, i, tv);
        st3(D.positions, i, np);
    }
}

// ======================================================================== heat
// heat_transfer_cell (:3764-3810) over one cell
__device__ __forceinline__ float heat_cell(const DevParams& P, const SetView& v, const snowb_particle_data& O,
                                           GCell g, int ox, int oy, int oz, uint32_t skip, float3 p, float Ti,
                                           float kk)
{
    float res = 0.f;
    uint32_t s, e;
    if (v.range(P, g, ox, oy, oz, s, e))
        for (uint32_t j = s; j < e; ++j) {
            if (j == skip) continue;
            float3 dv = sub3(p, v.pos(j));
            float d2 = dot3(dv, dv);
            if (d2 < P.h2_lt) {
                const uint32_t oj = v.gi[j];
                res += (((O.mass[oj] / O.density[oj]) * kk) * (O.T[oj] - Ti)) * L_visc(P, sqrtf(d2));
            }
        }
    return res;
}
__device__ __forceinline__ float heat_sum(const DevParams& P, float dT, const SetView& v, const snowb_particle_data& O,
                                          GCell g, uint32_t skip, float3 p, float Ti, float kk)
{
    if (P.quirks == SNOWB_QUIRKS_REFERENCE) {
        // Q7: the reference passes the particle's own cell to all 27 calls
        const float s = heat_cell(P, v, O, g, 0, 0, 0, skip, p, Ti, kk);
        for (int k = 0; k < 27; ++k) dT += s;
        return dT;
    }
    FOR27 dT += heat_cell(P, v, O, g, ox, oy, oz, skip, p, Ti, kk);
    return dT;
}
// transfer_heat_sph / transfer_heat_dem (:3812-3937): new_T from T
__global__ void __launch_bounds__(256) k_heat(DevParams P, const DevState* __restrict__ S, SetView vs, SetView vd,
                                              Sets X, float dt)
{
    const uint32_t ns = S->n_sph, nd = S->n_dem;
    vs.n = ns; vd.n = nd;
    const float kww = ((4.f * P.k_water) * P.k_water) / (P.k_water + P.k_water);
    const float kss = ((4.f * P.k_snow) * P.k_snow) / (P.k_snow + P.k_snow);
    const float kws = ((4.f * P.k_water) * P.k_snow) / (P.k_water + P.k_snow);
    const float ksw = ((4.f * P.k_snow) * P.k_water) / (P.k_snow + P.k_water);
    GRID_LOOP(t, ns + nd) {
        const bool w = t < ns;
        const uint32_t i = w ? t : t - ns;
        const SetView& own = w ? vs : vd;
        const SetView& oth = w ? vd : vs;
        const snowb_particle_data& A = w ? X.sph : X.dem;
        const snowb_particle_data& B = w ? X.dem : X.sph;
        const uint32_t o = own.gi[i];
        float3 p = xyz(own.p4[i]); GCell g = grid_pos(P, p, own.scene(i));
        const float Ti = A.T[o];
        float dT = 0.f;
        dT = heat_sum(P, dT, own, A, g, i, p, Ti, w ? kww : kss);
        dT = heat_sum(P, dT, oth, B, g, SNOWB_UMAX, p, Ti, w ? kws : ksw);
        dT = dT / ((w ? P.C_water : P.C_snow) * A.density[o]);
        A.new_T[o] = Ti + dT * dt;
    }
}
// thrust::copy new_T -> T (:3968-3969) then environmental_heat_transfer (:4847-4859)
__global__ void k_heat_commit(const DevState* __restrict__ S, Sets X, float dTe, int env_sph, int env_dem)
{
    const uint32_t ns = S->n_sph, nd = S->n_dem;
    GRID_LOOP(t, ns + nd) {
        const bool w = t < ns;
        const uint32_t i = w ? t : t - ns;
        const snowb_particle_data& D = w ? X.sph : X.dem;
        float T = D.new_T[i];
        if (w ? env_sph : env_dem) T += dTe;
        D.T[i] = T;
    }
}

// ======================================================================== XSPH
// xsph_viscosity_cell{,_coupling} (:3419-3502): sum of (m_j/rho_j) (v_j - v_i) W, and
// xsph_sph_viscosity / xsph_dem_viscosity (:3504-3660), Jacobi: results go to out_vel
// (`limit`, the number of sorted particles processed, carries Q6 for the snow set).
// One warp per particle: lane k < 27 computes the partial sum of cell k (the reference's
// per-cell helper), then the partials are added to the running total in cell order with
// shuffles -- the same operations in the same order as one thread would do, with 27-way
// parallelism for the small sets XSPH works on.
// Most cells hold no neighbour of a given kind, and their partial is +0 in every component.
// Adding +0 leaves a float as it is, except -0, which becomes +0 (round to nearest), and
// doing it again changes nothing; so each run of +0 partials is replaced by one addition
// of +0, and only the other partials are fetched and added, in cell order.  (A NaN in the
// total comes from arithmetic here and is already the canonical NaN that +0 keeps.)
__device__ __forceinline__ float3 warp_ordered_sum(float3 acc, float3 part)
{
    const bool nz = (__float_as_uint(part.x) | __float_as_uint(part.y) | __float_as_uint(part.z)) != 0u;
    uint32_t m = __ballot_sync(0xffffffffu, nz) & ((1u << 27) - 1u);
    const float3 zero = f3(0.f, 0.f, 0.f);
    int next = 0;   // cells before `next` are in the total
    while (m) {
        const int k = __ffs(m) - 1;
        m &= m - 1u;
        if (k > next) acc = add3(acc, zero);   // the +0 partials of cells next .. k-1
        float3 v;
        v.x = __shfl_sync(0xffffffffu, part.x, k);
        v.y = __shfl_sync(0xffffffffu, part.y, k);
        v.z = __shfl_sync(0xffffffffu, part.z, k);
        acc = add3(acc, v);
        next = k + 1;
    }
    if (next < 27) acc = add3(acc, zero);
    return acc;
}

// =============================================== PBF + contact corrections of the water set
// compute_pbf_sph_correction (:3070-3184), compute_sph_dem_distance_correction (:2061-2110)
// and compute_sph_sph_distance_correction (:1586-1646, :2164-2217) for the water particles,
// one warp per particle: lane k < 27 computes the per-cell partial of cell k for each sum
// (own water, coupling to snow, boundary, contacts) and the partials are added in cell
// order with shuffles -- the sums the one-thread loops form, with 27 cells in flight.  The
// water set is small (a few thousand particles at a time), so one thread per particle
// left the GPU nearly idle while each thread walked its neighbours.
// apply: the water part of k_apply follows at once for particles within the launch limit
// (the pass's p is k_apply's sorted position; the correction it would read is acc)
__global__ void __launch_bounds__(256) k_pbf_water_warp(DevParams P, DevState* __restrict__ S, SetView vs,
                                                        SetView vd, SetView vb, Sets X, Sorted ss, Sorted sd,
                                                        Sorted sb, float dt, StageFlags F, int apply, SortTrack ts)
{
    const uint32_t ns = S->n_sph;
    if (ns > PBF_WARP_MAX_WATER) return;   // k_pbf runs the water terms one thread each
    vs.n = ns; vd.n = S->n_dem; vb.n = S->n_b;
    const uint32_t lane = threadIdx.x & 31u;
    const bool cl = lane < 27u;
    const int ox = (int)(lane % 3u) - 1, oy = (int)((lane / 3u) % 3u) - 1, oz = (int)(lane / 9u) - 1;
    const float3 z = f3(0.f, 0.f, 0.f);
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < ns; i += nwarps) {
        const uint32_t o = vs.gi[i];
        const float3 p = xyz(vs.p4[i]);
        const GCell g = grid_pos(P, p, vs.scene(i));
        const float li = ss.lambda[i];
        float3 c = z;
        c = warp_ordered_sum(c, cl ? pbf_own_cell(P, vs, p, g, ox, oy, oz, i, li, ss.lambda, X.sph.lambda, ss.contrib,
                                                  X.sph.contrib, dt) : z);
        c = warp_ordered_sum(c, cl ? pbf_cpl_cell(P, vd, p, g, ox, oy, oz, i, li, sd.lambda, X.dem.lambda, dt) : z);
        c = warp_ordered_sum(c, cl ? pbf_bnd_cell(P, vb, p, g, ox, oy, oz, li, sb.lambda, X.bnd.lambda, dt) : z);
        c = sc3(P.inv_rho0, c);
        const float ci = X.sph.contrib[o];
        c = sc3(ci, c);
        if (nan3(c)) c = z;
        float3 acc = add3(ldv3(X.sph.correction, o), c);
        const float w0 = X.sph.massInv[o];
        // the contact terms are scaled by (1 - contrib): with contrib == 1 they add a zero to
        // a correction that is never -0 here, which leaves it unchanged
        if (F.correct_dem && ci != 1.f) {     // compute_sph_dem_distance_correction
            float3 d = warp_ordered_sum(z, cl ? contact_cell(P, vd, p, g, ox, oy, oz, SNOWB_UMAX, w0, sd.invm,
                                                             X.dem.massInv) : z);
            d = sc3(1.f - ci, d);
            if (nan3(d)) d = z;
            acc = add3(acc, sc3(P.k_stretch, d));
        }
        if (F.sph_sph && ci != 1.f) {         // compute_sph_sph_distance_correction (contrib <= 0.99 only)
            float3 d = ci <= 0.99f
                ? warp_ordered_sum(z, cl ? contact_cell(P, vs, p, g, ox, oy, oz, i, w0, ss.invm, X.sph.massInv) : z)
                : add3(z, z);
            d = sc3(1.f - ci, d);
            if (nan3(d)) d = z;
            acc = add3(acc, d);
        }
        if (lane == 0) {
            if (apply && i < launch_limit(P, S->n0_sph, ns)) apply_one(P, X.sph, ts, o, p, acc, vs.scene(i));
            else st3(X.sph.correction, o, acc);
        }
    }
}
__device__ __forceinline__ float3 xsph_cell(const DevParams& P, const SetView& v, const snowb_particle_data& O,
                                            const snowb_float3* vel, float3 p, GCell g, int ox, int oy, int oz,
                                            uint32_t skip, float3 vi)
{
    float3 cs = f3(0.f, 0.f, 0.f);
    uint32_t s, e;
    if (v.range(P, g, ox, oy, oz, s, e))
        for (uint32_t j = s; j < e; ++j) {
            if (j == skip) continue;
            float3 dv = sub3(p, v.pos(j));
            float d2 = dot3(dv, dv);
            if (d2 < P.h2_lt) {
                const uint32_t oj = v.gi[j];
                float3 vij = sub3(ldv3(vel, oj), vi);
                float a = O.mass[oj] / O.density[oj];
                float wgt = W_poly6(P, sqrtf(d2));
                cs = add3(cs, f3((a * vij.x) * wgt, (a * vij.y) * wgt, (a * vij.z) * wgt));
            }
        }
    return cs;
}
__global__ void __launch_bounds__(256) k_xsph_warp(DevParams P, const DevState* __restrict__ S, SetView vown,
                                                   SetView voth, snowb_particle_data A, snowb_particle_data B,
                                                   int own_is_sph, float visc, snowb_float3* __restrict__ out_vel)
{
    const uint32_t ns = S->n_sph, nd = S->n_dem;
    vown.n = own_is_sph ? ns : nd;
    voth.n = own_is_sph ? nd : ns;
    const uint32_t limit = own_is_sph ? ns
                         : (P.quirks == SNOWB_QUIRKS_REFERENCE ? umin32(coverage(ns), nd) : nd);
    const int lane = threadIdx.x & 31;
    const int ox = lane % 3 - 1, oy = (lane / 3) % 3 - 1, oz = lane / 9 - 1;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = warp; i < limit; i += nwarps) {
        const uint32_t o = vown.gi[i];
        const float3 p = xyz(vown.p4[i]);
        const GCell g = grid_pos(P, p, vown.scene(i));
        const float3 vi = ldv3(A.velocity, o);
        const float3 z = f3(0.f, 0.f, 0.f);
        float3 part = lane < 27 ? xsph_cell(P, vown, A, A.velocity, p, g, ox, oy, oz, i, vi) : z;
        float3 c = warp_ordered_sum(z, part);
        part = lane < 27 ? xsph_cell(P, voth, B, B.velocity, p, g, ox, oy, oz, SNOWB_UMAX, vi) : z;
        c = warp_ordered_sum(c, part);
        c = sc3(visc, c);
        if (lane == 0) st3(out_vel, o, add3(vi, c));
    }
}
// write the Jacobi results back (only the processed particles)
// The same sums with one thread per particle, for sets large enough to fill the GPU with
// threads (the warp form's 27-way split then costs more than it hides): the cell partials
// are added in the same cell order as warp_ordered_sum adds them.
__global__ void __launch_bounds__(256) k_xsph_thread(DevParams P, const DevState* __restrict__ S, SetView vown,
                                                     SetView voth, snowb_particle_data A, snowb_particle_data B,
                                                     int own_is_sph, float visc, snowb_float3* __restrict__ out_vel)
{
    const uint32_t ns = S->n_sph, nd = S->n_dem;
    vown.n = own_is_sph ? ns : nd;
    voth.n = own_is_sph ? nd : ns;
    const uint32_t limit = own_is_sph ? ns
                         : (P.quirks == SNOWB_QUIRKS_REFERENCE ? umin32(coverage(ns), nd) : nd);
    const float3 z = f3(0.f, 0.f, 0.f);
    GRID_LOOP(i, limit) {
        const uint32_t o = vown.gi[i];
        const float3 p = xyz(vown.p4[i]);
        const GCell g = grid_pos(P, p, vown.scene(i));
        const float3 vi = ldv3(A.velocity, o);
        float3 c = z;
        FOR27 c = add3(c, xsph_cell(P, vown, A, A.velocity, p, g, ox, oy, oz, i, vi));
        FOR27 c = add3(c, xsph_cell(P, voth, B, B.velocity, p, g, ox, oy, oz, SNOWB_UMAX, vi));
        c = sc3(visc, c);
        st3(out_vel, o, add3(vi, c));
    }
}
// Sets processed by XSPH above this many particles take the one-thread form.
constexpr uint32_t XSPH_WARP_MAX = 65536;
__global__ void k_xsph_commit(DevParams P, const DevState* __restrict__ S, SetView vown, int own_is_sph,
                              const snowb_float3* __restrict__ in_vel, snowb_float3* __restrict__ vel)
{
    const uint32_t ns = S->n_sph, nd = S->n_dem;
    const uint32_t limit = own_is_sph ? ns
                         : (P.quirks == SNOWB_QUIRKS_REFERENCE ? umin32(coverage(ns), nd) : nd);
    GRID_LOOP(i, limit) {
        const uint32_t o = vown.gi[i];
        st3(vel, o, ldv3(in_vel, o));
    }
}

// ===================================================================== misc
// compute_boundary_volume_d (:303-346) with sph_boundary_volume (:159-192); reads the
// caller's sorted positions directly (one-time setup).
__global__ void k_boundary_volume(DevParams P, snowb_cell_data cd, const float* __restrict__ mass,
                                  float* __restrict__ volume, uint32_t n, const uint32_t* __restrict__ sid_o)
{
    GRID_LOOP(i, n) {
        const uint32_t o = cd.grid_index[i];
        float3 p = ldv3(cd.sorted_pos, i);
        float rho = mass[o] * P.W0;
        GCell g = grid_pos(P, p, sid_o ? sid_o[o] : 0u);
        FOR27 {
            float cs = 0.f;
            uint32_t h = grid_hash(P, g, ox, oy, oz);
            uint32_t s = cd.cell_start[h];
            if (s != SNOWB_EMPTY) {
                uint32_t e = cd.cell_end[h];
                for (uint32_t j = s; j < e; ++j) {
                    if (j == i) continue;
                    float3 dv = sub3(p, ldv3(cd.sorted_pos, j));
                    float d2 = dot3(dv, dv);
                    if (d2 < P.h2_lt) cs += mass[cd.grid_index[j]] * W_poly6(P, sqrtf(d2));
                }
            }
            rho += cs;
        }
        volume[o] = mass[o] / rho;
    }
}
// compact sorted view of the boundary set: p4 = (pos, volume), invm/mass by sorted index
__global__ void k_boundary_prep(snowb_cell_data cd, const float* __restrict__ volume, const float* __restrict__ invm,
                                const float* __restrict__ mass, uint32_t n, float4* __restrict__ p4,
                                float* __restrict__ invm_s, float* __restrict__ mass_s,
                                const uint32_t* __restrict__ sid_o, uint32_t* __restrict__ sid_s)
{
    GRID_LOOP(i, n) {
        const uint32_t o = cd.grid_index[i];
        float3 q = ldv3(cd.sorted_pos, i);
        p4[i] = make_float4(q.x, q.y, q.z, volume[o]);
        invm_s[i] = invm[o];
        mass_s[i] = mass[o];
        if (sid_s) sid_s[i] = sid_o[o];
    }
}
__global__ void k_set_state(DevState* S, uint32_t ns, uint32_t nd, uint32_t nb)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S->n_sph = ns; S->n_dem = nd; S->n_b = nb;
        S->n0_sph = ns; S->n0_dem = nd;
        S->n_freeze = 0; S->n_melt = 0; S->changed = 0; S->new_sph = ns; S->new_dem = nd;
        // the caller may have changed the tail slots between calls: the first compaction
        // of a call cleans the tail as the reference's does every substep
        S->tail_dirty = 1u;
        // ... and the particles: the first sort point of a call sorts both sets in full
        for (int k = 0; k < 2; ++k) { S->moved[k] = 1u; S->sorts_full[k] = 0u; S->sorts_kept[k] = 0u; }
        for (int c = 0; c < 8; ++c) S->sc_count[c] = 0u;
        S->clean_hi[0] = SNOWB_UMAX; S->clean_hi[1] = SNOWB_UMAX;
    }
}
// batched runs: every live slot's scene id must name a scene of the batch
__global__ void k_check_scenes(DevParams P, DevState* S, const uint32_t* __restrict__ sph,
                               const uint32_t* __restrict__ dem, const uint32_t* __restrict__ bnd)
{
    const uint32_t ns = S->n_sph, nd = S->n_dem, nb = S->n_b;
    const uint32_t n = ns > nd ? (ns > nb ? ns : nb) : (nd > nb ? nd : nb);
    GRID_LOOP(i, n) {
        bool bad = (i < ns && sph[i] > P.scene_mask) || (i < nd && dem[i] > P.scene_mask) ||
                   (i < nb && bnd[i] > P.scene_mask);
        if (bad) atomicOr(&S->err, SNOWB_DEVERR_SCENE);
    }
}

// FP64 heat-energy and momentum partial sums (deterministic two-level reduction)
__global__ void k_energy_partial(const snowb_particle_data sph, uint32_t ns, const snowb_particle_data dem,
                                 uint32_t nd, double Cw, double Cs, double* __restrict__ part)
{
    __shared__ double sm[4][256];
    double a[4] = {0, 0, 0, 0};
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < ns + nd; t += gridDim.x * blockDim.x) {
        const bool w = t < ns;
        const uint32_t i = w ? t : t - ns;
        const snowb_particle_data& D = w ? sph : dem;
        double m = (double)D.mass[i];
        float3 v = ldv3(D.velocity, i);
        a[0] += m * (w ? Cw : Cs) * (double)D.T[i];
        a[1] += m * (double)v.x; a[2] += m * (double)v.y; a[3] += m * (double)v.z;
    }
    for (int k = 0; k < 4; ++k) sm[k][threadIdx.x] = a[k];
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st)
            for (int k = 0; k < 4; ++k) sm[k][threadIdx.x] += sm[k][threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) part[4 * blockIdx.x + k] = sm[k][0];
}
__global__ void k_energy_final(const double* __restrict__ part, int nblocks, double* __restrict__ out)
{
    if (threadIdx.x < 4) {
        double s = 0;
        for (int b = 0; b < nblocks; ++b) s += part[4 * b + threadIdx.x];
        out[threadIdx.x] = s;
    }
}

}  // namespace snowb
