// adjoint.cuh -- reverse-mode kernels of the substep (the project's adjoint; the reference
// has none).
//
// The adjoint differentiates the substep as the forward kernels compute it in the fixed
// quirk mode, with every discrete decision of the forward pass held fixed: neighbour sets
// (support tests d < h, d < 2r, d <= 2r), interlink topology (records snapshotted at each
// iteration) and link-breaking masks, the C > 0 clamp, the friction static/kinetic branch,
// wall reflections, the floor clamp and the speed clamp.  No particle changes phase inside
// a differentiated substep and every contrib is 1 (the fields the adjoint assumes).
//
// All adjoint and field arrays are in original index order (like the caller's state); the
// gathers run over the sorted views of the positions being differentiated, exactly like
// the forward neighbour loops.  Every kernel is a gather: a particle accumulates every
// term in which it takes part, from its own constraint and from its neighbours', so no
// atomics are needed except for the scalar parameter gradients.
//
// Notation: r = x_i - x_j, d = |r|.  For a radial vector function F(r) = f(d) r its
// Jacobian is J = f I + (f'(d)/d) r r^T (symmetric, even in r).
#pragma once
#include "common.cuh"
#include "solver.cuh"

namespace snowb {

// fields and their adjoints, one block per particle set (water, snow, boundary)
struct AdjField {
    float *rho, *C, *S, *lam;     // density, constraint, gradient-square sum, lambda
    float *lamb, *rhob, *Sb;      // adjoints of lambda, rho, S
};
// reverse-pass arrays of the water and snow sets (float3 arrays as snowb_float3)
struct AdjSet {
    snowb_float3* xb;     // adjoint of the positions being differentiated
    snowb_float3* u;      // sor * adjoint of the corrected positions (input of the constraint reverse)
    snowb_float3* x0b;    // adjoint of the substep-start positions after integration (friction, finalize)
    const snowb_float3* x0p;   // those positions (tape)
};
// scalar parameter gradients, accumulated in double
struct AdjParams {
    double* g;   // [0] k_refreezing (interlink), [1] k_stretch, [2] k_water, [3] k_snow
};

__device__ __forceinline__ float3 mv3(float a, float3 x, float b, float3 r, float rx)
{
    // (a I + b r r^T) x with rx = r . x
    return f3(a * x.x + b * r.x * rx, a * x.y + b * r.y * rx, a * x.z + b * r.z * rx);
}
// J_spiky(r) y
__device__ __forceinline__ float3 jv_spiky(const DevParams& P, float3 r, float d, float3 y)
{
    const float q = P.h - d, de = d + P.keps;
    const float f = P.spiky_G * (q * q / de);
    const float fp = P.spiky_G * (-2.f * q / de - (q * q) / (de * de));
    const float b = d > 0.f ? fp / d : 0.f;
    return mv3(f, y, b, r, dot3(r, y));
}
// J_poly6-gradient(r) y   (G_poly6 = pG (h^2-d^2)^2 r)
__device__ __forceinline__ float3 jv_gpoly6(const DevParams& P, float3 r, float d, float3 y)
{
    const float q = P.h * P.h - d * d;
    const float f = P.poly6_G * q * q;
    const float b = -4.f * P.poly6_G * q;   // f'(d)/d
    return mv3(f, y, b, r, dot3(r, y));
}
// contact direction phi(r) = (d - 2r)/(d + eps) r and its Jacobian
__device__ __forceinline__ float3 phi_contact(const DevParams& P, float3 r, float d)
{
    return sc3((d - P.two_r) / (d + P.pbd_eps), r);
}
__device__ __forceinline__ float3 jv_contact(const DevParams& P, float3 r, float d, float3 y, float L)
{
    // L = rest length (2r for contact, the link length for interlinks)
    const float de = d + P.pbd_eps;
    const float f = (d - L) / de;
    const float fp = (P.pbd_eps + L) / (de * de);
    const float b = d > 0.f ? fp / d : 0.f;
    return mv3(f, y, b, r, dot3(r, y));
}
// 2 J_spiky(r) G_spiky(r) = d/dr |G_spiky(r)|^2
__device__ __forceinline__ float3 grad_gsq(const DevParams& P, float3 r, float d)
{
    const float3 G = G_spiky(P, r, d);
    return sc3(2.f, jv_spiky(P, r, d, G));
}

// ---------------------------------------------------------------- fields at positions
// density, C, gradient-square sum and lambda of every particle of the three sets (the
// quantities of k_density<true>, fixed quirks), stored in original order.
__global__ void __launch_bounds__(128) ka_fields(DevParams P, uint32_t nw, uint32_t ns, uint32_t nb, SetView vw,
                                                 SetView vs, SetView vb, Sets X, AdjField fw, AdjField fs,
                                                 AdjField fb)
{
    vw.n = nw; vs.n = ns; vb.n = nb;
    GRID_LOOP(t, nw + ns + nb) {
        const int set = t < nw ? 0 : (t < nw + ns ? 1 : 2);
        const uint32_t i = set == 0 ? t : (set == 1 ? t - nw : t - nw - ns);
        const SetView& own = set == 0 ? vw : (set == 1 ? vs : vb);
        const uint32_t o = own.gi[i];
        const float3 p = xyz(own.p4[i]);
        const GCell g = grid_pos(P, p);
        const float wi = set == 2 ? P.rho0 * X.bnd.volume[o] : (set == 0 ? X.sph.mass[o] : X.dem.mass[o]);
        const float mi = set == 0 ? X.sph.mass[o] : (set == 1 ? X.dem.mass[o] : X.bnd.mass[o]);
        float rho = wi * P.W0, S = 0.f;
        for (int k = 0; k < 3; ++k) {
            const SetView& v = k == 0 ? vw : (k == 1 ? vs : vb);
            const bool self = k == set;
            FOR27 {
                uint32_t s, e;
                if (!v.range(P, g, ox, oy, oz, s, e)) continue;
                for (uint32_t j = s; j < e; ++j) {
                    if (self && j == i) continue;
                    const float4 q = v.p4[j];
                    const float3 r = sub3(p, xyz(q));
                    const float d2 = dot3(r, r);
                    if (!(d2 < P.h2_lt)) continue;
                    const float d = sqrtf(d2);
                    const float wj = k == 2 ? P.rho0 * q.w : q.w;
                    rho += wj * W_poly6(P, d);
                    // lambda denominator scale (modes of the three lambda kernels)
                    float sc = P.inv_rho0;
                    if (set != 2 && k == 2) sc = P.inv_rho0 * ((P.rho0 * q.w) / mi);
                    if (set == 2 && k == 2) sc = P.inv_rho0 * ((P.rho0 * q.w) / X.bnd.mass[v.gi[j]]);
                    const float3 G = G_spiky(P, r, d);
                    S += (sc * sc) * dot3(G, G);
                }
            }
        }
        const AdjField& F = set == 0 ? fw : (set == 1 ? fs : fb);
        const float C = (rho / P.rho0) - 1.f > 0.f ? (rho / P.rho0) - 1.f : 0.f;
        F.rho[o] = rho;
        F.C[o] = C;
        F.S[o] = S;
        F.lam[o] = -C / (S + P.eps);
    }
}

// ------------------------------------------------- lambda adjoint from the PBF terms
// lambda-bar of every particle from u (sor times the adjoint of the corrected water
// positions), then C-, S- and rho-bar (rho-bar is added to, so other terms at the same
// positions can be accumulated first).
__global__ void __launch_bounds__(128) ka_pbf_lambar(DevParams P, uint32_t nw, uint32_t ns, uint32_t nb, SetView vw,
                                                     SetView vs, SetView vb, Sets X, AdjField fw, AdjField fs,
                                                     AdjField fb, AdjSet aw)
{
    vw.n = nw; vs.n = ns; vb.n = nb;
    GRID_LOOP(t, nw + ns + nb) {
        const int set = t < nw ? 0 : (t < nw + ns ? 1 : 2);
        const uint32_t i = set == 0 ? t : (set == 1 ? t - nw : t - nw - ns);
        const SetView& own = set == 0 ? vw : (set == 1 ? vs : vb);
        const uint32_t o = own.gi[i];
        const float3 p = xyz(own.p4[i]);
        const GCell g = grid_pos(P, p);
        float lb = 0.f;
        if (set == 0) {
            const float ci = X.sph.contrib[o];
            const float3 ui = ldv3(aw.u, o);
            float acc = 0.f;
            for (int k = 0; k < 3; ++k) {
                const SetView& v = k == 0 ? vw : (k == 1 ? vs : vb);
                FOR27 {
                    uint32_t s, e;
                    if (!v.range(P, g, ox, oy, oz, s, e)) continue;
                    for (uint32_t j = s; j < e; ++j) {
                        if (k == 0 && j == i) continue;
                        const float3 r = sub3(p, xyz(v.p4[j]));
                        const float d2 = dot3(r, r);
                        const float d = sqrtf(d2);
                        if (k == 0 && d2 < P.h2_lt) {
                            const uint32_t oj = v.gi[j];
                            const float cj = X.sph.contrib[oj];
                            const float3 uj = ldv3(aw.u, oj);
                            acc += (ci * cj) * dot3(sub3(ui, uj), G_spiky(P, r, d));
                        } else if (k == 1 && d2 < P.r2_le) {
                            acc += ci * dot3(ui, G_poly6(P, r, d));
                        } else if (k == 2 && d2 < P.h2_lt) {
                            acc += ci * dot3(ui, G_spiky(P, r, d));
                        }
                    }
                }
            }
            lb = acc * P.inv_rho0;
        } else {
            // snow and boundary particles take part in the water particles' PBF sums
            float acc = 0.f;
            FOR27 {
                uint32_t s, e;
                if (!vw.range(P, g, ox, oy, oz, s, e)) continue;
                for (uint32_t j = s; j < e; ++j) {
                    const float3 r = sub3(p, xyz(vw.p4[j]));   // r = x_i - x_k, the water term uses -r
                    const float d2 = dot3(r, r);
                    const uint32_t ok = vw.gi[j];
                    const float ck = X.sph.contrib[ok];
                    const float3 uk = ldv3(aw.u, ok);
                    const float d = sqrtf(d2);
                    if (set == 1 && d2 < P.r2_le) acc -= ck * dot3(uk, G_poly6(P, r, d));
                    if (set == 2 && d2 < P.h2_lt) acc -= ck * dot3(uk, G_spiky(P, r, d));
                }
            }
            lb = acc * P.inv_rho0;
        }
        const AdjField& F = set == 0 ? fw : (set == 1 ? fs : fb);
        const float den = F.S[o] + P.eps;
        const float Cb = -lb / den;
        F.lamb[o] = lb;
        F.Sb[o] = lb * F.C[o] / (den * den);
        if ((F.rho[o] / P.rho0) - 1.f > 0.f) F.rhob[o] += Cb * P.inv_rho0;
    }
}

// ------------------------------------------ position adjoint of one iteration (gather)
// xb (water, snow) += every position derivative at the iteration's input positions: PBF
// direct terms (lambda held), lambda through S and rho, contact terms, and the density
// terms of rho-bar (which also carries the XSPH and heat contributions at these
// positions when they were accumulated before).  pbf != 0 adds the constraint terms;
// pbf == 0 runs the density part alone (heat, substep start).
__global__ void __launch_bounds__(128) ka_pos_rev(DevParams P, uint32_t nw, uint32_t ns, uint32_t nb, SetView vw,
                                                  SetView vs, SetView vb, Sets X, AdjField fw, AdjField fs,
                                                  AdjField fb, AdjSet aw, AdjSet as, AdjParams G, int pbf, int contact)
{
    vw.n = nw; vs.n = ns; vb.n = nb;
    float kst_acc = 0.f;
    GRID_LOOP(t, nw + ns) {
        const int set = t < nw ? 0 : 1;
        const uint32_t i = set == 0 ? t : t - nw;
        const SetView& own = set == 0 ? vw : vs;
        const uint32_t o = own.gi[i];
        const float3 p = xyz(own.p4[i]);
        const GCell g = grid_pos(P, p);
        const AdjField& Fi = set == 0 ? fw : fs;
        const AdjSet& Ai = set == 0 ? aw : as;
        const snowb_particle_data& Di = set == 0 ? X.sph : X.dem;
        const float mi = Di.mass[o], wi_inv = Di.massInv[o], ci = Di.contrib[o];
        const float rhob_i = Fi.rhob[o], Sb_i = Fi.Sb[o];
        const float lam_i = pbf ? Fi.lam[o] : 0.f;
        const float3 ui = pbf ? ldv3(Ai.u, o) : f3(0.f, 0.f, 0.f);
        float3 xb = f3(0.f, 0.f, 0.f);
        float3 kst_dir = f3(0.f, 0.f, 0.f);
        for (int k = 0; k < 3; ++k) {
            const SetView& v = k == 0 ? vw : (k == 1 ? vs : vb);
            const AdjField& Fj = k == 0 ? fw : (k == 1 ? fs : fb);
            const bool self = k == set;
            FOR27 {
                uint32_t s, e;
                if (!v.range(P, g, ox, oy, oz, s, e)) continue;
                for (uint32_t j = s; j < e; ++j) {
                    if (self && j == i) continue;
                    const float4 q = v.p4[j];
                    const float3 r = sub3(p, xyz(q));
                    const float d2 = dot3(r, r);
                    if (!(d2 < P.h2_lt)) continue;
                    const float d = sqrtf(d2);
                    const uint32_t oj = v.gi[j];
                    const float wj = k == 2 ? P.rho0 * q.w : q.w;
                    // density: d rho_i/dx_i = w_j Gp(r); d rho_j/dx_i = w_i Gp(r)
                    xb = add3(xb, sc3(wj * rhob_i + mi * Fj.rhob[oj], G_poly6(P, r, d)));
                    if (!pbf) continue;
                    // S through lambda: s_ij^2 Sbar_i + s_ji^2 Sbar_j
                    {
                        float sij = P.inv_rho0, sji = P.inv_rho0;
                        if (k == 2) sij = P.inv_rho0 * ((P.rho0 * q.w) / mi);
                        const float a = (sij * sij) * Sb_i + (sji * sji) * Fj.Sb[oj];
                        xb = add3(xb, sc3(a, grad_gsq(P, r, d)));
                    }
                    if (set == 0) {
                        // water: PBF own / coupling / boundary terms
                        if (k == 0) {
                            const float cj = X.sph.contrib[oj];
                            const float3 uj = ldv3(aw.u, oj);
                            const float a = (ci * cj) * P.inv_rho0 * (lam_i + Fj.lam[oj]);
                            xb = add3(xb, sc3(a, jv_spiky(P, r, d, sub3(ui, uj))));
                        } else if (k == 1) {
                            if (d2 < P.r2_le) {
                                const float a = ci * P.inv_rho0 * (lam_i + Fj.lam[oj]);
                                xb = add3(xb, sc3(a, jv_gpoly6(P, r, d, ui)));
                            }
                            if (contact && d2 < P.r2_lt) {
                                // snow particle j pushed by this water particle: -k_st c_j kappa_ji Jc u_j
                                const float wj_inv = X.dem.massInv[oj];
                                const float kap = (-wj_inv) * (1.f / (wj_inv + wi_inv));
                                const float a = -(P.k_stretch * X.dem.contrib[oj]) * kap;
                                xb = add3(xb, sc3(a, jv_contact(P, r, d, ldv3(as.u, oj), P.two_r)));
                            }
                        } else {
                            const float a = ci * P.inv_rho0 * (lam_i + Fj.lam[oj]);
                            xb = add3(xb, sc3(a, jv_spiky(P, r, d, ui)));
                        }
                    } else {
                        // snow: coupling term of water neighbours, contact terms
                        if (k == 0) {
                            if (d2 < P.r2_le) {
                                const float ck = X.sph.contrib[oj];
                                const float a = -(ck * P.inv_rho0) * (Fj.lam[oj] + lam_i);
                                xb = add3(xb, sc3(a, jv_gpoly6(P, r, d, ldv3(aw.u, oj))));
                            }
                            if (contact && d2 < P.r2_lt) {
                                const float wj_inv = X.sph.massInv[oj];
                                const float kap = (-wi_inv) * (1.f / (wi_inv + wj_inv));
                                const float a = (P.k_stretch * ci) * kap;
                                xb = add3(xb, sc3(a, jv_contact(P, r, d, ui, P.two_r)));
                                kst_dir = add3(kst_dir, sc3(ci * kap, phi_contact(P, r, d)));
                            }
                        } else if (k == 1) {
                            if (d2 < P.r2_lt) {
                                const float wj_inv = X.dem.massInv[oj];
                                const float kij = ci * ((-wi_inv) * (1.f / (wi_inv + wj_inv)));
                                const float kji = X.dem.contrib[oj] * ((-wj_inv) * (1.f / (wj_inv + wi_inv)));
                                const float3 y = sub3(sc3(kij, ui), sc3(kji, ldv3(as.u, oj)));
                                xb = add3(xb, jv_contact(P, r, d, y, P.two_r));
                            }
                        } else {
                            if (d2 < P.r2_lt) {
                                const float wj_inv = X.bnd.massInv[oj];
                                const float kij = ci * ((-wi_inv) * (1.f / (wi_inv + wj_inv)));
                                xb = add3(xb, jv_contact(P, r, d, sc3(kij, ui), P.two_r));
                            }
                        }
                    }
                }
            }
        }
        st3(Ai.xb, o, add3(ldv3(Ai.xb, o), xb));
        if (set == 1) kst_acc += dot3(ui, kst_dir);
    }
    // k_stretch gradient: warp sum, one atomic per warp
    for (int s = 16; s > 0; s >>= 1) kst_acc += __shfl_down_sync(0xffffffffu, kst_acc, s);
    if ((threadIdx.x & 31) == 0 && kst_acc != 0.f) atomicAdd(G.g + 1, (double)kst_acc);
}

// --------------------------------------------------------------- interlink adjoint
// records snapshotted at the iteration's start; masks of the forward (d <= brk L, d <= h,
// |res| <= 1 per end) recomputed from the same positions.
__device__ __forceinline__ bool link_live(const DevParams& P, float3 r, float d, float L, float wi, float wj,
                                          float3& res)
{
    if (L == 0.f) return false;
    if (d > P.brk * L) return false;
    if (d > P.h) return false;
    const float ws = wi + wj, C = d - L;
    const float3 n3 = div3(r, d + P.pbd_eps);
    res = sc3(((P.k_ref * -wi) * (1.f / ws)) * C, n3);
    if (len3(res) > 1.f || nan3(res) || inf3(res)) return false;
    return true;
}
// Lbar (per slot) accumulates the adjoint of the link's rest length from both ends' terms,
// for the links formed in this substep (their length is the distance at formation).
__global__ void ka_interlink_rev(DevParams P, uint32_t ns, const snowb_float3* __restrict__ x,
                                 const uint32_t* __restrict__ rec, const float* __restrict__ len,
                                 const float* __restrict__ invm, AdjSet as, AdjParams G, float* Lbar)
{
    const uint32_t M = P.maxc;
    float kref_acc = 0.f;
    GRID_LOOP(i, ns) {
        const float3 xi = ldv3(x, i);
        const float3 ui = ldv3(as.u, i);
        const float wi = invm[i];
        float3 xb = f3(0.f, 0.f, 0.f);
        for (uint32_t s = M * i; s < M * (i + 1); ++s) {
            const uint32_t j = rec[s];
            if (j == SNOWB_UMAX || j == i || j >= ns) continue;
            const float L = len[s];
            const float3 r = sub3(xi, ldv3(x, j));
            const float d = len3(r);
            const float wj = invm[j];
            float3 res;
            float lb = 0.f;
            if (link_live(P, r, d, L, wi, wj, res)) {
                const float K = (P.k_ref * -wi) * (1.f / (wi + wj));
                xb = add3(xb, sc3(K, jv_contact(P, r, d, ui, L)));
                if (P.k_ref != 0.f) kref_acc += dot3(ui, res) / P.k_ref;
                lb -= K * dot3(ui, r) / (d + P.pbd_eps);          // d res / dL = -K r / (d + eps)
            }
            // the partner's term on this particle (its own record of the link, same length)
            const float3 rj = sc3(-1.f, r);
            const float3 uj = ldv3(as.u, j);
            float3 resj;
            if (link_live(P, rj, d, L, wj, wi, resj)) {
                const float Kj = (P.k_ref * -wj) * (1.f / (wj + wi));
                xb = sub3(xb, sc3(Kj, jv_contact(P, rj, d, uj, L)));
                lb -= Kj * dot3(uj, rj) / (d + P.pbd_eps);
            }
            Lbar[s] += lb;
        }
        st3(as.xb, i, add3(ldv3(as.xb, i), xb));
    }
    for (int s = 16; s > 0; s >>= 1) kref_acc += __shfl_down_sync(0xffffffffu, kref_acc, s);
    if ((threadIdx.x & 31) == 0 && kref_acc != 0.f) atomicAdd(G.g + 0, (double)kref_acc);
}

// links formed in this substep (slot empty at the substep's start, filled at the first
// iteration): their rest length is |x0_i - x0_j| at the formation positions x0.  Lbar
// carries each slot's rest-length adjoint from later substeps; it is consumed (zeroed)
// here, where the length came into being.
__global__ void ka_linkform_rev(DevParams P, uint32_t ns, const snowb_float3* __restrict__ x0,
                                const uint32_t* __restrict__ rec_pre, const uint32_t* __restrict__ rec0,
                                float* Lbar, snowb_float3* xb)
{
    const uint32_t M = P.maxc;
    GRID_LOOP(i, ns) {
        const float3 xi = ldv3(x0, i);
        float3 acc = f3(0.f, 0.f, 0.f);
        for (uint32_t s = M * i; s < M * (i + 1); ++s) {
            const uint32_t j = rec0[s];
            if (j == SNOWB_UMAX || rec_pre[s] != SNOWB_UMAX || j >= ns) continue;
            const float lb = Lbar[s];
            Lbar[s] = 0.f;
            const float3 r = sub3(xi, ldv3(x0, j));
            const float d = len3(r);
            if (d > 0.f && lb != 0.f) acc = add3(acc, sc3(lb / d, r));
        }
        st3(xb, i, add3(ldv3(xb, i), acc));
    }
}

// ---------------------------------------------------------------- friction adjoint
// vector-Jacobian product of friction_term: ub = adjoint of the result; returns the
// adjoints of dx and of r (the pair vector p_i - p_j).
__device__ __forceinline__ void friction_vjp(const DevParams& P, float3 dx, float w0, float w1, float d, float3 r,
                                             float3 ub, float3& dxb, float3& rb)
{
    const float ws = w0 + w1;
    const float de = d + P.pbd_eps;
    const float3 n = div3(r, de);
    const float pen = P.two_r - d;
    const float dn = dot3(dx, n);
    const float3 dxt = sub3(dx, sc3(dn, n));
    const float len = len3(dxt);
    float3 ab = sc3(-(w0 / ws), ub);   // adjoint of the (scaled) tangential displacement
    float3 tb = ab;                    // adjoint of dxt
    float pen_b = 0.f;
    if (len > P.mu_s * pen) {
        const float den = len + 0.000001f;
        const float c = (P.mu_k * pen) / den;
        if (c < 1.f) {
            const float adt = dot3(ab, dxt);
            tb = sc3(c, ab);
            if (len > 0.f) tb = add3(tb, sc3(-adt * (P.mu_k * pen) / (den * den) / len, dxt));
            pen_b = adt * P.mu_k / den;
        }
    }
    // dxt = dx - (dx.n) n
    const float tn = dot3(tb, n);
    dxb = sub3(tb, sc3(tn, n));
    const float3 nb = sub3(sc3(-tn, dx), sc3(dn, tb));
    // n = r / (d + eps): J_n = I/de - r r^T / (d de^2)
    const float rn = dot3(r, nb);
    rb = sub3(sc3(1.f / de, nb), sc3(d > 0.f ? rn / (d * de * de) : 0.f, r));
    // pen = 2r - d
    if (d > 0.f) rb = sub3(rb, sc3(pen_b / d, r));
}
// snow particles at the friction pass's positions (sorted view vs) and the start
// positions after integration x0p; u = sor * adjoint of the positions after friction.
__global__ void __launch_bounds__(128) ka_friction_rev(DevParams P, uint32_t ns, uint32_t nb, SetView vs, SetView vb,
                                                       Sets X, AdjSet as)
{
    vs.n = ns; vb.n = nb;
    GRID_LOOP(i, ns) {
        const uint32_t o = vs.gi[i];
        const float3 p = xyz(vs.p4[i]);
        const GCell g = grid_pos(P, p);
        const float3 op0 = ldv3(as.x0p, o);
        const float w0 = X.dem.massInv[o];
        const float3 ui = ldv3(as.u, o);
        float3 pb = f3(0.f, 0.f, 0.f), x0b = f3(0.f, 0.f, 0.f);
        FOR27 {
            uint32_t s, e;
            if (!vs.range(P, g, ox, oy, oz, s, e)) continue;
            for (uint32_t j = s; j < e; ++j) {
                if (j == i) continue;
                const float3 pp1 = xyz(vs.p4[j]);
                const float3 r = sub3(p, pp1);
                const float d2 = dot3(r, r);
                if (!(d2 < P.r2_le)) continue;
                const float d = sqrtf(d2);
                const uint32_t oj = vs.gi[j];
                const float3 op1 = ldv3(as.x0p, oj);
                const float w1 = X.dem.massInv[oj];
                const float3 dx = add3(sub3(p, op0), sub3(pp1, op1));
                float3 dxb, rb;
                friction_vjp(P, dx, w0, w1, d, r, ui, dxb, rb);        // term of i
                pb = add3(pb, add3(dxb, rb));
                x0b = sub3(x0b, dxb);
                friction_vjp(P, dx, w1, w0, d, sc3(-1.f, r), ldv3(as.u, oj), dxb, rb);   // term of j
                pb = add3(pb, sub3(dxb, rb));
                x0b = sub3(x0b, dxb);
            }
        }
        FOR27 {
            uint32_t s, e;
            if (!vb.range(P, g, ox, oy, oz, s, e)) continue;
            for (uint32_t j = s; j < e; ++j) {
                const float3 r = sub3(p, xyz(vb.p4[j]));
                const float d2 = dot3(r, r);
                if (!(d2 < P.r2_le)) continue;
                const float d = sqrtf(d2);
                float3 dxb, rb;
                friction_vjp(P, sub3(p, op0), w0, X.bnd.massInv[vb.gi[j]], d, r, ui, dxb, rb);
                pb = add3(pb, add3(dxb, rb));
                x0b = sub3(x0b, dxb);
            }
        }
        st3(as.xb, o, add3(ldv3(as.xb, o), pb));
        st3(as.x0b, o, add3(ldv3(as.x0b, o), x0b));
    }
}

// -------------------------------------------------------------------- XSPH adjoint
// XSPH of set A (own) over A and B with velocities vA, vB, viscosity c; gb = adjoint of
// A's new velocities.  One launch handles both roles: threads [0, nA) are particles of A
// (own sum: velocity, position and density adjoints), threads [nA, nA + nB) particles of
// B (as neighbours of A).  Outputs are added to vbA/vbB (velocity adjoints), xbA/xbB and
// rhobA/rhobB.  A's own velocity adjoint keeps its identity term.
__global__ void __launch_bounds__(128) ka_xsph_rev(DevParams P, uint32_t nA, uint32_t nB, SetView vA, SetView vB,
                                                   const snowb_float3* __restrict__ velA,
                                                   const snowb_float3* __restrict__ velB,
                                                   const float* __restrict__ massA, const float* __restrict__ massB,
                                                   const float* __restrict__ rhoA, const float* __restrict__ rhoB,
                                                   float c, const snowb_float3* __restrict__ gb,
                                                   snowb_float3* vbA, snowb_float3* vbB, snowb_float3* xbA,
                                                   snowb_float3* xbB, float* rhobA, float* rhobB)
{
    vA.n = nA; vB.n = nB;
    GRID_LOOP(t, nA + nB) {
        const bool inA = t < nA;
        const uint32_t i = inA ? t : t - nA;
        const SetView& own = inA ? vA : vB;
        const uint32_t o = own.gi[i];
        const float3 p = xyz(own.p4[i]);
        const GCell g = grid_pos(P, p);
        const float3 vi = ldv3(inA ? velA : velB, o);
        const float mi = (inA ? massA : massB)[o], rhoi = (inA ? rhoA : rhoB)[o];
        const float ai = mi / rhoi;
        float3 vb = f3(0.f, 0.f, 0.f), xb = f3(0.f, 0.f, 0.f);
        float rb = 0.f;
        if (inA) {
            const float3 gi = ldv3(gb, o);
            float wsum = 0.f;
            for (int k = 0; k < 2; ++k) {
                const SetView& v = k == 0 ? vA : vB;
                FOR27 {
                    uint32_t s, e;
                    if (!v.range(P, g, ox, oy, oz, s, e)) continue;
                    for (uint32_t j = s; j < e; ++j) {
                        if (k == 0 && j == i) continue;
                        const float3 r = sub3(p, xyz(v.p4[j]));
                        const float d2 = dot3(r, r);
                        if (!(d2 < P.h2_lt)) continue;
                        const float d = sqrtf(d2);
                        const uint32_t oj = v.gi[j];
                        const float3 vj = ldv3(k == 0 ? velA : velB, oj);
                        const float aj = (k == 0 ? massA : massB)[oj] / (k == 0 ? rhoA : rhoB)[oj];
                        const float W = W_poly6(P, d);
                        wsum += aj * W;
                        // own term: c a_j (v_j - v_i) W(r)
                        xb = add3(xb, sc3(c * aj * dot3(sub3(vj, vi), gi), G_poly6(P, r, d)));
                        if (k == 0) {
                            // i as neighbour j' of A-particle j: c a_i (v_i - v_j) W, adjoint g_j
                            const float3 gj = ldv3(gb, oj);
                            vb = add3(vb, sc3(c * ai * W, gj));
                            xb = add3(xb, sc3(c * ai * dot3(sub3(vi, vj), gj), G_poly6(P, r, d)));
                            rb += -c * (mi / (rhoi * rhoi)) * W * dot3(sub3(vi, vj), gj);
                        }
                    }
                }
            }
            vb = add3(vb, sc3(1.f - c * wsum, gi));
            st3(vbA, o, add3(ldv3(vbA, o), vb));
            st3(xbA, o, add3(ldv3(xbA, o), xb));
            rhobA[o] += rb;
        } else {
            FOR27 {
                uint32_t s, e;
                if (!vA.range(P, g, ox, oy, oz, s, e)) continue;
                for (uint32_t j = s; j < e; ++j) {
                    const float3 r = sub3(p, xyz(vA.p4[j]));
                    const float d2 = dot3(r, r);
                    if (!(d2 < P.h2_lt)) continue;
                    const float d = sqrtf(d2);
                    const uint32_t oj = vA.gi[j];
                    const float3 vj = ldv3(velA, oj);
                    const float3 gj = ldv3(gb, oj);
                    const float W = W_poly6(P, d);
                    vb = add3(vb, sc3(c * ai * W, gj));
                    xb = add3(xb, sc3(c * ai * dot3(sub3(vi, vj), gj), G_poly6(P, r, d)));
                    rb += -c * (mi / (rhoi * rhoi)) * W * dot3(sub3(vi, vj), gj);
                }
            }
            st3(vbB, o, add3(ldv3(vbB, o), vb));
            st3(xbB, o, add3(ldv3(xbB, o), xb));
            rhobB[o] += rb;
        }
    }
}

// -------------------------------------------------------------------- heat adjoint
// T1_i = T_i + dt/(C_i rho_i) sum_j (m_j/rho_j) kh_ij (T_j - T_i) L(d_ij), neighbours in
// both sets (fixed quirks).  Tb = adjoint of T1 in, T0b = adjoint of T out; rho-bar and
// position adjoints added; conductivity gradients accumulated.
__device__ __forceinline__ float kh(float ki, float kj) { return ((4.f * ki) * kj) / (ki + kj); }
__global__ void __launch_bounds__(128) ka_heat_rev(DevParams P, uint32_t nw, uint32_t ns, SetView vw, SetView vs,
                                                   Sets X, const float* __restrict__ Tw, const float* __restrict__ Ts,
                                                   const float* __restrict__ Tbw, const float* __restrict__ Tbs,
                                                   float* T0bw, float* T0bs, AdjField fw, AdjField fs, AdjSet aw,
                                                   AdjSet as, AdjParams G, float dt)
{
    vw.n = nw; vs.n = ns;
    float gkw = 0.f, gks = 0.f;
    GRID_LOOP(t, nw + ns) {
        const int set = t < nw ? 0 : 1;
        const uint32_t i = set == 0 ? t : t - nw;
        const SetView& own = set == 0 ? vw : vs;
        const uint32_t o = own.gi[i];
        const float3 p = xyz(own.p4[i]);
        const GCell g = grid_pos(P, p);
        const float Ti = (set == 0 ? Tw : Ts)[o];
        const float Tbi = (set == 0 ? Tbw : Tbs)[o];
        const float ki = set == 0 ? P.k_water : P.k_snow;
        const float Ci = set == 0 ? P.C_water : P.C_snow;
        const float mi = (set == 0 ? X.sph.mass : X.dem.mass)[o];
        const float rhoi = (set == 0 ? fw.rho : fs.rho)[o];
        const float bi = dt / (Ci * rhoi);
        float T0b = 0.f, lsum = 0.f, dT = 0.f, rb = 0.f;
        float3 xb = f3(0.f, 0.f, 0.f);
        for (int k = 0; k < 2; ++k) {
            const SetView& v = k == 0 ? vw : vs;
            const float kj = k == 0 ? P.k_water : P.k_snow;
            const float Cj = k == 0 ? P.C_water : P.C_snow;
            const float kk = kh(ki, kj);
            // d kh / d k_water and d kh / d k_snow of this pair
            float dkw, dks;
            if (set == k) { dkw = set == 0 ? 2.f : 0.f; dks = set == 1 ? 2.f : 0.f; }
            else {
                const float s2 = (P.k_water + P.k_snow) * (P.k_water + P.k_snow);
                dkw = 4.f * P.k_snow * P.k_snow / s2;
                dks = 4.f * P.k_water * P.k_water / s2;
            }
            FOR27 {
                uint32_t s, e;
                if (!v.range(P, g, ox, oy, oz, s, e)) continue;
                for (uint32_t j = s; j < e; ++j) {
                    if (k == set && j == i) continue;
                    const float3 r = sub3(p, xyz(v.p4[j]));
                    const float d2 = dot3(r, r);
                    if (!(d2 < P.h2_lt)) continue;
                    const float d = sqrtf(d2);
                    const uint32_t oj = v.gi[j];
                    const float Tj = (k == 0 ? Tw : Ts)[oj];
                    const float Tbj = (k == 0 ? Tbw : Tbs)[oj];
                    const float mj = (k == 0 ? X.sph.mass : X.dem.mass)[oj];
                    const float rhoj = (k == 0 ? fw.rho : fs.rho)[oj];
                    const float bj = dt / (Cj * rhoj);
                    const float L = L_visc(P, d);
                    const float aij = (mj / rhoj) * kk, aji = (mi / rhoi) * kk;
                    // temperatures
                    lsum += aij * L;
                    T0b += Tbj * bj * aji * L;
                    dT += aij * (Tj - Ti) * L;
                    // this particle's density in the neighbour's term
                    rb += Tbj * bj * (-(mi / (rhoi * rhoi)) * kk) * (Ti - Tj) * L;
                    // positions through L(d): dL/dx_i = -visc_lap r/d
                    const float a = Tbi * bi * aij * (Tj - Ti) + Tbj * bj * aji * (Ti - Tj);
                    if (d > 0.f) xb = add3(xb, sc3(a * (-P.visc_lap) / d, r));
                    // conductivities (own term only: every pair is counted once per end)
                    const float q = Tbi * bi * (mj / rhoj) * (Tj - Ti) * L;
                    gkw += q * dkw;
                    gks += q * dks;
                }
            }
        }
        T0b += Tbi * (1.f - bi * lsum);
        rb += -Tbi * (bi / rhoi) * dT;
        (set == 0 ? T0bw : T0bs)[o] = T0b;
        (set == 0 ? fw.rhob : fs.rhob)[o] += rb;
        const AdjSet& A = set == 0 ? aw : as;
        st3(A.xb, o, add3(ldv3(A.xb, o), xb));
    }
    for (int s = 16; s > 0; s >>= 1) {
        gkw += __shfl_down_sync(0xffffffffu, gkw, s);
        gks += __shfl_down_sync(0xffffffffu, gks, s);
    }
    if ((threadIdx.x & 31) == 0) {
        if (gkw != 0.f) atomicAdd(G.g + 2, (double)gkw);
        if (gks != 0.f) atomicAdd(G.g + 3, (double)gks);
    }
}

// --------------------------------------------------- integrate / finalize adjoints
// finalize: v = (x_new - x0p)/dt, x = x_new.  xb (in: adjoint of the final positions,
// out: adjoint of x_new), vb in: adjoint of v; x0b -= vb/dt.
__global__ void ka_finalize_rev(uint32_t n, float dt, const snowb_float3* __restrict__ vb, snowb_float3* xb,
                                snowb_float3* x0b)
{
    GRID_LOOP(i, n) {
        const float3 v = div3(ldv3(vb, i), dt);
        st3(xb, i, add3(ldv3(xb, i), v));
        st3(x0b, i, sub3(ldv3(x0b, i), v));
    }
}
// integrate_one with cd_on, branches recomputed from (x0, v0).  In: xpb (adjoint of the
// predicted positions), x0b (adjoint of the positions array after integration).  Out:
// xout (adjoint of x0, added), vout (adjoint of v0, written).
__global__ void ka_integrate_rev(DevParams P, uint32_t n, float dt, int cd_on, const snowb_float3* __restrict__ x0,
                                 const snowb_float3* __restrict__ v0, const snowb_float3* __restrict__ xpb,
                                 const snowb_float3* __restrict__ x0b, snowb_float3* xout, snowb_float3* vout)
{
    GRID_LOOP(i, n) {
        const float3 xp_b = ldv3(xpb, i);
        float3 posb = add3(ldv3(x0b, i), xp_b);
        float3 tb = sc3(dt, xp_b);
        float3 tv = add3(ldv3(v0, i), f3(dt * P.gx, dt * P.gy, dt * P.gz));
        tv = f3(tv.x * P.damping, tv.y * P.damping, tv.z * P.damping);
        const float3 pos = ldv3(x0, i);
        bool floor_fix = false;
        if (cd_on) {
            // forward, remembering each reflection: component, sign source, applied
            float3 st[5];
            int hit[5] = {0, 0, 0, 0, 0};
            const float3 tp = add3(pos, sc3(dt, tv));
            st[0] = tv;
            if (tp.x + P.r >= P.wx1) { hit[0] = 1; tv.x = -fabsf(tv.x); tv = sc3(P.b_damping, tv); }
            st[1] = tv;
            if (tp.x - P.r <= P.wx0) { hit[1] = 1; tv.x = fabsf(tv.x); tv = sc3(P.b_damping, tv); }
            st[2] = tv;
            if (tp.z + P.r >= P.wz1) { hit[2] = 1; tv.z = -fabsf(tv.z); tv = sc3(P.b_damping, tv); }
            st[3] = tv;
            if (tp.z - P.r <= P.wz0) { hit[3] = 1; tv.z = fabsf(tv.z); tv = sc3(P.b_damping, tv); }
            st[4] = tv;
            if (pos.y - P.r <= P.floor_y) { hit[4] = 1; floor_fix = true; tv.y = fabsf(tv.y); tv = sc3(P.b_damping, tv); }
            const float sp = len3(tv);
            if (sp > P.max_speed) {
                const float3 th = div3(tv, sp);
                tb = sc3(P.max_speed / sp, sub3(tb, sc3(dot3(th, tb), th)));
            }
            // reverse through the reflections: tv' = bd * (component sign-flipped)
            if (hit[4]) { tb = sc3(P.b_damping, tb); tb.y *= (st[4].y > 0.f ? 1.f : (st[4].y < 0.f ? -1.f : 0.f)); }
            if (hit[3]) { tb = sc3(P.b_damping, tb); tb.z *= (st[3].z > 0.f ? 1.f : (st[3].z < 0.f ? -1.f : 0.f)); }
            if (hit[2]) { tb = sc3(P.b_damping, tb); tb.z *= (st[2].z > 0.f ? -1.f : (st[2].z < 0.f ? 1.f : 0.f)); }
            if (hit[1]) { tb = sc3(P.b_damping, tb); tb.x *= (st[1].x > 0.f ? 1.f : (st[1].x < 0.f ? -1.f : 0.f)); }
            if (hit[0]) { tb = sc3(P.b_damping, tb); tb.x *= (st[0].x > 0.f ? -1.f : (st[0].x < 0.f ? 1.f : 0.f)); }
        }
        if (floor_fix) posb.y = 0.f;
        st3(vout, i, sc3(P.damping, tb));
        st3(xout, i, add3(ldv3(xout, i), posb));
    }
}
// recording checks: the adjoint assumes contrib == 1 and no phase change
__global__ void ka_check_contrib(uint32_t nw, uint32_t ns, const float* __restrict__ cw, const float* __restrict__ cs,
                                 uint32_t* viol)
{
    GRID_LOOP(t, nw + ns) {
        const float c = t < nw ? cw[t] : cs[t - nw];
        if (c != 1.f) atomicOr(viol, 2u);
    }
}
__global__ void ka_check_phase(const DevState* __restrict__ S, uint32_t* viol)
{
    if (blockIdx.x == 0 && threadIdx.x == 0 && S->changed) atomicOr(viol, 1u);
}
// out = s * a
__global__ void ka_scale3(uint32_t n, snowb_float3* out, float s, const snowb_float3* __restrict__ a)
{
    GRID_LOOP(i, n) st3(out, i, sc3(s, ldv3(a, i)));
}
// out = a + s * b  (float3 arrays, first n entries)
__global__ void ka_axpy3(uint32_t n, snowb_float3* out, const snowb_float3* __restrict__ a, float s,
                         const snowb_float3* __restrict__ b)
{
    GRID_LOOP(i, n) st3(out, i, add3(ldv3(a, i), sc3(s, ldv3(b, i))));
}

}  // namespace snowb
