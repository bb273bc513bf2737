// common.cuh -- shared device definitions for libsnowb200 (sm_100a).
//
// Arithmetic contract (identical in the CPU oracle, so results are bit-exact): every
// expression is evaluated as the reference writes it, left to right, each operation
// rounded separately -- dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z as in helper_math.h,
// length = sqrt(dot) -- with correctly rounded sqrt and '/', and no fused multiply-add
// (the library is built with -fmad=false).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/snow_b200.h"

#define SNOWB_EMPTY 0xFFFFFFFFu
#define SNOWB_UMAX 0xFFFFFFFFu

namespace snowb {

// Derived solver constants, passed by value to every kernel.
struct DevParams {
    float h, r, two_r, poly6, poly6_G, spiky_G, visc_lap, keps, pbd_eps;
    float rho0, inv_rho0, eps, scorr_coeff, scorr_div, W0;
    float gx, gy, gz, damping, max_speed, min_speed, b_damping, mu_s, mu_k, k_stretch;
    float k_water, k_snow, C_water, C_snow, Tf, blending, sor, sph_visc, dem_visc;
    float Th, k_ref, brk;
    float ox, oy, oz, csx, csy, csz;
    uint32_t gsx, gsy, gsz, ncells, maxc;
    // Batched scenes: scene s owns the block of sgx x gsy x sgz cells starting at
    // x = (s % batch_nx) * sgx, z = (s / batch_nx) * sgz, and wraps inside it exactly as a
    // single scene wraps in its own grid.  batch_nx = 0: one scene, sgx = gsx, sgz = gsz.
    // batch_nx and the scene count are powers of two; ids are masked into range (an id out
    // of range is reported by k_check_scenes).
    uint32_t sgx, sgz, batch_nx, batch_shift, scene_mask;
    // Exact squared-distance cut-offs: d < h  <=>  d2 < h2_lt, d < 2r <=> d2 < r2_lt,
    // d <= 2r <=> d2 < r2_le, where d = sqrt_rn(d2) (sqrt_rn is monotone).
    float h2_lt, r2_lt, r2_le;
    // box-culling thresholds: the cut-offs with a relative safety margin
    float h2_cull, r2_cull;
    // walls at x = wx0, wx1 and z = wz0, wz1, floor at y = floor_y (the reference: +-1, 0)
    float wx0, wx1, wz0, wz1, floor_y;
    int quirks;
    // scorr_coeff is +0 (the reference's setting) and the s_corr quotient stays finite: the
    // s_corr term is then -0 at every distance inside the support (for dt > 0), and adding
    // -0 leaves a sum unchanged, so the PBF passes do not evaluate it.  scorr_cpl_off: the
    // same for the coupling term of the reference quirk mode, (-scorr_coeff * 0) * x^4 * dt^2,
    // which is -0 whenever scorr_coeff has no sign bit and the quotient stays finite.
    int scorr_off, scorr_cpl_off;
};

// Device-resident counters, one block per library context.
struct DevState {
    uint32_t n_sph, n_dem, n_b;     // current set sizes
    uint32_t n0_sph, n0_dem;        // sizes at the start of the substep (launch sizes)
    uint32_t n_freeze, n_melt;      // particles changing phase in this substep
    uint32_t changed;               // n_freeze + n_melt > 0
    uint32_t new_sph, new_dem;      // sizes after compaction
    uint32_t err;                   // error bits (SNOWB_DEVERR_*)
    uint32_t tail_dirty;            // a link pass wrote slots beyond the snow set (stale cell range)
    uint32_t n_active;              // particles the link prefilter kept for the last link pass
    uint32_t n_links;               // links added by the last link pass
    uint32_t n_nl_ovf;              // neighbour lists that overflowed in the last density+lambda pass
    uint32_t pad;
    // Sort skipping.  moved[k]: set k must be sorted in full at its next sort point (a
    // particle's cell differs from its key at the set's last sort, the set was compacted, or
    // a call started).  resort[k]: the decision of the current sort point, taken from moved
    // by the set's hash pass.  sorts_full/sorts_kept count the decisions since the call
    // started.
    uint32_t moved[2], resort[2];
    uint32_t sorts_full[2], sorts_kept[2];
    // a snow particle moved more than FR_LIST_MOVE since the iteration's neighbour lists
    // were built (set by k_apply, cleared by the density+lambda pass)
    uint32_t far_move;
    uint32_t sc_count[8];           // super-cells listed for each link colour (SCList)
    uint32_t clean_hi[2];           // per set: every slot from here on is clean (k_commit_sizes)
};
#define SNOWB_DEVERR_SCATTER 1u
#define SNOWB_DEVERR_SCENE 2u      // a batched scene id >= the scene count

// ---------------------------------------------------------------- float3 helpers
__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 sc3(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 div3(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Packed two-lane FP32 arithmetic of sm_100 (add/sub/mul.rn.f32x2).  Each instruction alone
// rounds each lane as the scalar operation does, but ptxas contracts a packed multiply
// feeding a packed add into a fused multiply-add even with .rn and -fmad=false (measured:
// about 21% of d2_pair results differ from the separately rounded ones in the last bits),
// so packed results serve only as screens with a margin, never as values.
__device__ __forceinline__ uint64_t pk2(float a, float b)
{
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float2 upk2(uint64_t v)
{
    float a, b;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
    return make_float2(a, b);
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b)
{
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b)
{
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b)
{
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
// p broadcast to both lanes, per coordinate
struct P2 {
    uint64_t x, y, z;
};
__device__ __forceinline__ P2 bcast2(float3 p) { return P2{pk2(p.x, p.x), pk2(p.y, p.y), pk2(p.z, p.z)}; }
// dot3(sub3(p, q0), sub3(p, q0)) and the same for q1, two candidates per instruction, to
// within a few ulps (see above)
__device__ __forceinline__ float2 d2_pair(const P2& p, float4 q0, float4 q1)
{
    const uint64_t dx = sub2(p.x, pk2(q0.x, q1.x));
    const uint64_t dy = sub2(p.y, pk2(q0.y, q1.y));
    const uint64_t dz = sub2(p.z, pk2(q0.z, q1.z));
    return upk2(add2(add2(mul2(dx, dx), mul2(dy, dy)), mul2(dz, dz)));
}
__device__ __forceinline__ float len3(float3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ bool nan3(float3 a) { return isnan(a.x) || isnan(a.y) || isnan(a.z); }
__device__ __forceinline__ bool inf3(float3 a) { return isinf(a.x) || isinf(a.y) || isinf(a.z); }
__device__ __forceinline__ float3 xyz(float4 a) { return f3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 ld3(const snowb_float3* p, uint32_t i)
{
    const float* q = reinterpret_cast<const float*>(p) + 3ull * i;
    return f3(__ldg(q), __ldg(q + 1), __ldg(q + 2));
}
__device__ __forceinline__ float3 ldv3(const snowb_float3* p, uint32_t i)   // plain (non-nc) load
{
    const float* q = reinterpret_cast<const float*>(p) + 3ull * i;
    return f3(q[0], q[1], q[2]);
}
__device__ __forceinline__ void st3(snowb_float3* p, uint32_t i, float3 v)
{
    float* q = reinterpret_cast<float*>(p) + 3ull * i;
    q[0] = v.x; q[1] = v.y; q[2] = v.z;
}

// ------------------------------------------------------------- SPH kernels :30-137
__device__ __forceinline__ float W_poly6(const DevParams& P, float d)
{
    if (d >= 0.f && d < P.h) {
        float h2 = P.h * P.h, d2 = d * d, q = h2 - d2;
        float q3 = q * q * q;
        return P.poly6 * q3;
    }
    return 0.f;
}
__device__ __forceinline__ float3 G_poly6(const DevParams& P, float3 v, float d)
{
    if (d >= 0.f && d < P.h) {
        float h2 = P.h * P.h, d2 = d * d, q = h2 - d2, q2 = q * q;
        return sc3(P.poly6_G * q2, v);
    }
    return f3(0.f, 0.f, 0.f);
}
__device__ __forceinline__ float3 G_spiky(const DevParams& P, float3 v, float d)
{
    if (d >= 0.f && d < P.h) {
        float q = P.h - d, q2 = q * q;
        return sc3(P.spiky_G * (q2 / (d + P.keps)), v);
    }
    return f3(0.f, 0.f, 0.f);
}
__device__ __forceinline__ float L_visc(const DevParams& P, float d)
{
    if (d >= 0.f && d < P.h) return P.visc_lap * (P.h - d);
    return 0.f;
}
__device__ __forceinline__ float scorr_of(const DevParams& P, float d, float dt)
{
    float x = W_poly6(P, d) / P.scorr_div;
    float x4 = (x * x) * (x * x);
    return ((-P.scorr_coeff * x4) * dt) * dt;
}
// s_corr of the coupling term (:982-1034); the reference mode multiplies scorr_coeff by 0
__device__ __forceinline__ float lam_scorr_cpl(const DevParams& P, float lsum, float d, float dt)
{
    const bool ref = P.quirks == SNOWB_QUIRKS_REFERENCE;
    if ((ref ? P.scorr_cpl_off : P.scorr_off) && dt > 0.f) return lsum;
    float x = W_poly6(P, d) / P.scorr_div;
    float x4 = (x * x) * (x * x);
    float sc = ref ? ((((-P.scorr_coeff) * 0.f) * x4) * dt) * dt : ((-P.scorr_coeff * x4) * dt) * dt;
    return lsum + sc;
}
// (li + lj) + s_corr(d), the lambda factor of a PBF term
__device__ __forceinline__ float lam_scorr(const DevParams& P, float lsum, float d, float dt)
{
    return (P.scorr_off && dt > 0.f) ? lsum : lsum + scorr_of(P, d, dt);
}
// W_poly6 and G_spiky for a distance that passed the exact support test (0 <= d < h): the
// same operations without the range test
__device__ __forceinline__ float W_poly6_in(const DevParams& P, float d)
{
    float h2 = P.h * P.h, d2 = d * d, q = h2 - d2;
    float q3 = q * q * q;
    return P.poly6 * q3;
}
__device__ __forceinline__ float3 G_spiky_in(const DevParams& P, float3 v, float d)
{
    float q = P.h - d, q2 = q * q;
    return sc3(P.spiky_G * (q2 / (d + P.keps)), v);
}

// ------------------------------------------------------------------ grid :141-157
// grid cell of a particle: coordinates in its scene (unwrapped) and the scene block base
struct GCell {
    int x, y, z;
    uint32_t bx, bz;
};
__device__ __forceinline__ GCell grid_pos(const DevParams& P, float3 p, uint32_t scene = 0u)
{
    GCell g;
    g.x = __float2int_rz(floorf((p.x - P.ox) / P.csx));
    g.y = __float2int_rz(floorf((p.y - P.oy) / P.csy));
    g.z = __float2int_rz(floorf((p.z - P.oz) / P.csz));
    scene &= P.scene_mask;
    g.bx = (scene & (P.batch_nx - 1u)) * P.sgx;
    g.bz = (scene >> P.batch_shift) * P.sgz;
    return g;
}
// hash of cell g + (dx,dy,dz), each axis wrapped in the scene's grid (calcGridHash :151-157)
__device__ __forceinline__ uint32_t grid_hash(const DevParams& P, GCell g, int dx, int dy, int dz)
{
    uint32_t x = (((uint32_t)g.x + (uint32_t)dx) & (P.sgx - 1u)) + g.bx;
    uint32_t y = ((uint32_t)g.y + (uint32_t)dy) & (P.gsy - 1u);
    uint32_t z = (((uint32_t)g.z + (uint32_t)dz) & (P.sgz - 1u)) + g.bz;
    return (z * P.gsy) * P.gsx + y * P.gsx + x;
}

// launch coverage of the reference's compute_grid_size(n, 512) (:348-357)
__device__ __host__ __forceinline__ uint32_t coverage(uint32_t n)
{
    if (n == 0) return 0;
    uint32_t t = n < 512u ? n : 512u;
    uint32_t b = (n % t) ? n / t + 1 : n / t;
    return b * t;
}
__device__ __host__ __forceinline__ uint32_t umin32(uint32_t a, uint32_t b) { return a < b ? a : b; }
__device__ __host__ __forceinline__ uint32_t umax32(uint32_t a, uint32_t b) { return a > b ? a : b; }

// The 27 neighbour cells of a particle, computed once and shared by every set and pass of
// a kernel: wrapped per-axis hash terms (hash = z term + y term + x term, the value of
// grid_hash) and a mask of the cells whose box lies at squared distance >= cut2 from p
// (bit (oz+1)*9 + (oy+1)*3 + (ox+1)), with the same face arithmetic as range_culled.
struct Nbhd {
    uint32_t x0, x1, x2, y0, y1, y2, z0, z1, z2;   // terms for offsets -1, 0, +1
    uint32_t far;
    __device__ __forceinline__ uint32_t hash(int ox, int oy, int oz) const
    {
        const uint32_t z = oz < 0 ? z0 : (oz > 0 ? z2 : z1);
        const uint32_t y = oy < 0 ? y0 : (oy > 0 ? y2 : y1);
        const uint32_t x = ox < 0 ? x0 : (ox > 0 ? x2 : x1);
        return z + y + x;
    }
};
__device__ __forceinline__ Nbhd make_nbhd(const DevParams& P, GCell g, float3 p, float cut2)
{
    Nbhd nb;
    float lo[3], hi[3];
    const float m = 1e-6f;
    const uint32_t gx = (uint32_t)g.x, gy = (uint32_t)g.y, gz = (uint32_t)g.z, plane = P.gsy * P.gsx;
    nb.x0 = ((gx - 1u) & (P.sgx - 1u)) + g.bx;
    nb.x1 = (gx & (P.sgx - 1u)) + g.bx;
    nb.x2 = ((gx + 1u) & (P.sgx - 1u)) + g.bx;
    nb.y0 = ((gy - 1u) & (P.gsy - 1u)) * P.gsx;
    nb.y1 = (gy & (P.gsy - 1u)) * P.gsx;
    nb.y2 = ((gy + 1u) & (P.gsy - 1u)) * P.gsx;
    nb.z0 = (((gz - 1u) & (P.sgz - 1u)) + g.bz) * plane;
    nb.z1 = ((gz & (P.sgz - 1u)) + g.bz) * plane;
    nb.z2 = (((gz + 1u) & (P.sgz - 1u)) + g.bz) * plane;
    lo[0] = fmaxf((p.x - ((float)g.x * P.csx + P.ox)) - m, 0.f);
    hi[0] = fmaxf((((float)(g.x + 1) * P.csx + P.ox) - p.x) - m, 0.f);
    lo[1] = fmaxf((p.y - ((float)g.y * P.csy + P.oy)) - m, 0.f);
    hi[1] = fmaxf((((float)(g.y + 1) * P.csy + P.oy) - p.y) - m, 0.f);
    lo[2] = fmaxf((p.z - ((float)g.z * P.csz + P.oz)) - m, 0.f);
    hi[2] = fmaxf((((float)(g.z + 1) * P.csz + P.oz) - p.z) - m, 0.f);
    nb.far = 0u;
#pragma unroll
    for (int c = 0; c < 27; ++c) {
        const int ox = c % 3 - 1, oy = (c / 3) % 3 - 1, oz = c / 9 - 1;
        if ((ox | oy | oz) == 0) continue;
        const float gx = ox < 0 ? lo[0] : (ox > 0 ? hi[0] : 0.f);
        const float gy = oy < 0 ? lo[1] : (oy > 0 ? hi[1] : 0.f);
        const float gz = oz < 0 ? lo[2] : (oz > 0 ? hi[2] : 0.f);
        if (gx * gx + gy * gy + gz * gz >= cut2) nb.far |= 1u << c;
    }
    return nb;
}

// Sorted view of one particle set for the 27-cell neighbor loops.  Entries j < n come
// from the compact float4 copy written at the last sort; a stale cell range (cells the
// reference leaves uncleared) may reach j >= n, which reads the caller's arrays exactly
// as the reference does.
struct SetView {
    const uint32_t* cs;     // cell_start
    const uint32_t* ce;     // cell_end
    const uint32_t* gi;     // grid_index (sorted -> original)
    const uint32_t* gh;     // grid_hash (sorted)
    const uint32_t* sid;    // scene id per sorted particle (batched runs only, else null)
    const float4* p4;       // sorted (x, y, z, w) with w = mass (fluid/snow) or volume (boundary)
    const snowb_float3* sp; // caller's sorted_pos (float3)
    const float* wsrc;      // original-order source of the .w attribute (stale path)
    uint32_t n;

    __device__ __forceinline__ float4 pw(uint32_t j) const
    {
        if (j < n) return __ldg(p4 + j);
        float3 q = ld3(sp, j);
        return make_float4(q.x, q.y, q.z, wsrc[gi[j]]);
    }
    __device__ __forceinline__ float3 pos(uint32_t j) const
    {
        if (j < n) { float4 t = __ldg(p4 + j); return f3(t.x, t.y, t.z); }
        return ld3(sp, j);
    }
    // attribute kept in a sorted copy (valid for j < n) with its original-order source
    __device__ __forceinline__ float attr(const float* sorted, const float* orig, uint32_t j) const
    {
        return j < n ? __ldg(sorted + j) : orig[gi[j]];
    }
    __device__ __forceinline__ uint32_t scene(uint32_t i) const { return sid ? __ldg(sid + i) : 0u; }
    __device__ __forceinline__ bool range(const DevParams& P, GCell g, int ox, int oy, int oz,
                                          uint32_t& s, uint32_t& e) const
    {
        uint32_t h = grid_hash(P, g, ox, oy, oz);
        s = __ldg(cs + h);
        if (s == SNOWB_EMPTY) return false;
        e = __ldg(ce + h);
        return true;
    }
    // As range(), but a cell that holds only current members (its first entry is in the
    // current sort and carries its hash) and whose box lies at squared distance >= cut2
    // from p is reported empty: every member is then beyond the support, so all its terms
    // are exact zeros.  Stale ranges (members anywhere) are never culled.
    // range_culled with the neighbourhood precomputed (same culling rule)
    __device__ __forceinline__ bool range_nb(const Nbhd& nb, int ox, int oy, int oz, uint32_t& s, uint32_t& e) const
    {
        const uint32_t h = nb.hash(ox, oy, oz);
        s = __ldg(cs + h);
        if (s == SNOWB_EMPTY) return false;
        e = __ldg(ce + h);
        if ((nb.far >> ((oz + 1) * 9 + (oy + 1) * 3 + (ox + 1))) & 1u)
            if (s < n && __ldg(gh + s) == h) return false;
        return true;
    }
    __device__ __forceinline__ bool range_culled(const DevParams& P, GCell g, int ox, int oy, int oz, float3 p,
                                                 float cut2, uint32_t& s, uint32_t& e) const
    {
        uint32_t h = grid_hash(P, g, ox, oy, oz);
        s = __ldg(cs + h);
        if (s == SNOWB_EMPTY) return false;
        e = __ldg(ce + h);
        if (ox | oy | oz) {
            float gx = 0.f, gy = 0.f, gz = 0.f;
            const float m = 1e-6f;   // covers the rounding of the face coordinates
            if (ox < 0) gx = p.x - ((float)g.x * P.csx + P.ox);
            if (ox > 0) gx = ((float)(g.x + 1) * P.csx + P.ox) - p.x;
            if (oy < 0) gy = p.y - ((float)g.y * P.csy + P.oy);
            if (oy > 0) gy = ((float)(g.y + 1) * P.csy + P.oy) - p.y;
            if (oz < 0) gz = p.z - ((float)g.z * P.csz + P.oz);
            if (oz > 0) gz = ((float)(g.z + 1) * P.csz + P.oz) - p.z;
            gx = fmaxf(gx - m, 0.f); gy = fmaxf(gy - m, 0.f); gz = fmaxf(gz - m, 0.f);
            const float b2 = gx * gx + gy * gy + gz * gz;
            if (b2 >= cut2 && s < n && __ldg(gh + s) == h) return false;
        }
        return true;
    }
};

#define FOR27 _Pragma("unroll 1") for (int oz = -1; oz <= 1; ++oz) _Pragma("unroll 1") for (int oy = -1; oy <= 1; ++oy) _Pragma("unroll 1") for (int ox = -1; ox <= 1; ++ox)

// grid-stride loop over [0, n)
#define GRID_LOOP(i, n) for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

}  // namespace snowb
