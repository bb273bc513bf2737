// render.cuh -- headless point-sprite rendering of a particle set (the reference draws its
// particles with point_sprite_vs.glsl / point_sprite_temperature_vs.glsl and
// point_sprite_fs.glsl through OpenGL; here the same vertex and fragment arithmetic runs as
// CUDA kernels into a device image, with no graphics API).
//
// Vertex stage (per particle): clip = projection * view * (x, 1); the point is dropped when
// its centre leaves the clip volume; window position ((ndc + 1) / 2) * (width, height),
// depth (ndc.z + 1) / 2; sprite side point_size / |camera - x| pixels; light direction
// normalize(light_pos - (view * (x, 1)).xyz); colour = point colour, or (temperature
// variant) mix(coolest, hottest, (T - T_cool) / (T_hot - T_cool)).
// Fragment stage (per covered pixel, centres inside the sprite square): point coordinate
// with the upper-left origin, n.xy = 2 pc - 1, n.z = 1 - |n.xy|^2, discarded when negative,
// else n.z = sqrt(n.z); colour = clamp(dot(light_dir, n) * colour, 0, 1), alpha 1.
// Depth test LESS with draw order = particle index: a pixel keeps the smallest
// (depth, draw, index), packed into one 64-bit key so atomicMin resolves it; a second pass
// shades each pixel from its winning particle, so the image does not depend on thread order.
#pragma once
#include "common.cuh"

namespace snowb {

struct RenderCam {
    float V[16], Pm[16];    // column-major view and projection
    float cam[3], light[3];
    float point_size;
    uint32_t W, H;
};
struct RenderColour {
    float rgb[3];
    int temp;               // 1: temperature colours
    float cool[3], hot[3], t_cool, t_hot;
};
__device__ __forceinline__ float4 mat_vec(const float* M, float x, float y, float z, float w)
{
    // column-major: out_r = sum_c M[c*4 + r] v_c, summed in column order
    float4 o;
    o.x = ((M[0] * x + M[4] * y) + M[8] * z) + M[12] * w;
    o.y = ((M[1] * x + M[5] * y) + M[9] * z) + M[13] * w;
    o.z = ((M[2] * x + M[6] * y) + M[10] * z) + M[14] * w;
    o.w = ((M[3] * x + M[7] * y) + M[11] * z) + M[15] * w;
    return o;
}
struct SpriteVtx {
    bool live;
    float xw, yw, depth, side;
    float3 ldir, col;
};
__device__ __forceinline__ SpriteVtx sprite_vertex(const RenderCam& c, const RenderColour& rc, float3 p, float T)
{
    SpriteVtx v;
    const float4 e = mat_vec(c.V, p.x, p.y, p.z, 1.f);
    const float4 cl = mat_vec(c.Pm, e.x, e.y, e.z, e.w);
    v.live = cl.w > 0.f && cl.x >= -cl.w && cl.x <= cl.w && cl.y >= -cl.w && cl.y <= cl.w && cl.z >= -cl.w &&
             cl.z <= cl.w;
    const float nx = cl.x / cl.w, ny = cl.y / cl.w, nz = cl.z / cl.w;
    v.xw = (nx + 1.f) * 0.5f * (float)c.W;
    v.yw = (ny + 1.f) * 0.5f * (float)c.H;
    v.depth = (nz + 1.f) * 0.5f;
    const float3 dv = f3(c.cam[0] - p.x, c.cam[1] - p.y, c.cam[2] - p.z);
    v.side = c.point_size / sqrtf(dot3(dv, dv));
    float3 l = f3(c.light[0] - e.x, c.light[1] - e.y, c.light[2] - e.z);
    const float ll = sqrtf(dot3(l, l));
    v.ldir = f3(l.x / ll, l.y / ll, l.z / ll);
    if (rc.temp) {
        const float a = (T - rc.t_cool) / (rc.t_hot - rc.t_cool);
        v.col = f3(rc.cool[0] * (1.f - a) + rc.hot[0] * a, rc.cool[1] * (1.f - a) + rc.hot[1] * a,
                   rc.cool[2] * (1.f - a) + rc.hot[2] * a);
    } else {
        v.col = f3(rc.rgb[0], rc.rgb[1], rc.rgb[2]);
    }
    return v;
}
// pixel range covered by a sprite: centres px + 0.5 in [xw - side/2, xw + side/2)
__device__ __forceinline__ void sprite_span(float c, float side, uint32_t lim, int& a, int& b)
{
    const float lo = c - 0.5f * side, hi = c + 0.5f * side;
    a = (int)ceilf(lo - 0.5f);
    b = (int)ceilf(hi - 0.5f);   // exclusive
    if (a < 0) a = 0;
    if (b > (int)lim) b = (int)lim;
}
// gl_PointCoord * 2 - 1 of pixel (px, py) in a sprite of side `side` centred at (xw, yw)
// (upper-left point-coordinate origin)
__device__ __forceinline__ void point_coord(float xw, float yw, float side, int px, int py, float& nx, float& ny)
{
    const float pcx = (((float)px + 0.5f) - (xw - 0.5f * side)) / side;
    const float pcy = ((yw + 0.5f * side) - ((float)py + 0.5f)) / side;
    nx = pcx * 2.f - 1.f;
    ny = pcy * 2.f - 1.f;
}
// fragment: false when discarded; shaded colour in rgb
__device__ __forceinline__ bool sprite_fragment(const SpriteVtx& v, int px, int py, float3& rgb)
{
    float nx, ny;
    point_coord(v.xw, v.yw, v.side, px, py, nx, ny);
    float nz = 1.f - (nx * nx + ny * ny);
    if (nz < 0.f) return false;
    nz = sqrtf(nz);
    const float diff = (v.ldir.x * nx + v.ldir.y * ny) + v.ldir.z * nz;
    rgb = f3(fminf(fmaxf(diff * v.col.x, 0.f), 1.f), fminf(fmaxf(diff * v.col.y, 0.f), 1.f),
             fminf(fmaxf(diff * v.col.z, 0.f), 1.f));
    return true;
}
__global__ void kr_depth(RenderCam c, RenderColour rc, const snowb_float3* __restrict__ pos,
                         const float* __restrict__ T, uint32_t n, uint32_t draw,
                         unsigned long long* __restrict__ zbuf)
{
    GRID_LOOP(i, n) {
        const SpriteVtx v = sprite_vertex(c, rc, ldv3(pos, i), T ? T[i] : 0.f);
        if (!v.live) continue;
        int x0, x1, y0, y1;
        sprite_span(v.xw, v.side, c.W, x0, x1);
        sprite_span(v.yw, v.side, c.H, y0, y1);
        uint32_t db;
        memcpy(&db, &v.depth, 4);
        const unsigned long long key = ((unsigned long long)db << 32) | ((unsigned long long)draw << 27) | i;
        for (int py = y0; py < y1; ++py)
            for (int px = x0; px < x1; ++px) {
                float3 rgb;
                if (sprite_fragment(v, px, py, rgb)) atomicMin(zbuf + (size_t)py * c.W + px, key);
            }
    }
}
__global__ void kr_shade(RenderCam c, RenderColour rc, const snowb_float3* __restrict__ pos,
                         const float* __restrict__ T, uint32_t draw, const unsigned long long* __restrict__ zbuf,
                         float* __restrict__ rgba)
{
    GRID_LOOP(k, c.W * c.H) {
        const unsigned long long key = zbuf[k];
        if (key == ~0ull || ((key >> 27) & 31ull) != draw) continue;
        const uint32_t i = (uint32_t)(key & ((1u << 27) - 1u));
        const SpriteVtx v = sprite_vertex(c, rc, ldv3(pos, i), T ? T[i] : 0.f);
        float3 rgb = f3(0.f, 0.f, 0.f);
        sprite_fragment(v, (int)(k % c.W), (int)(k / c.W), rgb);
        rgba[4 * (size_t)k] = rgb.x;
        rgba[4 * (size_t)k + 1] = rgb.y;
        rgba[4 * (size_t)k + 2] = rgb.z;
        rgba[4 * (size_t)k + 3] = 1.f;
    }
}
__global__ void kr_clear(uint32_t npix, unsigned long long* zbuf, float* rgba, float4 clear)
{
    GRID_LOOP(k, npix) {
        zbuf[k] = ~0ull;
        rgba[4 * (size_t)k] = clear.x; rgba[4 * (size_t)k + 1] = clear.y; rgba[4 * (size_t)k + 2] = clear.z;
        rgba[4 * (size_t)k + 3] = clear.w;
    }
}

}  // namespace snowb
