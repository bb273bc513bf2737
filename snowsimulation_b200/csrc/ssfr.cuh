// ssfr.cuh -- screen-space fluid rendering as CUDA kernels into device images.  This is the
// reference's default view (Renderer::Render with m_b_render_fluid, Renderer.cpp:92-109):
// snow drawn as point sprites into a scene image, the water's sphere depth, smoothed by a
// separable bilateral filter, its additive thickness, and a full-screen composite that
// refracts the scene through the water surface.  Same arithmetic as the shaders, no graphics
// API; every image is width x height, row 0 at the bottom as in a GL framebuffer.
//
//  - sphere depth (point_depth_vs.glsl / point_depth_fs.glsl, Renderer::RenderSceneDepth
//    :404-483 for the snow, RenderFluidDepth :485-540 for the water): clip = PV (x, 1),
//    sprite side point_size / clip.w, eye = V (x, 1); per covered pixel n.xy = 2 pc - 1,
//    discarded when |n.xy|^2 > 1, n.z = sqrt(1 - |n.xy|^2); depth = (P (eye + r n, 1)).z / .w
//    written as the fragment depth (clamped to 0..1 by the depth buffer), depth test LESS
//    against the cleared 1: the buffer keeps the minimum.
//  - thickness (ssfr_thickness_*.glsl, RenderThickness :602-646): same sprites, additive
//    blending of n.z * 0.005 into a buffer cleared to the clear colour, no depth test (the
//    target has no depth attachment).  The sum is accumulated in 32.32 fixed point (each
//    term rounded to 2^-32), so it does not depend on the order of the atomics.
//  - bilateral smoothing (bilateral_fs.glsl, SmoothDepth :542-600): first along y, then
//    along x (blur_dir = (1, 1/H), then (1/W, 1)): taps x = -R, -R+1, .. <= R, nearest
//    texel with GL_REPEAT wrap (RenderTargetTexture.h:19-22), taps at depth >= 1 skipped,
//    weight exp(-(x s)^2) exp(-((d_tap - d) f)^2); depth <= 0 gives 0, depth >= 1 gives 1.
//  - composite (ssfr_fluid_fs.glsl, RenderFluid :648-690): eye position from depth through
//    the inverse projection, normal from the smaller of the one-sided differences, Phong
//    specular (exponent 1000), refraction of the scene with thickness-based transmission,
//    the shader's fresnel, diffuse and sky/ground reflection terms.
#pragma once
#include "render.cuh"

namespace snowb {

struct SsfrCam {
    float PV[16];           // projection * view (glm's product, column-major)
    float V[16], P[16];     // model_view (the model matrix is the identity) and projection
    float Pinv[16], Vinv[16];
    float point_size, radius;
    uint32_t W, H;
};
struct SsfrShade {
    float filter_radius, blur_scale, falloff;
    float light[4];         // light_color (rgb, w = surface weight)
    float clear[4];         // clear colour (thickness and scene background)
};

__device__ __forceinline__ float3 f3sub(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 f3norm(float3 v)
{
    const float l = sqrtf(dot3(v, v));
    return f3(v.x / l, v.y / l, v.z / l);
}
__device__ __forceinline__ float smoothstep_f(float e0, float e1, float x)
{
    float t = (x - e0) / (e1 - e0);
    t = fminf(fmaxf(t, 0.f), 1.f);
    return t * t * (3.f - 2.f * t);
}
__device__ __forceinline__ float mix_f(float a, float b, float t) { return a * (1.f - t) + b * t; }
__device__ __forceinline__ uint32_t wrap_texel(int i, uint32_t n)
{
    const int m = i % (int)n;
    return (uint32_t)(m < 0 ? m + (int)n : m);
}

struct DepthVtx {
    bool live;
    float xw, yw, side;
    float3 eye;
};
__device__ __forceinline__ DepthVtx depth_vertex(const SsfrCam& c, float3 p)
{
    DepthVtx v;
    const float4 cl = mat_vec(c.PV, p.x, p.y, p.z, 1.f);
    const float4 e = mat_vec(c.V, p.x, p.y, p.z, 1.f);
    v.live = cl.w > 0.f && cl.x >= -cl.w && cl.x <= cl.w && cl.y >= -cl.w && cl.y <= cl.w && cl.z >= -cl.w &&
             cl.z <= cl.w;
    v.xw = (cl.x / cl.w + 1.f) * 0.5f * (float)c.W;
    v.yw = (cl.y / cl.w + 1.f) * 0.5f * (float)c.H;
    v.side = c.point_size / cl.w;
    v.eye = f3(e.x, e.y, e.z);
    return v;
}
// n.xy of a covered pixel and r2 = |n.xy|^2; false when the fragment is discarded
__device__ __forceinline__ bool sphere_coord(const DepthVtx& v, int px, int py, float& nx, float& ny, float& nz)
{
    point_coord(v.xw, v.yw, v.side, px, py, nx, ny);
    const float r2 = nx * nx + ny * ny;
    if (r2 > 1.f) return false;
    nz = sqrtf(1.f - r2);
    return true;
}

// Sphere depth of n particles into depth (float bits, cleared to 1.0): minimum over fragments.
__global__ void ks_sphere_depth(SsfrCam c, const snowb_float3* __restrict__ pos, uint32_t n, uint32_t* __restrict__ depth)
{
    GRID_LOOP(i, n) {
        const DepthVtx v = depth_vertex(c, ldv3(pos, i));
        if (!v.live) continue;
        int x0, x1, y0, y1;
        sprite_span(v.xw, v.side, c.W, x0, x1);
        sprite_span(v.yw, v.side, c.H, y0, y1);
        for (int py = y0; py < y1; ++py)
            for (int px = x0; px < x1; ++px) {
                float nx, ny, nz;
                if (!sphere_coord(v, px, py, nx, ny, nz)) continue;
                const float ex = v.eye.x + nx * c.radius, ey = v.eye.y + ny * c.radius, ez = v.eye.z + nz * c.radius;
                const float4 cl = mat_vec(c.P, ex, ey, ez, 1.f);
                float d = cl.z / cl.w;
                if (!(d < 1.f)) continue;             // LESS against the cleared 1 (NaN fails too)
                d = d > 0.f ? d : 0.f;                // clamp to 0..1 (and -0 to +0)
                atomicMin(depth + (size_t)py * c.W + px, __float_as_uint(d));
            }
    }
}

// Thickness of n particles, 32.32 fixed point per pixel.
__global__ void ks_thickness(SsfrCam c, const snowb_float3* __restrict__ pos, uint32_t n,
                             unsigned long long* __restrict__ thick)
{
    GRID_LOOP(i, n) {
        const DepthVtx v = depth_vertex(c, ldv3(pos, i));
        if (!v.live) continue;
        int x0, x1, y0, y1;
        sprite_span(v.xw, v.side, c.W, x0, x1);
        sprite_span(v.yw, v.side, c.H, y0, y1);
        for (int py = y0; py < y1; ++py)
            for (int px = x0; px < x1; ++px) {
                float nx, ny, nz;
                if (!sphere_coord(v, px, py, nx, ny, nz)) continue;
                const float t = nz * 0.005f;
                atomicAdd(thick + (size_t)py * c.W + px, __float2ull_rn(t * 4294967296.f));
            }
    }
}
__device__ __forceinline__ float thickness_value(unsigned long long q, float clear_r)
{
    return clear_r + __ull2float_rn(q) * 2.3283064365386963e-10f;   // 2^-32
}

// One bilateral pass: horizontal = 0 filters along y, 1 along x.
__global__ void ks_bilateral(SsfrCam c, SsfrShade s, const float* __restrict__ in, float* __restrict__ out,
                             int horizontal)
{
    GRID_LOOP(k, c.W * c.H) {
        const int px = (int)(k % c.W), py = (int)(k / c.W);
        const float depth = in[k];
        if (depth <= 0.f) { out[k] = 0.f; continue; }
        if (depth >= 1.f) { out[k] = 1.f; continue; }
        float sum = 0.f, wsum = 0.f;
        for (float x = -s.filter_radius; x <= s.filter_radius; x += 1.f) {
            size_t t;
            if (horizontal) t = (size_t)py * c.W + wrap_texel((int)floorf(((float)px + 0.5f) + x), c.W);
            else t = (size_t)wrap_texel((int)floorf(((float)py + 0.5f) + x), c.H) * c.W + px;
            const float sd = in[t];
            if (sd >= 1.f) continue;
            const float r = x * s.blur_scale;
            const float w = expf(-r * r);
            const float r2 = (sd - depth) * s.falloff;
            const float g = expf(-r2 * r2);
            sum += sd * w * g;
            wsum += w * g;
        }
        if (wsum > 0.f) sum /= wsum;
        out[k] = sum < 1.f ? fmaxf(sum, 0.f) : 1.f;
    }
}

__device__ __forceinline__ float3 uv_to_eye(const SsfrCam& c, float u, float v, float z)
{
    const float4 e = mat_vec(c.Pinv, u * 2.f - 1.f, v * 2.f - 1.f, z, 1.f);
    return f3(e.x / e.w, e.y / e.w, e.z / e.w);
}

// Full-screen composite into rgba.
__global__ void ks_compose(SsfrCam c, SsfrShade s, const float* __restrict__ D, const unsigned long long* __restrict__ TH,
                           const float* __restrict__ scene, const float* __restrict__ SD, float* __restrict__ out)
{
    const float iw = 1.f / (float)c.W, ih = 1.f / (float)c.H;
    GRID_LOOP(k, c.W * c.H) {
        const int px = (int)(k % c.W), py = (int)(k / c.W);
        const float depth = D[k];
        const float sdep = SD[k];
        const float thick = fmaxf(thickness_value(TH[k], s.clear[0]), 0.3f);
        float4 o;
        if (depth == 0.f) {
            o = make_float4(0.f, 0.f, 0.f, 0.f);
        } else if (depth == 1.f || depth >= sdep) {
            o = make_float4(scene[4 * k], scene[4 * k + 1], scene[4 * k + 2], scene[4 * k + 3]);
        } else {
            const float u = ((float)px + 0.5f) / (float)c.W, v = ((float)py + 0.5f) / (float)c.H;
            const float3 eye = uv_to_eye(c, u, v, depth);
            const size_t row = (size_t)py * c.W;
            const float3 zl = f3sub(eye, uv_to_eye(c, u - iw, v, D[row + wrap_texel(px - 1, c.W)]));
            const float3 zr = f3sub(uv_to_eye(c, u + iw, v, D[row + wrap_texel(px + 1, c.W)]), eye);
            const float3 zt = f3sub(uv_to_eye(c, u, v + ih, D[(size_t)wrap_texel(py + 1, c.H) * c.W + px]), eye);
            const float3 zb = f3sub(eye, uv_to_eye(c, u, v - ih, D[(size_t)wrap_texel(py - 1, c.H) * c.W + px]));
            const float3 dx = fabsf(zr.z) < fabsf(zl.z) ? zr : zl;
            const float3 dy = fabsf(zb.z) < fabsf(zt.z) ? zb : zt;
            const float3 nrm = f3norm(f3(dx.y * dy.z - dy.y * dx.z, dx.z * dy.x - dy.z * dx.x, dx.x * dy.y - dy.x * dx.y));
            const float4 wp = mat_vec(c.Vinv, eye.x, eye.y, eye.z, 1.f);
            const float4 l4 = mat_vec(c.V, 0.f, 1.f, 0.f, 0.f);
            const float3 l = f3(l4.x, l4.y, l4.z);
            const float3 ne = f3norm(eye);
            const float3 vd = f3(-ne.x, -ne.y, -ne.z);
            const float3 hv = f3norm(f3(vd.x + l.x, vd.y + l.y, vd.z + l.z));
            const float spec = powf(fmaxf(0.f, dot3(nrm, hv)), 1000.f);
            const float rs = (1.33f * 0.025f) * smoothstep_f(0.1f, 0.4f, wp.y);
            const float ru = u + nrm.x * rs * 0.75f, rv = v + nrm.y * rs * 1.f;
            const size_t rt = (size_t)wrap_texel((int)floorf(rv * (float)c.H), c.H) * c.W +
                              wrap_texel((int)floorf(ru * (float)c.W), c.W);
            const float tr0 = expf(-(0.9804f - s.light[0]) * thick);
            const float tr1 = expf(-(1.0f - s.light[1]) * thick);
            const float tr2 = expf(-(0.7255f - s.light[2]) * thick);
            const float3 refr = f3(scene[4 * rt] * tr0, scene[4 * rt + 1] * tr1, scene[4 * rt + 2] * tr2);
            const float3 lv = f3norm(f3(wp.x - 0.f, wp.y - 1000.f, wp.z - 0.f));
            const float ddl = (lv.x * -0.f + lv.y * -1.f) + lv.z * -0.f;
            const float att = fmaxf(smoothstep_f(0.95f, 1.0f, fabsf(ddl)), 0.05f);
            const float ln = dot3(l, nrm) * att;
            const float fres = 0.1f + 0.9f * powf(fminf(0.f, 1.f - dot3(nrm, vd)), 5.f);
            const float mx = mix_f(1.f, 1.f, ln * 0.5f + 0.5f);
            const float3 dif = f3(s.light[0] * mx * (1.f - s.light[3]), s.light[1] * mx * (1.f - s.light[3]),
                                  s.light[2] * mx * (1.f - s.light[3]));
            const float sky0 = 0.8078f * 1.2f, sky1 = 0.4784f * 1.2f, sky2 = 0.2078f * 1.2f;
            const float nv = dot3(nrm, vd);
            const float3 re = f3(vd.x - 2.f * nv * nrm.x, vd.y - 2.f * nv * nrm.y, vd.z - 2.f * nv * nrm.z);
            const float4 rw = mat_vec(c.Vinv, re.x, re.y, re.z, 0.f);
            const float ss = smoothstep_f(0.15f, 0.25f, rw.y);
            const float3 refl = f3(1.f + mix_f(1.f, sky0, ss), 1.f + mix_f(1.f, sky1, ss), 1.f + mix_f(1.f, sky2, ss));
            o.x = dif.x + (mix_f(refr.x, refl.x, fres) + spec) * s.light[3];
            o.y = dif.y + (mix_f(refr.y, refl.y, fres) + spec) * s.light[3];
            o.z = dif.z + (mix_f(refr.z, refl.z, fres) + spec) * s.light[3];
            o.w = 1.f;
        }
        out[4 * k] = o.x; out[4 * k + 1] = o.y; out[4 * k + 2] = o.z; out[4 * k + 3] = o.w;
    }
}
__global__ void ks_fill(uint32_t npix, uint32_t* __restrict__ depth_bits, uint32_t value,
                        unsigned long long* __restrict__ thick)
{
    GRID_LOOP(k, npix) {
        if (depth_bits) depth_bits[k] = value;
        if (thick) thick[k] = 0ull;
    }
}

}  // namespace snowb
