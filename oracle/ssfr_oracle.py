"""CPU restatement of the screen-space fluid pipeline (TEST INFRASTRUCTURE -- the checker
for libsnowb200's snowb_ssfr_* entry points).  Follows point_depth_vs/fs.glsl,
ssfr_thickness_vs/fs.glsl, bilateral_fs.glsl and ssfr_fluid_fs.glsl as the reference's
Renderer drives them (Renderer.cpp:404-690), with GL's point rasterisation (pixel centres
inside the sprite square, upper-left point-coordinate origin), nearest-texel sampling with
GL_REPEAT wrap (RenderTargetTexture.h:19-22), depth test LESS against a buffer cleared to 1.

Every float32 operation is the one the CUDA kernels perform, in the same order, so sphere
depth and thickness compare bit for bit; the smoothing and the composite call exp and pow,
whose last bits differ between libm and CUDA, so those compare within a stated tolerance.
The camera matrices (projection * view and the inverses) are the library's own
(snowb_ssfr_matrices), passed in as `mats`.
"""
import numpy as np

f32 = np.float32
TWO_M32 = f32(2.0 ** -32)


def _mv(M, x, y, z, w):
    M = [f32(v) for v in M]
    return (((M[0] * x + M[4] * y) + M[8] * z) + M[12] * w, ((M[1] * x + M[5] * y) + M[9] * z) + M[13] * w,
            ((M[2] * x + M[6] * y) + M[10] * z) + M[14] * w, ((M[3] * x + M[7] * y) + M[11] * z) + M[15] * w)


def _span(c, side, lim):
    lo, hi = c - f32(0.5) * side, c + f32(0.5) * side
    a, b = int(np.ceil(lo - f32(0.5))), int(np.ceil(hi - f32(0.5)))
    return max(a, 0), min(b, lim)


def _sprites(mats, cam, pos):
    """Yield (eye, px, py, nx, ny, nz) for every covered, non-discarded fragment."""
    PV, V = mats["PV"], mats["V"]
    W, H = int(cam["width"]), int(cam["height"])
    ps = f32(cam["point_size"])
    for p in np.asarray(pos, f32):
        x, y, z = (f32(v) for v in p)
        c = _mv(PV, x, y, z, f32(1))
        e = _mv(V, x, y, z, f32(1))
        if not (c[3] > 0 and all(-c[3] <= c[k] <= c[3] for k in range(3))):
            continue
        xw = (c[0] / c[3] + f32(1)) * f32(0.5) * f32(W)
        yw = (c[1] / c[3] + f32(1)) * f32(0.5) * f32(H)
        side = ps / c[3]
        x0, x1 = _span(xw, side, W)
        y0, y1 = _span(yw, side, H)
        for py in range(y0, y1):
            for px in range(x0, x1):
                pcx = ((f32(px) + f32(0.5)) - (xw - f32(0.5) * side)) / side
                pcy = ((yw + f32(0.5) * side) - (f32(py) + f32(0.5))) / side
                nx, ny = pcx * f32(2) - f32(1), pcy * f32(2) - f32(1)
                r2 = nx * nx + ny * ny
                if r2 > f32(1):
                    continue
                yield e, px, py, nx, ny, np.sqrt(f32(1) - r2)


def sphere_depth(mats, cam, pos, radius, depth=None):
    """Minimum sphere depth (H x W float32, 1 = empty) of the particles."""
    W, H = int(cam["width"]), int(cam["height"])
    d = np.ones((H, W), f32) if depth is None else depth
    r = f32(radius)
    for e, px, py, nx, ny, nz in _sprites(mats, cam, pos):
        c = _mv(mats["P"], e[0] + nx * r, e[1] + ny * r, e[2] + nz * r, f32(1))
        z = c[2] / c[3]
        if not z < f32(1):
            continue
        z = z if z > 0 else f32(0)
        if z < d[py, px]:
            d[py, px] = z
    return d


def thickness_fixed(mats, cam, pos):
    """32.32 fixed-point thickness sums (H x W uint64)."""
    W, H = int(cam["width"]), int(cam["height"])
    t = np.zeros((H, W), np.uint64)
    for _, px, py, _, _, nz in _sprites(mats, cam, pos):
        q = np.rint(np.float64(nz * f32(0.005)) * 2.0 ** 32)
        t[py, px] += np.uint64(q)
    return t


def thickness_value(q, clear_r):
    return f32(clear_r) + q.astype(f32) * TWO_M32


def smooth_pass(d, filter_radius, blur_scale, falloff, horizontal):
    """One bilateral pass (along x when horizontal, else along y) over H x W depths."""
    d = np.asarray(d, f32)
    H, W = d.shape
    out = np.empty_like(d)
    R, bs, fo = f32(filter_radius), f32(blur_scale), f32(falloff)
    s = np.zeros_like(d)
    ws = np.zeros_like(d)
    xs = []
    x = -R
    while x <= R:
        xs.append(x)
        x = x + f32(1)
    rows, cols = np.indices((H, W))
    for x in xs:
        if horizontal:
            t = np.floor((cols.astype(f32) + f32(0.5)) + x).astype(np.int64) % W
            sd = d[rows, t]
        else:
            t = np.floor((rows.astype(f32) + f32(0.5)) + x).astype(np.int64) % H
            sd = d[t, cols]
        r = x * bs
        w = np.exp(f32(-r * r)).astype(f32)
        r2 = (sd - d) * fo
        g = np.exp(-r2 * r2).astype(f32)
        use = sd < f32(1)
        s = np.where(use, s + sd * w * g, s).astype(f32)
        ws = np.where(use, ws + w * g, ws).astype(f32)
    s = np.where(ws > 0, s / np.where(ws > 0, ws, f32(1)), s).astype(f32)
    s = np.where(s < f32(1), np.maximum(s, f32(0)), f32(1)).astype(f32)
    out[...] = np.where(d <= 0, f32(0), np.where(d >= 1, f32(1), s))
    return out


def smooth(d, filter_radius=10.0, blur_scale=0.1, falloff=65.0):
    return smooth_pass(smooth_pass(d, filter_radius, blur_scale, falloff, False), filter_radius, blur_scale, falloff,
                       True)


def _mva(M, x, y, z, w):
    return _mv(M, x, y, z, w)


def _norm(x, y, z):
    l = np.sqrt((x * x + y * y) + z * z)
    return x / l, y / l, z / l


def _smoothstep(e0, e1, x):
    t = (x - f32(e0)) / (f32(e1) - f32(e0))
    t = np.minimum(np.maximum(t, f32(0)), f32(1))
    return t * t * (f32(3) - f32(2) * t)


def _mix(a, b, t):
    return a * (f32(1) - t) + b * t


def compose(mats, cam, D, TH, scene, SD, light=(1.0, 1.0, 1.0, 0.8), clear=(0.15, 0.15, 0.15, 0.0)):
    """The fluid composite (H x W x 4) from the smoothed water depth D, the fixed-point
    thickness TH, the scene image and the scene depth SD."""
    W, H = int(cam["width"]), int(cam["height"])
    D = np.asarray(D, f32)
    SD = np.asarray(SD, f32)
    scene = np.asarray(scene, f32)
    L = [f32(v) for v in light]
    thick = np.maximum(thickness_value(np.asarray(TH, np.uint64), clear[0]), f32(0.3))
    rows, cols = np.indices((H, W))
    u = (cols.astype(f32) + f32(0.5)) / f32(W)
    v = (rows.astype(f32) + f32(0.5)) / f32(H)
    iw, ih = f32(1) / f32(W), f32(1) / f32(H)
    Pinv, Vinv, V = mats["Pinv"], mats["Vinv"], mats["V"]

    def to_eye(uu, vv, z):
        e = _mva(Pinv, uu * f32(2) - f32(1), vv * f32(2) - f32(1), z, f32(1))
        return e[0] / e[3], e[1] / e[3], e[2] / e[3]

    def sub(a, b):
        return a[0] - b[0], a[1] - b[1], a[2] - b[2]

    with np.errstate(all="ignore"):
        eye = to_eye(u, v, D)
        zl = sub(eye, to_eye(u - iw, v, D[rows, (cols - 1) % W]))
        zr = sub(to_eye(u + iw, v, D[rows, (cols + 1) % W]), eye)
        zt = sub(to_eye(u, v + ih, D[(rows + 1) % H, cols]), eye)
        zb = sub(eye, to_eye(u, v - ih, D[(rows - 1) % H, cols]))
        px = np.abs(zr[2]) < np.abs(zl[2])
        dx = tuple(np.where(px, a, b) for a, b in zip(zr, zl))
        py = np.abs(zb[2]) < np.abs(zt[2])
        dy = tuple(np.where(py, a, b) for a, b in zip(zb, zt))
        n = _norm(dx[1] * dy[2] - dy[1] * dx[2], dx[2] * dy[0] - dy[2] * dx[0], dx[0] * dy[1] - dy[0] * dx[1])
        wp = _mva(Vinv, eye[0], eye[1], eye[2], f32(1))
        l4 = _mv(V, f32(0), f32(1), f32(0), f32(0))
        ne = _norm(*eye)
        vd = (-ne[0], -ne[1], -ne[2])
        hv = _norm(vd[0] + l4[0], vd[1] + l4[1], vd[2] + l4[2])
        dnh = (n[0] * hv[0] + n[1] * hv[1]) + n[2] * hv[2]
        spec = np.power(np.maximum(f32(0), dnh), f32(1000)).astype(f32)
        rs = (f32(1.33) * f32(0.025)) * _smoothstep(0.1, 0.4, wp[1])
        ru = u + n[0] * rs * f32(0.75)
        rv = v + n[1] * rs * f32(1)
        tx = np.floor(ru * f32(W))
        ty = np.floor(rv * f32(H))
        ok = np.isfinite(tx) & np.isfinite(ty)
        tx = np.where(ok, tx, 0).astype(np.int64) % W
        ty = np.where(ok, ty, 0).astype(np.int64) % H
        tr = [np.exp(-(f32(a) - L[k]) * thick).astype(f32) for k, a in enumerate((0.9804, 1.0, 0.7255))]
        refr = [scene[ty, tx, k] * tr[k] for k in range(3)]
        lv = _norm(wp[0] - f32(0), wp[1] - f32(1000), wp[2] - f32(0))
        ddl = (lv[0] * f32(-0.0) + lv[1] * f32(-1)) + lv[2] * f32(-0.0)
        att = np.maximum(_smoothstep(0.95, 1.0, np.abs(ddl)), f32(0.05))
        ln = ((l4[0] * n[0] + l4[1] * n[1]) + l4[2] * n[2]) * att
        nv = (n[0] * vd[0] + n[1] * vd[1]) + n[2] * vd[2]
        fres = f32(0.1) + f32(0.9) * np.power(np.minimum(f32(0), f32(1) - nv), f32(5)).astype(f32)
        mx = _mix(f32(1), f32(1), ln * f32(0.5) + f32(0.5))
        dif = [L[k] * mx * (f32(1) - L[3]) for k in range(3)]
        sky = (f32(0.8078) * f32(1.2), f32(0.4784) * f32(1.2), f32(0.2078) * f32(1.2))
        re = tuple(vd[k] - f32(2) * nv * n[k] for k in range(3))
        rw = _mv(Vinv, re[0], re[1], re[2], f32(0))
        ss = _smoothstep(0.15, 0.25, rw[1])
        refl = [f32(1) + _mix(f32(1), sky[k], ss) for k in range(3)]
        fl = [dif[k] + (_mix(refr[k], refl[k], fres) + spec) * L[3] for k in range(3)]
    out = np.empty((H, W, 4), f32)
    for k in range(3):
        out[..., k] = fl[k]
    out[..., 3] = 1
    empty = D == 0
    out[empty] = 0
    sc = (D == 1) | (D >= SD)
    sc &= ~empty
    out[sc] = scene[sc]
    return out
