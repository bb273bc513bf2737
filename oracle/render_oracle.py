"""CPU restatement of the point-sprite shaders (TEST INFRASTRUCTURE -- the checker for
libsnowb200's snowb_render_points).  Follows point_sprite_vs.glsl,
point_sprite_temperature_vs.glsl and point_sprite_fs.glsl with GL's point rasterisation
(pixel centres inside the sprite square, upper-left point-coordinate origin), depth test
LESS in draw order, colours clamped to 0..1; every float32 operation in the order the CUDA
kernels use, so results compare bit for bit."""
import numpy as np

f32 = np.float32


def _mv(M, x, y, z, w):
    M = [f32(v) for v in M]
    return (((M[0] * x + M[4] * y) + M[8] * z) + M[12] * w, ((M[1] * x + M[5] * y) + M[9] * z) + M[13] * w,
            ((M[2] * x + M[6] * y) + M[10] * z) + M[14] * w, ((M[3] * x + M[7] * y) + M[11] * z) + M[15] * w)


def _vertex(cam, col, p, T):
    x, y, z = (f32(v) for v in p)
    e = _mv(cam["view"], x, y, z, f32(1))
    c = _mv(cam["projection"], *e)
    live = c[3] > 0 and all(-c[3] <= c[k] <= c[3] for k in range(3))
    nx, ny, nz = c[0] / c[3], c[1] / c[3], c[2] / c[3]
    W, H = cam["width"], cam["height"]
    xw = (nx + f32(1)) * f32(0.5) * f32(W)
    yw = (ny + f32(1)) * f32(0.5) * f32(H)
    depth = (nz + f32(1)) * f32(0.5)
    cp = [f32(v) for v in cam["camera_pos"]]
    dv = (cp[0] - x, cp[1] - y, cp[2] - z)
    side = f32(cam["point_size"]) / np.sqrt((dv[0] * dv[0] + dv[1] * dv[1]) + dv[2] * dv[2])
    lp = [f32(v) for v in cam["light_pos"]]
    l = (lp[0] - e[0], lp[1] - e[1], lp[2] - e[2])
    ll = np.sqrt((l[0] * l[0] + l[1] * l[1]) + l[2] * l[2])
    ldir = (l[0] / ll, l[1] / ll, l[2] / ll)
    if col.get("temperature") is not None:
        cool, hot, tc, th = col["temperature"]
        a = (f32(T) - f32(tc)) / (f32(th) - f32(tc))
        rgb = tuple(f32(cool[k]) * (f32(1) - a) + f32(hot[k]) * a for k in range(3))
    else:
        rgb = tuple(f32(v) for v in col["rgb"])
    return live, xw, yw, depth, side, ldir, rgb


def _span(c, side, lim):
    lo, hi = c - f32(0.5) * side, c + f32(0.5) * side
    a, b = int(np.ceil(lo - f32(0.5))), int(np.ceil(hi - f32(0.5)))
    return max(a, 0), min(b, lim)


def _fragment(v, px, py):
    _, xw, yw, _, side, ldir, rgb = v
    pcx = ((f32(px) + f32(0.5)) - (xw - f32(0.5) * side)) / side
    pcy = ((yw + f32(0.5) * side) - (f32(py) + f32(0.5))) / side
    nx, ny = pcx * f32(2) - f32(1), pcy * f32(2) - f32(1)
    nz = f32(1) - (nx * nx + ny * ny)
    if nz < 0:
        return None
    nz = np.sqrt(nz)
    d = (ldir[0] * nx + ldir[1] * ny) + ldir[2] * nz
    return tuple(min(max(d * c, f32(0)), f32(1)) for c in rgb)


def render(cam, draws):
    """draws: list of (positions (n x 3), temperatures or None, colour dict).  Returns the
    H x W x 4 image."""
    W, H = cam["width"], cam["height"]
    img = np.zeros((H, W, 4), f32)
    zb = np.full((H, W), np.inf, np.float64)
    for pos, temps, col in draws:
        for i in range(len(pos)):
            v = _vertex(cam, col, pos[i], temps[i] if temps is not None else 0.0)
            if not v[0]:
                continue
            x0, x1 = _span(v[1], v[4], W)
            y0, y1 = _span(v[2], v[4], H)
            for py in range(y0, y1):
                for px in range(x0, x1):
                    rgb = _fragment(v, px, py)
                    if rgb is not None and v[3] < zb[py, px]:
                        zb[py, px] = v[3]
                        img[py, px, :3] = rgb
                        img[py, px, 3] = 1.0
    return img
