"""Helpers shared by the tests: state comparison between two HostWorlds."""
import numpy as np

# fields that are scratch in both implementations (not part of the compared state)
SCRATCH = {"new_index"}


def _eq(a, b):
    if a.dtype.kind == "f":
        both_nan = np.isnan(a) & np.isnan(b)
        return np.where(both_nan, True, a == b)
    return a == b


def diff_worlds(a, b, sets=("sph", "dem", "bnd"), cells=("sph_cd", "dem_cd", "b_cd"), atol=0.0):
    """List of (where, n_bad, max_abs) for every array that differs (atol 0 = bit-exact)."""
    out = []
    if (a.n_sph, a.n_dem) != (b.n_sph, b.n_dem):
        out.append(("sizes", (a.n_sph, a.n_dem), (b.n_sph, b.n_dem)))
    for s in sets:
        for k, x in getattr(a, s).items():
            if k in SCRATCH:
                continue
            y = getattr(b, s)[k]
            _cmp(out, "%s.%s" % (s, k), x, y, atol)
    for c in cells:
        for k, x in getattr(a, c).items():
            _cmp(out, "%s.%s" % (c, k), x, getattr(b, c)[k], atol)
    return out


def _cmp(out, where, x, y, atol):
    if x.shape != y.shape:
        out.append((where, "shape", (x.shape, y.shape)))
        return
    if atol and x.dtype.kind == "f":
        x64, y64 = x.astype(np.float64), y.astype(np.float64)
        fin = np.isfinite(x64) & np.isfinite(y64)
        bad = (~fin & ~_eq(x, y)) | (fin & (np.abs(x64 - y64) > atol))
        md = float(np.max(np.abs(x64 - y64)[fin])) if fin.any() else 0.0
    else:
        bad = ~_eq(x, y)
        md = None
        if bad.any() and x.dtype.kind == "f":
            fin = np.isfinite(x) & np.isfinite(y)
            md = float(np.max(np.abs(x.astype(np.float64) - y.astype(np.float64))[fin])) if fin.any() else None
    if bad.any():
        idx = np.argwhere(bad)[0].tolist()
        out.append((where, int(bad.sum()), md, idx))


def live(world, set_name):
    n = world.n_sph if set_name == "sph" else world.n_dem
    return n


def track_ids(world):
    ids = np.concatenate([world.sph["trackId"][:world.n_sph], world.dem["trackId"][:world.n_dem]])
    return np.sort(ids)


def max_abs_diff(a, b, fields=("positions", "velocity", "T")):
    """Largest |a - b| per field over the live particles of both sets, matched by track id
    (the sets' slot orders agree when the runs are bit-exact, but need not otherwise)."""
    out = {}
    for f in fields:
        xs = []
        for w in (a, b):
            ids = np.concatenate([w.sph["trackId"][:w.n_sph], w.dem["trackId"][:w.n_dem]])
            val = np.concatenate([w.sph[f][:w.n_sph], w.dem[f][:w.n_dem]]).astype(np.float64)
            xs.append((ids, val))
        (ia, va), (ib, vb) = xs
        if not np.array_equal(np.sort(ia), np.sort(ib)):
            out[f] = None
            continue
        va, vb = va[np.argsort(ia)], vb[np.argsort(ib)]
        out[f] = float(np.abs(va - vb).max()) if len(va) else 0.0
    return out
