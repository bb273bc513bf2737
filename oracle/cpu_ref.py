"""ctypes wrapper of oracle/_ref/libsnowcpuref.so: the reference's own CPU neighbour search
(NeighborSearch::SpatialSearch, NeighborSearch.cpp:154-259) and XPBD distance-constraint
solver (ConstraintSolver::SolveXPBDConstraints, ConstraintSolver.cpp:51-72), built from the
reference's sources by cpu_ref_build.sh.

Measurement infrastructure: used for the reported CPU baselines and their tests only.
Neither routine is part of the substep that the product replaces; they are the reference's
only CPU code near that path and are timed beside the project's CPU restatement.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libsnowcpuref.so")
_lib = None

# SpatialSearch runs on the 8 OpenMP threads hard-wired at NeighborSearch.cpp:210; the
# XPBD solver is a sequential loop over the constraints (ConstraintSolver.cpp:60-69).
SPATIAL_SEARCH_THREADS = 8
XPBD_THREADS = 1


def available() -> bool:
    return os.path.exists(LIB_PATH)


def load():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError("%s is not built (oracle/cpu_ref_build.sh needs the reference sources)"
                                    % LIB_PATH)
        lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        lib.cpuref_spatial_search.argtypes = [P, ctypes.c_uint32, ctypes.c_float, ctypes.c_int, P, P]
        lib.cpuref_spatial_search.restype = ctypes.c_int
        lib.cpuref_xpbd_links.argtypes = [P, ctypes.c_uint32, P, P, P, ctypes.c_uint32, ctypes.c_float,
                                          ctypes.c_float, ctypes.c_int, ctypes.c_int, P, P]
        lib.cpuref_xpbd_links.restype = ctypes.c_int
        _lib = lib
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def spatial_search(pos, h, calls=1):
    """Returns (directed neighbour pairs, seconds per call) of the reference's SpatialSearch
    over the positions (n x 3) with radius h."""
    lib = load()
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    pairs = np.zeros(1, np.uint64)
    sec = np.zeros(1, np.float64)
    rc = lib.cpuref_spatial_search(_ptr(p), len(p), float(h), int(calls), _ptr(pairs), _ptr(sec))
    if rc != 0:
        raise RuntimeError("cpuref_spatial_search returned %d" % rc)
    return int(pairs[0]), float(sec[0])


def xpbd_links(pos, a, b, rest, mass, dt, iters=3, calls=1):
    """Returns (new positions, seconds per solve) of the reference's XPBD solver over one
    distance constraint per link (a[k], b[k], rest[k]), starting from pos."""
    lib = load()
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    a = np.ascontiguousarray(a, np.uint32)
    b = np.ascontiguousarray(b, np.uint32)
    r = np.ascontiguousarray(rest, np.float32)
    if not (len(a) == len(b) == len(r)):
        raise ValueError("link arrays differ in length")
    out = np.empty_like(p)
    sec = np.zeros(1, np.float64)
    rc = lib.cpuref_xpbd_links(_ptr(p), len(p), _ptr(a), _ptr(b), _ptr(r), len(a), float(mass), float(dt),
                               int(iters), int(calls), _ptr(sec), _ptr(out))
    if rc != 0:
        raise RuntimeError("cpuref_xpbd_links returned %d" % rc)
    return out, float(sec[0])


def link_pairs(connect_record, connect_length, n, maxc):
    """Unordered link pairs (i < j) with their rest lengths from interlink slot arrays
    (slot k of particle i at i * maxc + k, 0xFFFFFFFF empty)."""
    rec = np.asarray(connect_record[: n * maxc], np.uint32).reshape(n, maxc)
    ln = np.asarray(connect_length[: n * maxc], np.float32).reshape(n, maxc)
    i, k = np.nonzero(rec != 0xFFFFFFFF)
    j = rec[i, k].astype(np.int64)
    keep = i < j
    return i[keep].astype(np.uint32), j[keep].astype(np.uint32), ln[i[keep], k[keep]]
