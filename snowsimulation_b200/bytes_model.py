"""Algorithmic-bytes model of the substep (the roofline numerator).

Convention: each stage reads its per-particle inputs once and writes its outputs once
(neighbour re-reads count as cache hits), a float3 counts as 16 B, an interlink slot as
4 B index + 4 B length.  Bytes per particle and stage pass:
"""
# per-particle bytes of one pass of each stage
PASS = dict(
    S=76,     # hash + sort + cell build
    D=28,     # density
    L=28,     # lambda
    P=56,     # PBF correction
    X=56,     # contact (non-penetration) correction
    I=252,    # interlink: 25 slots x 8 B + 16 + 4 + 32
    A=84,     # apply correction
    F=52,     # friction
    H=32,     # heat conduction
    PC=8,     # phase-change check
    CR=428,   # link formation: 25 x 16 B (r+w) + 28
    G=88,     # integrate
    Fi=64,    # finalize
    V=56,     # XSPH
)


def per_particle_substep(iterations=3):
    """(water, snow, boundary) bytes per particle and substep."""
    p = PASS
    water = 2 * p["S"] + p["D"] + p["H"] + p["PC"] + p["G"] + p["Fi"] + p["V"] + \
        iterations * (2 * p["S"] + p["D"] + p["L"] + p["P"] + p["X"] + p["A"])
    snow = 2 * p["S"] + p["D"] + p["H"] + p["PC"] + p["CR"] + p["G"] + p["Fi"] + p["V"] + \
        iterations * (2 * p["S"] + p["D"] + p["L"] + p["P"] + p["X"] + p["I"] + p["A"] + p["F"] + p["A"])
    boundary = (1 + iterations) * p["D"] + iterations * p["L"]
    return water, snow, boundary


def substep_bytes(n_water, n_snow, n_boundary, iterations=3):
    w, s, b = per_particle_substep(iterations)
    return w * n_water + s * n_snow + b * n_boundary


def kernel_bytes(name, n_water, n_snow, n_boundary):
    """Algorithmic bytes of ONE launch of a library kernel (fused kernels sum their passes)."""
    p = PASS
    table = {
        "k_density": p["D"] * (n_water + n_snow + n_boundary),
        "k_lambda": p["L"] * (n_water + n_snow + n_boundary),
        "k_pbf": (p["P"] + p["X"]) * n_water + p["P"] * n_snow,
        "k_dem_corr": p["X"] * n_snow,
        # the interlink pass: the per-slot terms (25 slots x 8 B, the particle's position and
        # inverse mass) and their sum into the correction (16 B read + 16 B written)
        "k_link_terms": (p["I"] - 32) * n_snow,
        "k_link_sum": 32 * n_snow,
        "k_friction": p["F"] * n_snow,
        "k_heat": p["H"] * (n_water + n_snow),
        "k_integrate": p["G"] * (n_water + n_snow),
        "k_finalize": p["Fi"] * (n_water + n_snow),
        "k_xsph": p["V"] * n_water,
    }
    return table.get(name)
