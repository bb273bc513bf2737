"""Generate the golden fixtures of tests/golden/ from the reference's own solver.

Runs the reference (cuda_simulation.cu built with IEEE arithmetic by oracle/ref_build.sh,
on a GPU) on the seeded `tiny` scene with interlinks off, stopping at several stage
boundaries of the first substep, and stores the water and snow state (live particles)
plus the boundary density and lambda.  The CPU test test_cpu_golden.py checks the FP32
oracle against these files bit for bit.  Usage (GPU machine):
    python tests/golden/make_golden.py  [output directory, default tests/golden]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from snowsimulation_b200 import scene  # noqa: E402
from oracle.ref_runner import RefWorld  # noqa: E402

STOPS = (2, 3, 7, 12, 15, 16, 17, 90, 0)
FIELDS_SET = ("positions", "predict_positions", "velocity", "density", "C", "lambda_", "T", "contrib",
              "correction")


def golden_world():
    w = scene.tiny(seed=1)
    w.flags["use_interlink"] = False
    return w


def snapshot(W):
    out = {"n_sph": W.n_sph, "n_dem": W.n_dem}
    for sname, s, n in (("sph", W.sph, W.n_sph), ("dem", W.dem, W.n_dem)):
        for f in FIELDS_SET:
            out["%s_%s" % (sname, f)] = s[f][:n].copy()
    out["bnd_density"] = W.bnd["density"].copy()
    out["bnd_lambda_"] = W.bnd["lambda_"].copy()
    out["dem_cd_grid_index"] = W.dem_cd["grid_index"][: W.n_dem].copy()
    out["sph_cd_grid_index"] = W.sph_cd["grid_index"][: W.n_sph].copy()
    return out


def main():
    outdir = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__))
    os.makedirs(outdir, exist_ok=True)
    for stop in STOPS:
        r = RefWorld(golden_world(), "ieee").setup()
        r.step(stop_after=stop)
        snap = snapshot(r.to_host())
        r.close()
        np.savez_compressed(os.path.join(outdir, "ref_tiny_stage%02d.npz" % stop), **snap)
        print("wrote stage", stop)


if __name__ == "__main__":
    main()
