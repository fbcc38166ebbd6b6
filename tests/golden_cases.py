"""Load the golden fixtures (tests/golden/*.npz, produced by running the
reference's own code, see tests/golden/make_golden.py) as reference-style
argument dicts."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    """Simulation fixtures of the reference's own runs (the analysis_* files hold
    electrode LAT / CV / interpolation cases, c1_* the oracle's sheet run)."""
    return sorted(os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(f).startswith(("analysis_", "c1_")))


def analysis_names():
    """The electrode LAT / conduction-velocity fixtures (not the interpolation one)."""
    return sorted(os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLDEN, "analysis_*.npz"))
                  if not f.endswith("analysis_interp.npz"))


def interp_cases():
    """[(name, voxel, electrode_xyz, lat_electrode, lat_voxel)] of the reference's
    own interpolate_lat (tests/golden/analysis_interp.npz)."""
    g = np.load(os.path.join(GOLDEN, "analysis_interp.npz"), allow_pickle=False)
    return [(str(nm), g[f"{k}_voxel"], g[f"{k}_electrode"], g[f"{k}_lat_electrode"], g[f"{k}_lat_voxel"])
            for k, nm in enumerate(g["names"])]


def load(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)
    sp = {k[3:]: g[k].item() for k in g.files if k.startswith("sp_")}
    ap = {k[3:]: g[k].item() for k in g.files if k.startswith("ap_")}
    ap["s1_pacing_voxel_id"] = g["s1"]
    ap["s2_pacing_voxel_id"] = g["s2"]
    ap["node_flag"] = g["node_flag"]
    geom = {"neighbor_id_2d": g["neighbor_id_2d"], "Delta": float(g["Delta"]), "voxel": g["voxel"]}
    return dict(n=g["voxel"].shape[0], P_2d=g["P_2d"], geom=geom, sp=sp, ap=ap, g=g)
