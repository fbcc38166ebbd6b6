"""Generate ``tests/golden/analysis_*.npz``: electrode LAT and conduction
velocity computed by the reference's OWN, unmodified
``utility/lat_map.py::compute_electrode_lat`` and
``utility/conduction_velocity.py::compute``.

Test infrastructure only.  Needs the reference checkout (``/root/reference``),
which exists only where the fixtures are generated; the fixtures are committed
and nothing at test time reads the reference.  ``lat_map.py`` imports
matplotlib, scipy's interpolators and the reference's ``common`` module for its
plotting helpers; matplotlib and ``common`` are replaced by empty stub modules
(the two functions used here touch neither).

Inputs are seeded synthetic electrograms: a downstroke ``-tanh((t - t_act)/w)``
per electrode, with activation times from a point source (3-D shell surface)
or a plane wave (flat sheet, where every electrode has the same z and the
plane fit is rank-deficient), plus small noise.

Run:  python tests/golden/make_golden_analysis.py
"""
import importlib.util
import os
import sys
import types

import numpy as np

REF = os.environ.get("PHS_REFERENCE_DIR", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def _load():
    for name in ("matplotlib", "matplotlib.pyplot", "matplotlib.colors", "common", "PIL", "PIL.Image"):
        sys.modules.setdefault(name, types.ModuleType(name))
    pkg = types.ModuleType("ref_utility")
    pkg.__path__ = [os.path.join(REF, "utility")]
    sys.modules["ref_utility"] = pkg
    mods = {}
    for name in ("lat_map", "conduction_velocity"):
        spec = importlib.util.spec_from_file_location(f"ref_utility.{name}", os.path.join(REF, "utility", f"{name}.py"))
        m = importlib.util.module_from_spec(spec)
        sys.modules[f"ref_utility.{name}"] = m
        setattr(pkg, name, m)
        spec.loader.exec_module(m)
        mods[name] = m
    return mods["lat_map"], mods["conduction_velocity"]


def electrograms(xyz, t_act, T, w, rng, noise=1e-3):
    t = np.arange(T, dtype=np.float64)[:, None]
    egm = -np.tanh((t - t_act[None, :]) / w) + noise * rng.standard_normal((T, xyz.shape[0]))
    return egm


def cases():
    from pyheartsim_b200 import synthetic
    rng = np.random.default_rng(7)
    out = []
    # 3-D: electrodes at surface voxels of a small shell, point-source activation
    ijk = synthetic.shell((9.0, 8.0, 7.0), 0.4, 3, 2, 2.0, 4)
    vox = ijk * 0.4
    ids = np.sort(rng.choice(vox.shape[0], size=240, replace=False))
    src = vox[ids[0]]
    t_act = 20.0 + np.linalg.norm(vox[ids] - src, axis=1) / 0.6          # 0.6 mm/ms
    out.append(("analysis_shell", vox, ids, electrograms(vox[ids], t_act, 120, 1.5, rng)))
    # 2-D sheet (all z equal: rank-deficient plane fits), plane wave along x+y
    i, j = np.meshgrid(np.arange(40), np.arange(30), indexing="ij")
    vox2 = np.stack([i.ravel() * 0.4, j.ravel() * 0.4, np.zeros(i.size)], axis=1)
    ids2 = np.sort(rng.choice(vox2.shape[0], size=150, replace=False))
    t_act2 = 10.0 + (vox2[ids2, 0] * 0.8 + vox2[ids2, 1] * 0.6) / 0.9
    out.append(("analysis_sheet", vox2, ids2, electrograms(vox2[ids2], t_act2, 120, 1.0, rng)))
    # sparse electrodes in a 30 mm box: many with fewer than 4 points within 8 mm (NaN rows)
    vox3 = rng.uniform(0.0, 30.0, size=(400, 3))
    ids3 = np.sort(rng.choice(vox3.shape[0], size=60, replace=False))
    t_act3 = 15.0 + np.linalg.norm(vox3[ids3] - vox3[ids3[3]], axis=1) / 0.5
    out.append(("analysis_sparse", vox3, ids3, electrograms(vox3[ids3], t_act3, 200, 2.0, rng)))
    return out


def main():
    lat_map, cv = _load()
    for name, vox, ids, egm in cases():
        lat = lat_map.compute_electrode_lat(egm)
        vec, mag, mean = cv.compute({"electrogram_unipolar": egm},
                                    {"voxel": vox, "voxel_id_of_simulation_electrode": ids})
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), voxel=vox, electrode_ids=ids, egm=egm,
                            lat_electrode=np.asarray(lat), cv_vectors=vec, cv_magnitudes=mag,
                            cv_mean=np.float64(mean))
        print(name, egm.shape, "lat range", int(np.min(lat)), int(np.max(lat)), "nan rows",
              int(np.isnan(mag).sum()), "mean", mean)


if __name__ == "__main__":
    main()
