"""Generate ``tests/golden/analysis_*.npz``: electrode LAT, conduction
velocity and the LAT map interpolated onto voxels, computed by the reference's
OWN, unmodified ``utility/lat_map.py::compute_electrode_lat``,
``utility/lat_map.py::interpolate_lat`` and
``utility/conduction_velocity.py::compute``.

Test infrastructure only.  Needs a checkout of the reference, named by the
environment variable ``PHS_REFERENCE_DIR``; it exists only where the fixtures
are generated, the fixtures are committed and nothing at test time reads the
reference.  ``lat_map.py`` imports
matplotlib, scipy's interpolators and the reference's ``common`` module for its
plotting helpers; matplotlib and ``common`` are replaced by empty stub modules
(the two functions used here touch neither).

Inputs are seeded synthetic electrograms: a downstroke ``-tanh((t - t_act)/w)``
per electrode, with activation times from a point source (3-D shell surface)
or a plane wave (flat sheet, where every electrode has the same z and the
plane fit is rank-deficient), plus small noise.

``analysis_interp.npz`` holds the interpolation cases (``interpolate_lat``
of the reference on the electrode LAT of the cases above, with the electrodes
moved off the lattice by up to 0.05 mm, plus a 4 x 4
electrode grid 1 mm above a sheet, whose constant z is dropped and whose
border voxels lie outside the electrode hull); each case is checked to have no
voxel whose two nearest electrodes are at equal distance, so the nearest-
electrode fallback has one answer.

Run:  PHS_REFERENCE_DIR=<reference checkout> python tests/golden/make_golden_analysis.py
"""
import importlib.util
import os
import sys
import types

import numpy as np

REF = os.environ.get("PHS_REFERENCE_DIR", "")
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


def _check_no_nearest_ties(vox_r, el_r):
    """No voxel outside the electrode hull (the ones the nearest-electrode
    fallback fills) has two electrodes at (nearly) the same distance."""
    from scipy.interpolate import LinearNDInterpolator
    outside = np.isnan(LinearNDInterpolator(el_r, np.zeros(el_r.shape[0]))(vox_r))
    vox_r = vox_r[outside]
    d2 = ((vox_r[:, None, :] - el_r[None, :, :]) ** 2).sum(axis=2)
    s = np.sort(d2, axis=1)
    assert np.all(s[:, 1] - s[:, 0] > 1e-9 * np.maximum(s[:, 1], 1.0)), "nearest-electrode tie"


def interp_cases(lat_of):
    """(name, voxel, electrode_xyz) of the interpolation fixture."""
    from pyheartsim_b200 import synthetic
    out = []
    jit = np.random.default_rng(5)
    for name, vox, ids, _ in cases():
        # electrodes at the chosen voxels, moved by up to 0.05 mm in the
        # dimensions they span (a constant dimension stays constant), so that no
        # voxel outside their hull is equidistant from two of them
        el = vox[ids].copy()
        span = np.ptp(el, axis=0) > 0
        el[:, span] += jit.uniform(-0.05, 0.05, size=(el.shape[0], int(span.sum())))
        out.append((name, vox, el, lat_of[name]))
    i, j = np.meshgrid(np.arange(40), np.arange(30), indexing="ij")
    vox = np.stack([i.ravel() * 0.4, j.ravel() * 0.4, np.zeros(i.size)], axis=1)
    el = synthetic.electrodes_grid(40, 30, 0.4)
    rng = np.random.default_rng(11)
    out.append(("grid_above_sheet", vox, el, rng.integers(0, 60, size=el.shape[0])))
    return out


def main():
    if not REF or not os.path.isdir(os.path.join(REF, "utility")):
        raise SystemExit("set PHS_REFERENCE_DIR to a checkout of the reference")
    lat_map, cv = _load()
    lat_of = {}
    for name, vox, ids, egm in cases():
        lat = lat_map.compute_electrode_lat(egm)
        vec, mag, mean = cv.compute({"electrogram_unipolar": egm},
                                    {"voxel": vox, "voxel_id_of_simulation_electrode": ids})
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), voxel=vox, electrode_ids=ids, egm=egm,
                            lat_electrode=np.asarray(lat), cv_vectors=vec, cv_magnitudes=mag,
                            cv_mean=np.float64(mean))
        print(name, egm.shape, "lat range", int(np.min(lat)), int(np.max(lat)), "nan rows",
              int(np.isnan(mag).sum()), "mean", mean)
        lat_of[name] = np.asarray(lat)
    fx = {}
    for k, (name, vox, el, lat) in enumerate(interp_cases(lat_of)):
        active = np.ptp(el, axis=0) > 0
        lin = np.asarray(lat_map.interpolate_lat(vox, el, lat), dtype=np.float64)
        _check_no_nearest_ties(vox[:, active], el[:, active])
        fx.update({f"{k}_voxel": vox, f"{k}_electrode": el, f"{k}_lat_electrode": np.asarray(lat),
                   f"{k}_lat_voxel": lin})
        print("interp", name, vox.shape[0], "voxels", el.shape[0], "electrodes, dims", int(active.sum()),
              "outside the hull", int(np.isnan(lat_map.LinearNDInterpolator(el[:, active], lat)(vox[:, active])).sum()))
    fx["names"] = np.array([c[0] for c in interp_cases(lat_of)])
    np.savez_compressed(os.path.join(HERE, "analysis_interp.npz"), **fx)


if __name__ == "__main__":
    main()
