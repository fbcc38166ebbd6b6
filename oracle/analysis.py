"""CPU oracle of the electrogram analysis: electrode activation times and
conduction velocity.

TEST INFRASTRUCTURE ONLY (imported by ``tests/`` and ``bench.py``'s CPU leg;
never by the product package).

Restates, in numpy/scipy, jiyuehe/PyHeartSim:

* ``utility/lat_map.py:20-27``  compute_electrode_lat: argmax over time of the
  negative first difference of each electrode's signal, shifted so that the
  earliest electrode is 0;
* ``utility/lat_map.py:29-46``  interpolate_lat: linear interpolation of the
  electrode LAT over the voxels on the electrodes' Delaunay triangulation
  (scipy), nearest electrode outside the hull;
* ``utility/conduction_velocity.py:23-70``  compute: for every electrode, the
  electrodes within 8 mm (itself included), a least-squares plane
  ``lat = a x + b y + c z + d`` (numpy.linalg.lstsq, minimum-norm), velocity
  ``grad / |grad|^2`` and speed ``1 / |grad|`` when ``|grad|^2 > 1e-8``, NaN
  with fewer than 4 points; the mean speed ignores NaN.

Pinned against ``tests/golden/analysis_*.npz`` (the reference's own functions
run on seeded electrograms, ``tests/golden/make_golden_analysis.py``).
"""
import numpy as np
from scipy.spatial import cKDTree


def compute_electrode_lat(electrode_signal):
    """utility/lat_map.py:20-27."""
    s = np.asarray(electrode_signal)
    idx = np.argmax(-np.diff(s, axis=0), axis=0)
    return idx - np.min(idx)


def conduction_velocity(xyz, lat, radius=8.0):
    """utility/conduction_velocity.py:33-64 on electrode coordinates ``xyz``
    (n, 3) and activation times ``lat`` (n,).  Returns (vectors, speeds, mean)."""
    xyz = np.asarray(xyz, dtype=np.float64)
    lat = np.asarray(lat)
    n = xyz.shape[0]
    tree = cKDTree(xyz)
    vec = np.full((n, 3), np.nan)
    mag = np.full(n, np.nan)
    for i in range(n):
        idx = tree.query_ball_point(xyz[i], radius)
        if len(idx) < 4:
            continue
        A = np.column_stack((xyz[idx], np.ones(len(idx))))
        coef = np.linalg.lstsq(A, lat[idx], rcond=None)[0]
        g = coef[:3]
        g2 = np.dot(g, g)
        if g2 > 1e-8:
            vec[i] = g / g2
            mag[i] = 1.0 / np.linalg.norm(g)
    return vec, mag, np.nanmean(mag)


def compute(simulation_results, geometry_data):
    """Drop-in signature of utility/conduction_velocity.py:23."""
    lat = compute_electrode_lat(simulation_results['electrogram_unipolar'])
    xyz = geometry_data['voxel'][geometry_data['voxel_id_of_simulation_electrode'], :]
    return conduction_velocity(xyz, lat)


def interpolate_lat(voxel, electrode_voxel, lat_electrode):
    """utility/lat_map.py:29-46: drop the dimensions in which the electrodes do
    not vary, interpolate linearly on the Delaunay triangulation of the
    electrodes (scipy's LinearNDInterpolator, NaN outside the hull), and fill
    the voxels outside the hull with the nearest electrode's value (scipy's
    NearestNDInterpolator)."""
    from scipy.interpolate import LinearNDInterpolator, NearestNDInterpolator
    ev = np.asarray(electrode_voxel, dtype=np.float64)
    vx = np.asarray(voxel, dtype=np.float64)
    active = np.ptp(ev, axis=0) > 0
    er, vr = ev[:, active], vx[:, active]
    out = LinearNDInterpolator(er, lat_electrode)(vr)
    nan = np.isnan(out)
    if np.any(nan):
        out[nan] = NearestNDInterpolator(er, lat_electrode)(vr[nan])
    return out
