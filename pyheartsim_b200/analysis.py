"""Electrogram analysis on the GPU (C ABI ``phs_electrode_lat``,
``phs_conduction_velocity``, ``phs_interpolate_lat``), with the reference's
signatures:

* :func:`compute_electrode_lat` -- utility/lat_map.py:20-27;
* :func:`interpolate_lat` -- utility/lat_map.py:29-46 (linear inside the
  electrodes' Delaunay triangulation, nearest electrode outside);
* :func:`compute` -- utility/conduction_velocity.py:23-70 (electrode LAT, then
  a least-squares plane per electrode over the electrodes within 8 mm).

Inputs may be numpy arrays (copied to the device) or CUDA tensors (used in
place, e.g. an electrogram still on the device); results are numpy.
"""
import ctypes

import numpy as np

from . import _lib

RADIUS_MM = 8.0   # utility/conduction_velocity.py:37


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("analysis needs a CUDA device")
    return torch


def _dev(torch, a, dtype=None):
    t = a if isinstance(a, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(a))
    t = t.to(device="cuda")
    if dtype is not None:
        t = t.to(dtype)
    return t.contiguous()


def electrode_lat_device(egm, stream=None):
    """Electrode LAT of a (T, n_e) float32/float64 signal; int32 CUDA tensor."""
    torch = _torch()
    e = _dev(torch, egm)
    if e.dtype not in (torch.float32, torch.float64):
        e = e.to(torch.float64)
    T, ne = e.shape
    out = torch.empty(ne, dtype=torch.int32, device=e.device)
    s = (stream or torch.cuda.current_stream()).cuda_stream
    _lib.check(_lib.lib().phs_electrode_lat(T, ne, ctypes.c_void_p(e.data_ptr()), int(e.dtype == torch.float64),
                                            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(s)),
               "phs_electrode_lat")
    return out


def compute_electrode_lat(electrode_signal):
    """Drop-in of utility/lat_map.py:20-27 (int64 numpy result)."""
    return electrode_lat_device(electrode_signal).cpu().numpy().astype(np.int64)


def conduction_velocity(xyz, lat, radius=RADIUS_MM, stream=None):
    """(vectors (n, 3), speeds (n,), mean speed ignoring NaN)."""
    torch = _torch()
    x = _dev(torch, xyz, torch.float64)
    l = _dev(torch, lat, torch.float64)
    n = x.shape[0]
    vec = torch.empty((n, 3), dtype=torch.float64, device=x.device)
    mag = torch.empty(n, dtype=torch.float64, device=x.device)
    s = (stream or torch.cuda.current_stream()).cuda_stream
    _lib.check(_lib.lib().phs_conduction_velocity(n, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(l.data_ptr()),
                                                  float(radius), ctypes.c_void_p(vec.data_ptr()),
                                                  ctypes.c_void_p(mag.data_ptr()), ctypes.c_void_p(s)),
               "phs_conduction_velocity")
    mag_h = mag.cpu().numpy()
    return vec.cpu().numpy(), mag_h, float(np.nanmean(mag_h)) if np.any(~np.isnan(mag_h)) else float("nan")


def compute(simulation_results, geometry_data):
    """Drop-in of utility/conduction_velocity.py:23 -> (vectors, speeds, mean)."""
    lat = electrode_lat_device(simulation_results['electrogram_unipolar'])
    ids = np.asarray(geometry_data['voxel_id_of_simulation_electrode'])
    xyz = np.asarray(geometry_data['voxel'], dtype=np.float64)[ids, :]
    return conduction_velocity(xyz, lat)


def interpolate_lat(voxel, electrode_voxel, lat_electrode, stream=None):
    """Drop-in of utility/lat_map.py:29-46: electrode LAT spread over the voxels.

    As the reference: the dimensions in which the electrodes do not vary are
    dropped; the electrodes are triangulated (scipy.spatial.Delaunay, on the
    host -- the same Qhull triangulation LinearNDInterpolator builds); voxels
    inside the hull get the barycentric (linear) interpolation, voxels outside
    it the LAT of the nearest electrode.  The point location, interpolation and
    nearest search run on the GPU (``phs_interpolate_lat``).  Returns a float64
    numpy array (n_v,)."""
    from scipy.spatial import Delaunay
    torch = _torch()
    ev = np.asarray(electrode_voxel, dtype=np.float64)
    vx = np.asarray(voxel, dtype=np.float64)
    active = np.ptp(ev, axis=0) > 0
    er = np.ascontiguousarray(ev[:, active])
    vr = np.ascontiguousarray(vx[:, active])
    ndim = er.shape[1]
    if ndim not in (2, 3):
        raise ValueError(f"electrodes span {ndim} dimension(s); the triangulation needs 2 or 3")
    tri = Delaunay(er)
    ns = tri.simplices.shape[0]
    nbr = np.ascontiguousarray(tri.neighbors, dtype=np.int32)
    if nbr.max() >= ns:
        raise ValueError("inconsistent triangulation")
    d = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), device="cuda").to(dt)
    vals = d(np.asarray(lat_electrode, dtype=np.float64))
    pts, epts = d(vr), d(er)
    simp = d(tri.simplices, torch.int32)
    trans = d(tri.transform.reshape(ns, -1))
    nb = d(nbr, torch.int32)
    lo, hi = d(tri.min_bound), d(tri.max_bound)
    out = torch.empty(vr.shape[0], dtype=torch.float64, device=pts.device)
    s = (stream or torch.cuda.current_stream()).cuda_stream
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    _lib.check(_lib.lib().phs_interpolate_lat(vr.shape[0], ndim, p(pts), er.shape[0], p(epts), p(vals), ns, p(simp),
                                              p(trans), p(nb), p(lo), p(hi), p(out), ctypes.c_void_p(s)),
               "phs_interpolate_lat")
    return out.cpu().numpy()
