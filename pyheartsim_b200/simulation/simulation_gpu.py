"""Drop-in for the reference's ``simulation/simulation_gpu.py``.

``compute(n_voxel, P_2d, geometry_data, simulation_parameters,
arrhythmia_parameters)`` has the reference's signature and returns the same
arrays ``(u_hist (S, n), h_hist (S, n), physical_time (S,))``
(simulation/simulation_gpu.py:261-409).  The whole run executes on the GPU
through ``phs_simulate`` (include/phs.h): RK4 reaction, the CN right-hand
side and restarted GMRES in one persistent sm_100a kernel, the stimulus
schedule and the 1 kHz history on the device.

Differences from the reference, all deliberate:
* the plain form computes in FP64 (the reference stores FP32); pass
  ``dtype=np.float32`` for FP32 storage (FP64 dots and norms are kept);
* ``fast=True`` replaces CuPy's full 50-step cycles by a Givens early exit at
  the same tolerance (``tol`` relative, ``atol`` absolute);
* fewer than 5 steps is allowed (the reference's progress print divides by
  ``steps // 5``, simulation_gpu.py:359); a zero cycle length with
  ``arrhythmia_flag == 0`` raises instead of looping forever (pacing.py:138).
"""
import warnings

import numpy as np

from .. import _lib
from .. import instance as _instance


def compute(n_voxel, P_2d, geometry_data, simulation_parameters, arrhythmia_parameters, *,
            dtype=np.float64, fast=False, tol=1e-5, atol=1e-5, restart=None, method='gmres',
            pacing_duration=None, return_lat=False, return_info=False, max_steps=None, maxiter=10000):
    if method != 'gmres':
        raise ValueError(f"Unknown solver method: {method}. Use 'gmres'")
    precision = _lib.PREC_F64 if np.dtype(dtype) == np.float64 else _lib.PREC_F32
    if restart is None:
        restart = 20 if fast else 50
    inst = _instance.compile_instance(n_voxel, P_2d, geometry_data, simulation_parameters, arrhythmia_parameters,
                            full_cycles=not fast, tol=tol, atol=atol, restart=restart,
                            pacing_duration=pacing_duration, max_steps=max_steps, maxiter=maxiter)
    dt_np = _lib.np_dtype(precision)
    S, n = inst.n_samples, inst.n_voxel
    u_hist = np.zeros((S, n), dtype=dt_np)
    h_hist = np.zeros((S, n), dtype=dt_np)
    lat = np.full(n, -1, dtype=np.int32)
    n_saved = _lib.ctypes.c_int32(0)
    info = _lib.InstanceInfo()
    desc = inst.desc()
    st = _lib.lib().phs_simulate(_lib.ctypes.byref(desc), precision, _lib.vptr(u_hist), _lib.vptr(h_hist),
                                 _lib.ptr(lat, _lib.ctypes.c_int32), _lib.ctypes.byref(n_saved),
                                 _lib.ctypes.byref(info))
    if st == _lib.PHS_WARN_NO_CONVERGE:
        warnings.warn(f"Warning: GPU GMRES did not converge ({info.nonconverged} solves hit maxiter)")
    else:
        _lib.check(st, "phs_simulate")
    k = int(n_saved.value)
    t = inst.sample_times(k)
    t = t.astype(dt_np)
    out = (inst.to_caller(u_hist[:k]), inst.to_caller(h_hist[:k]), t)
    if return_lat:
        out = out + (inst.to_caller(lat),)
    if return_info:
        out = out + ({"steps": int(info.step), "arnoldi_steps": int(info.arnoldi_steps),
                      "solves": int(info.solves), "max_arnoldi": int(info.max_arnoldi),
                      "nonconverged": int(info.nonconverged)},)
    return out
