"""Drop-in for the reference's ``simulation/unipolar_electrogram_gpu.py``.

``compute(electrode_xyz, voxel, D0, c_voxel, action_potential, Delta,
neighbor_id_2d, batch_size=50)`` returns the normalised unipolar electrogram
(T, n_e) like simulation/unipolar_electrogram_gpu.py:71-152.

The reference adds one FP32 atomic per (voxel, electrode, time).  Here the
gradient stencil (simulation/unipolar_electrogram_equation_parts.py:60-103),
the distances with the 1 mm clamp (:41-58), c_voxel and D0 are folded into a
lead field M (n_v x n_e) built in FP64 on the device, and the electrogram is
the contraction V @ M:
* ``mode='fp64'`` (default, the plain drop-in): FP64 lead field and contraction;
* ``mode='bf16x3'``: V and M split into BF16 hi/lo pairs, three tcgen05
  products with FP32 accumulation (relative L2 error ~1e-5 on rotor data).
``batch_size`` is accepted for signature compatibility; the contraction does
not need time batches.
"""
import numpy as np

from .. import _lib


def incoming_gradient_terms(neighbor_id_2d):
    """CSR (ptr, src, dir) of the gradient terms that reach each voxel w.

    Voxel v contributes +g/(2 Delta) to its +d neighbour and -g/(2 Delta) to its
    -d neighbour when both exist (the reference zeroes the gradient otherwise,
    unipolar_electrogram_equation_parts.py:91-101).  dir = +-(d+1).
    """
    nb = np.asarray(neighbor_id_2d)
    n = nb.shape[0]
    tgt, src, dirs = [], [], []
    v = np.arange(n, dtype=np.int64)
    for d in range(3):
        p, m = nb[:, 2 * d], nb[:, 2 * d + 1]
        ok = (p >= 0) & (m >= 0)
        tgt += [p[ok], m[ok]]
        src += [v[ok], v[ok]]
        dirs += [np.full(int(ok.sum()), d + 1, np.int8), np.full(int(ok.sum()), -(d + 1), np.int8)]
    tgt = np.concatenate(tgt).astype(np.int64)
    src = np.concatenate(src).astype(np.int32)
    dirs = np.concatenate(dirs).astype(np.int8)
    order = np.argsort(tgt, kind='stable')
    ptr = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(np.bincount(tgt, minlength=n), out=ptr[1:])
    return ptr, np.ascontiguousarray(src[order]), np.ascontiguousarray(dirs[order])


def d0_array(D0, n_voxel):
    """(n, 9) row-major tensors, or None when every tensor is the identity."""
    if D0 is None:
        return None
    D = np.asarray(D0, dtype=np.float64).reshape(n_voxel, 9)
    if np.all(D == np.eye(3).reshape(1, 9)):
        return None
    return np.ascontiguousarray(D)


def compute(electrode_xyz, voxel, D0, c_voxel, action_potential, Delta, neighbor_id_2d, batch_size=50, *,
            mode='fp64', dtype=np.float64):
    V = np.ascontiguousarray(np.asarray(action_potential, dtype=np.float64))
    xyz = np.ascontiguousarray(np.asarray(voxel, dtype=np.float64))
    exyz = np.ascontiguousarray(np.asarray(electrode_xyz, dtype=np.float64).reshape(-1, 3))
    c = np.ascontiguousarray(np.asarray(c_voxel, dtype=np.float64))
    T, n_v = V.shape
    n_e = exyz.shape[0]
    if xyz.shape != (n_v, 3) or c.shape != (n_v,):
        raise ValueError("voxel must be (n_v, 3) and c_voxel (n_v,) matching action_potential (T, n_v)")
    ptr, src, dirs = incoming_gradient_terms(neighbor_id_2d)
    D = d0_array(D0, n_v)
    m = {'fp64': _lib.EGM_F64, 'bf16x3': _lib.EGM_BF16X3}[mode]
    out = np.zeros((T, n_e), dtype=np.float64)
    C = _lib.ctypes
    st = _lib.lib().phs_electrogram(T, n_v, n_e, _lib.ptr(V, C.c_double), _lib.ptr(xyz, C.c_double),
                                    _lib.ptr(exyz, C.c_double), _lib.ptr(c, C.c_double),
                                    _lib.ptr(D, C.c_double) if D is not None else None,
                                    _lib.ptr(ptr, C.c_int32), _lib.ptr(src, C.c_int32), _lib.ptr(dirs, C.c_int8),
                                    float(Delta), m, _lib.ptr(out, C.c_double))
    _lib.check(st, "phs_electrogram")
    return out.astype(dtype, copy=False)
