"""Compile the reference's inputs into one device instance (``phs_instance_desc``).

Input is exactly what ``simulation/simulation_gpu.py::compute`` receives:
``n_voxel``, ``P_2d`` (n, 21), ``geometry_data`` ({'neighbor_id_2d', 'Delta'}),
``simulation_parameters`` and ``arrhythmia_parameters``.  The reference builds a
CSR Laplacian with a Python loop (simulation/simulation_gpu.py:138-225); here the
same operator is kept matrix-free as a compacted table:

* ``nb6[n, k]``   the six face neighbours, ``-1`` remapped to 0 exactly as the
                  reference does before building L (simulation_gpu.py:296-297);
* ``coef6[n, k]`` ``P_2d[n,20] / (4 Delta^2) * P_2d[n,k]`` with the permanent
                  block (node_flag == 4) applied to column 20 (simulation_gpu.py:312-313);
* ``vflags[n]``   S1 / S2 membership and the temporary block (node_flag == 3);

so ``(L u)[n] = sum_k coef6[n,k] * (u[nb6[n,k]] - u[n])`` is the reference's
row n (its diagonal is minus the sum of the neighbour entries).

Anisotropic tensors (D0 != I) add the cross terms of simulation_gpu.py:171-217.
The face ones (P_2d[:,6..8]) enter the +d neighbour with + and the -d neighbour
with -, so they fold into ``coef6``; the edge ones (P_2d[:,9..14]) are six
antisymmetric pairs per row, ``coef_edge[n,p] * (u[a] - u[b])`` with
``(a, b) = nb_edge[n, 2p:2p+2]``.  Both forms keep the row sum at zero, as the
reference's diagonal does.
"""
import numpy as np

from . import _lib
from .simulation import pacing


def _spread_bits(x):
    """Spread the low 21 bits of x to every third bit (Morton interleave)."""
    x = x.astype(np.uint64) & np.uint64(0x1fffff)
    for sh, m in ((32, 0x1f00000000ffff), (16, 0x1f0000ff0000ff), (8, 0x100f00f00f00f00f),
                  (4, 0x10c30c30c30c30c3), (2, 0x1249249249249249)):
        x = (x | (x << np.uint64(sh))) & np.uint64(m)
    return x


def locality_order(geometry_data, n, kind="rows"):
    """Device order of the voxels, from the lattice coordinates ``voxel / Delta``.

    ``rows`` (default): lexicographic (z, y, x) with x fastest, so rows along x
    are contiguous; inside a tile of consecutive voxels the +-x and most +-y
    neighbours are present, and the neighbours outside the tile are the +-z ones
    for whole warps at a time (the stencil's recomputation stays uniform across
    a warp).  ``morton``: Z-curve order (fewer neighbours outside a tile, but
    they are scattered across the lanes of a warp).
    Returns ``order`` (device index -> caller index), or None when the geometry
    carries no coordinates."""
    vox = geometry_data.get('voxel') if hasattr(geometry_data, 'get') else None
    if vox is None:
        return None
    vox = np.asarray(vox, dtype=np.float64)
    if vox.shape != (n, 3):
        return None
    ijk = np.rint(vox / float(geometry_data['Delta'])).astype(np.int64)
    ijk -= ijk.min(axis=0)
    if kind == "rows":
        return np.lexsort((ijk[:, 0], ijk[:, 1], ijk[:, 2]))
    if ijk.max() >= (1 << 21):
        return None
    code = _spread_bits(ijk[:, 0]) | (_spread_bits(ijk[:, 1]) << np.uint64(1)) | \
        (_spread_bits(ijk[:, 2]) << np.uint64(2))
    return np.argsort(code, kind='stable')


# Edge cross-term pairs (+ neighbour column, - neighbour column, P_2d column),
# in the order of simulation/simulation_gpu.py:199-206.
EDGE_PAIRS = ((6, 8, 9), (9, 7, 10), (14, 16, 11), (17, 15, 12), (10, 12, 13), (13, 11, 14))


class CompiledInstance:
    """Host arrays + scalars of one instance, and the ctypes descriptor over them."""

    def __init__(self, **kw):
        self.__dict__.update(kw)
        self._desc = None

    def desc(self):
        """ctypes ``phs_instance_desc`` referencing this object's arrays (keep self alive)."""
        d = _lib.InstanceDesc()
        d.n_voxel = self.n_voxel
        d.model = self.model
        d.restart = self.restart
        d.nb6 = _lib.ptr(self.nb6, _lib.ctypes.c_int32)
        iso = getattr(self, "cw", None) is not None
        d.coef6 = None if iso else _lib.ptr(self.coef6, _lib.ctypes.c_double)
        d.cw = _lib.ptr(self.cw, _lib.ctypes.c_double) if iso else None
        d.mask6 = _lib.ptr(self.mask6, _lib.ctypes.c_uint8) if iso else None
        d.vflags = _lib.ptr(self.vflags, _lib.ctypes.c_uint8)
        d.vparams = _lib.ptr(self.vparams, _lib.ctypes.c_double) if self.vparams is not None else None
        for i in range(5):
            d.params[i] = float(self.params[i])
        d.dt = self.dt
        d.j_stim = self.j_stim
        d.n_steps = self.n_steps
        d.stim = _lib.ptr(self.stim, _lib.ctypes.c_uint8)
        d.tblock_steps = self.tblock_steps
        d.sample_stride = self.sample_stride
        d.n_samples = self.n_samples
        d.save_h = self.save_h
        d.full_cycles = self.full_cycles
        d.u0 = self.u0
        d.h0 = self.h0
        d.tol = self.tol
        d.atol = self.atol
        d.maxiter = self.maxiter
        d.guess = int(getattr(self, "guess", 0))
        edge = getattr(self, "coef_edge", None) is not None
        d.nb_edge = _lib.ptr(self.nb_edge, _lib.ctypes.c_int32) if edge else None
        d.coef_edge = _lib.ptr(self.coef_edge, _lib.ctypes.c_double) if edge else None
        self._desc = d
        return d

    def to_caller(self, a):
        """Map device-ordered voxel data (last axis) back to the caller's order."""
        return a if self.inv is None else a[..., self.inv]

    def sample_times(self, n_saved):
        """physical_time of the first ``n_saved`` samples: the sample taken after
        step k is stamped ``k * dt * time_scale`` (simulation_gpu.py:395-407)."""
        if self.sample_stride > 0:
            steps = np.arange(n_saved, dtype=np.int64) * self.sample_stride
        else:
            steps = np.arange(n_saved, dtype=np.int64)
        return (steps.astype(np.float64) * self.dt) * self.time_scale


def step_counts(simulation_parameters):
    """(n_steps, n_samples, stride), simulation/simulation_gpu.py:286-290, 355-356."""
    t_final = float(simulation_parameters['t_final'])
    dt = simulation_parameters['dt']
    ts = simulation_parameters['time_scale']
    if simulation_parameters['heart_model_flag'] == 0:
        n_samples = int(np.round(t_final))
    else:
        n_samples = int(np.round(t_final * ts))
    n_steps = int(np.round(t_final / dt))
    stride = int(1 / (dt * ts))
    return n_steps, n_samples, stride


def tblock_steps(n_steps, dt):
    """Steps run with the temporary-block operator: model_time = step*dt in
    [0, 350*dt) (simulation/simulation_gpu.py:365-370)."""
    t = np.arange(n_steps, dtype=np.float64) * dt
    on = (t >= 0) & (t < 350 * dt)
    k = int(on.sum())
    if k and not on[:k].all():
        raise AssertionError("temporary block window is not a prefix of the run")
    return k


def instance_scalars(simulation_parameters, arrhythmia_parameters, *, full_cycles=True, tol=1e-5, atol=1e-5,
                     restart=50, maxiter=10000, pacing_duration=None, save_h=True, max_steps=None, guess=None):
    """The per-instance scalars and the pacing schedule (everything but the
    per-voxel tables), and the S1 / S2 voxel ids (caller order, int64)."""
    model = int(simulation_parameters['heart_model_flag'])
    if model not in (0, 1):
        raise ValueError("heart_model_flag must be 0 (Mitchell-Schaeffer) or 1 (Aliev-Panfilov)")
    flag = simulation_parameters['arrhythmia_flag']
    dt = simulation_parameters['dt']
    n_steps, n_samples, stride = step_counts(simulation_parameters)
    if max_steps is not None:
        n_steps = min(n_steps, int(max_steps))
    s1, s2, s1_t, jmag, pdur, s2_t = pacing.assign_pacing_parameters(
        arrhythmia_parameters, flag, simulation_parameters, pacing_duration)
    stim = pacing.schedule(n_steps, dt, arrhythmia_parameters, simulation_parameters, flag, s1_t, pdur, s2_t)
    s1 = np.atleast_1d(np.asarray(s1, dtype=np.int64)) if np.size(s1) else np.zeros(0, np.int64)
    s2 = np.atleast_1d(np.asarray(s2, dtype=np.int64)) if np.size(s2) else np.zeros(0, np.int64)
    u0, h0 = (0.0, 1.0) if model == 0 else (0.0, 0.0)
    sc = dict(model=model, restart=int(min(restart, 50)), dt=float(dt), j_stim=float(jmag), n_steps=int(n_steps),
              stim=np.ascontiguousarray(stim, dtype=np.uint8), sample_stride=int(stride), n_samples=int(n_samples),
              save_h=int(bool(save_h)), full_cycles=int(bool(full_cycles)), u0=u0, h0=h0, tol=float(tol),
              atol=float(atol), maxiter=int(maxiter), time_scale=simulation_parameters['time_scale'],
              guess=int((not full_cycles) if guess is None else bool(guess)))
    return sc, s1, s2


def compile_instance(n_voxel, P_2d, geometry_data, simulation_parameters, arrhythmia_parameters, *,
                     full_cycles=True, tol=1e-5, atol=1e-5, restart=50, maxiter=10000,
                     pacing_duration=None, save_h=True, max_steps=None, reorder="rows", guess=None):
    """Build a :class:`CompiledInstance` with the reference's semantics.

    ``full_cycles=True`` keeps CuPy's GMRES(restart) behaviour (the plain
    drop-in); ``False`` stops each solve as soon as the Givens residual
    estimate meets the same tolerance.  With ``reorder`` ("rows" by default,
    "morton", or False) and voxel coordinates in ``geometry_data``, voxels are
    stored in that order on the device; results are mapped back with
    :meth:`CompiledInstance.to_caller`.  ``guess`` (default: on for the
    early-exit form, off for the plain form) starts each solve from u* plus the
    previous step's diffusion increment instead of u*.
    """
    n = int(n_voxel)
    P = np.asarray(P_2d, dtype=np.float64)
    if P.shape != (n, 21):
        raise ValueError(f"P_2d must be ({n}, 21), got {P.shape}")
    nb = np.asarray(geometry_data['neighbor_id_2d'])
    if nb.ndim != 2 or nb.shape[0] != n or nb.shape[1] < 6:
        raise ValueError("neighbor_id_2d must be (n_voxel, 18)")
    if np.any(nb[:, :6] < -1) or np.any(nb[:, :6] >= n):
        raise ValueError("neighbor_id_2d holds indices outside [-1, n_voxel)")
    cross_face = np.any(P[:, 6:9] != 0)
    cross_edge = np.any(P[:, 9:15] != 0)
    if cross_edge and (nb.shape[1] < 18 or np.any(nb[:, 6:18] < -1) or np.any(nb[:, 6:18] >= n)):
        raise ValueError("edge cross terms need neighbor_id_2d columns 6..17 in [-1, n_voxel)")
    Delta = float(geometry_data['Delta'])
    sc, s1, s2 = instance_scalars(simulation_parameters, arrhythmia_parameters, full_cycles=full_cycles, tol=tol,
                                  atol=atol, restart=restart, maxiter=maxiter, pacing_duration=pacing_duration,
                                  save_h=save_h, max_steps=max_steps, guess=guess)
    node_flag = np.asarray(arrhythmia_parameters['node_flag'])

    c = P[:, 20].copy()
    c[node_flag == 4] = 0.0                       # permanent block
    nb6 = nb[:, :6].astype(np.int64).copy()
    nb6[nb6 == -1] = 0                            # the reference's -1 -> 0 remap
    Dc = c / (4 * Delta ** 2)
    coef6 = Dc[:, None] * P[:, :6]
    if cross_face:
        sign = np.array([1.0, -1.0, 1.0, -1.0, 1.0, -1.0])
        coef6 = coef6 + (Dc[:, None] * P[:, [6, 6, 7, 7, 8, 8]]) * sign
    nb_edge = coef_edge = None
    if cross_edge:
        pairs = np.array(EDGE_PAIRS)
        nb_edge = nb[:, pairs[:, :2].ravel()].astype(np.int64)
        nb_edge[nb_edge == -1] = 0
        coef_edge = Dc[:, None] * P[:, pairs[:, 2]]
    vflags = np.zeros(n, dtype=np.uint8)
    vflags[s1] |= _lib.VFLAG_S1
    vflags[s2] |= _lib.VFLAG_S2
    vflags[node_flag == 3] |= _lib.VFLAG_TBLOCK

    mp = P[:, 15:20]
    uniform = bool(np.all(mp == mp[0:1]))
    params = mp[0].copy() if n else np.zeros(5)
    vparams = None if uniform else np.ascontiguousarray(mp)
    # isotropic rows: every non-zero coefficient of a row is the same value
    nz = coef6 != 0
    cw = np.where(nz.any(axis=1), coef6[np.arange(n), nz.argmax(axis=1)], 0.0)
    mask6 = (nz * (1 << np.arange(6))).sum(axis=1).astype(np.uint8)
    if not np.array_equal(coef6, cw[:, None] * nz):
        cw = mask6 = None
    order = locality_order(geometry_data, n, reorder) if reorder else None
    if order is not None and np.array_equal(order, np.arange(n)):
        order = None
    inv = None
    if order is not None:
        inv = np.empty(n, dtype=np.int64)
        inv[order] = np.arange(n)
        nb6 = inv[nb6[order]]
        coef6 = coef6[order]
        vflags = vflags[order]
        if cw is not None:
            cw, mask6 = cw[order], mask6[order]
        if vparams is not None:
            vparams = np.ascontiguousarray(vparams[order])
        if nb_edge is not None:
            nb_edge = inv[nb_edge[order]]
            coef_edge = coef_edge[order]
    sc["tblock_steps"] = tblock_steps(sc["n_steps"], sc["dt"]) if np.any(node_flag == 3) else 0
    return CompiledInstance(
        n_voxel=n, nb6=np.ascontiguousarray(nb6, dtype=np.int32),
        coef6=np.ascontiguousarray(coef6), vflags=vflags, vparams=vparams, params=params,
        Delta=Delta, order=order, inv=inv, **sc,
        cw=None if cw is None else np.ascontiguousarray(cw), mask6=None if mask6 is None else np.ascontiguousarray(mask6),
        nb_edge=None if nb_edge is None else np.ascontiguousarray(nb_edge, dtype=np.int32),
        coef_edge=None if coef_edge is None else np.ascontiguousarray(coef_edge))
