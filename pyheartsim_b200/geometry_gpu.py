"""Geometry and operator tables built on the GPU.

The reference prepares the stepper's inputs on the host: one KDTree query per
neighbour (utility/voxelization.py:102-152, ``find_neighbor_voxel_ids``), a loop
for P_2d (simulation/equation_parts.py:36-114, ``heart_model_equation_parts``)
and a loop for the CSR Laplacian (simulation/simulation_gpu.py:138-225).  This
module runs the same steps on the device through the C ABI
(``phs_lattice_neighbors``, ``phs_equation_parts``, ``phs_operator_flags``,
``phs_operator_tables``):

* :func:`find_neighbor_voxel_ids` and :func:`heart_model_equation_parts` keep
  the reference's signatures and return numpy arrays (bit-identical);
* :func:`compile_instance` goes from voxel coordinates and per-voxel parameters
  to an engine instance whose tables never leave the device
  (``phs_instance_desc.device_tables``), with the same tables, order and
  scalars as :func:`pyheartsim_b200.instance.compile_instance` builds on the
  host from the reference's inputs.

torch provides the device buffers and the stream; the work is the library's.
"""
import ctypes

import numpy as np

from . import _lib
from .instance import CompiledInstance, instance_scalars, tblock_steps

_MS_KEYS = ("tau_open_voxel", "tau_close_voxel", "tau_in_voxel", "tau_out_voxel", "v_gate_voxel")
_AP_KEYS = ("k_voxel", "a_voxel", "epsilon_0_voxel", "mu1_voxel", "mu2_voxel")


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("geometry_gpu needs a CUDA device")
    return torch


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream(torch, stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def lattice_neighbors(ijk, order=True, stream=None):
    """Device neighbour table of integer lattice coordinates.

    ``ijk``: (n, 3) integer array or CUDA tensor.  Returns ``(nb18, order)`` as
    CUDA int32 tensors ((n, 18), -1 for absent, and the (z, y, x) row order, or
    None)."""
    torch = _torch()
    t = torch.as_tensor(ijk, device="cuda").to(torch.int32).contiguous()
    n = t.shape[0]
    if t.ndim != 2 or t.shape[1] != 3 or n == 0:
        raise ValueError("ijk must be (n, 3) with n > 0")
    nb18 = torch.empty((n, 18), dtype=torch.int32, device=t.device)
    od = torch.empty(n, dtype=torch.int32, device=t.device) if order else None
    _lib.check(_lib.lib().phs_lattice_neighbors(n, _ptr(t), _ptr(nb18), _ptr(od), _stream(torch, stream)),
               "phs_lattice_neighbors")
    return nb18, od


def find_neighbor_voxel_ids(voxel):
    """Drop-in of utility/voxelization.py:102-152: ``voxel`` in lattice units
    (the reference queries neighbours at offsets of 1 with a 0.1 tolerance), so
    coordinates are rounded to the nearest lattice point.  Returns (n, 18) int64."""
    v = np.asarray(voxel, dtype=np.float64)
    ijk = np.rint(v)
    if np.any(np.abs(v - ijk) >= 0.1):
        raise ValueError("voxel coordinates must lie within 0.1 of integer lattice points")
    nb18, _ = lattice_neighbors(ijk.astype(np.int32), order=False)
    return nb18.cpu().numpy().astype(np.int64)


def _par(simulation_parameters, parameter, n):
    keys = _MS_KEYS if simulation_parameters['heart_model_flag'] == 0 else _AP_KEYS
    cols = [np.broadcast_to(np.asarray(parameter[k], dtype=np.float64), (n,)) for k in keys]
    cols.append(np.broadcast_to(np.asarray(parameter['c_voxel'], dtype=np.float64), (n,)))
    return np.ascontiguousarray(np.stack(cols, axis=1))


def equation_parts(simulation_parameters, nb18, D0, parameter, stream=None):
    """P_2d (n, 21) float64 CUDA tensor from a device neighbour table."""
    torch = _torch()
    n = nb18.shape[0]
    par = torch.as_tensor(_par(simulation_parameters, parameter, n), device=nb18.device)
    d0 = None
    if D0 is not None:
        d0 = torch.as_tensor(np.ascontiguousarray(np.asarray(D0, dtype=np.float64).reshape(n, 9)),
                             device=nb18.device)
    P = torch.empty((n, 21), dtype=torch.float64, device=nb18.device)
    _lib.check(_lib.lib().phs_equation_parts(n, _ptr(nb18), _ptr(d0), _ptr(par), _ptr(P), _stream(torch, stream)),
               "phs_equation_parts")
    return P


def heart_model_equation_parts(simulation_parameters, n_voxel, D0, neighbor_id_2d, parameter):
    """Drop-in of simulation/equation_parts.py:36-114 on the device; returns
    numpy (n, 21), bit-identical to the reference.  ``D0`` may be a list of 3x3
    tensors (the reference's form), an (n, 3, 3) array or None (identity)."""
    torch = _torch()
    nb = torch.as_tensor(np.ascontiguousarray(np.asarray(neighbor_id_2d, dtype=np.int32)), device="cuda")
    if nb.shape != (n_voxel, 18):
        raise ValueError("neighbor_id_2d must be (n_voxel, 18)")
    if D0 is not None and not isinstance(D0, np.ndarray):
        D0 = np.stack([np.asarray(d, dtype=np.float64) for d in D0])
    return equation_parts(simulation_parameters, nb, D0, parameter).cpu().numpy()


class DeviceInstance(CompiledInstance):
    """An instance whose per-voxel tables live in CUDA tensors.  ``desc()``
    hands the device pointers to the engine (``device_tables = 1``); the
    tensors stay referenced by this object."""

    def desc(self):
        d = _lib.InstanceDesc()
        d.n_voxel = self.n_voxel
        d.model = self.model
        d.restart = self.restart
        d.nb6 = ctypes.cast(_ptr(self.nb6_t), ctypes.POINTER(ctypes.c_int32))
        iso = self.cw is not None
        d.coef6 = None if iso else ctypes.cast(_ptr(self.coef6_t), ctypes.POINTER(ctypes.c_double))
        d.cw = ctypes.cast(_ptr(self.cw_t), ctypes.POINTER(ctypes.c_double)) if iso else None
        d.mask6 = ctypes.cast(_ptr(self.mask6_t), ctypes.POINTER(ctypes.c_uint8)) if iso else None
        d.vflags = ctypes.cast(_ptr(self.vflags_t), ctypes.POINTER(ctypes.c_uint8))
        d.vparams = (ctypes.cast(_ptr(self.vparams_t), ctypes.POINTER(ctypes.c_double))
                     if self.vparams_t is not None else None)
        for i in range(5):
            d.params[i] = float(self.params[i])
        d.dt = self.dt
        d.j_stim = self.j_stim
        d.n_steps = self.n_steps
        d.stim = _lib.ptr(self.stim, ctypes.c_uint8)
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
        d.guess = int(self.guess)
        if self.nb_edge_t is not None:
            d.nb_edge = ctypes.cast(_ptr(self.nb_edge_t), ctypes.POINTER(ctypes.c_int32))
            d.coef_edge = ctypes.cast(_ptr(self.coef_edge_t), ctypes.POINTER(ctypes.c_double))
        d.device_tables = 1
        self._desc = d
        return d

    def release_tables(self):
        """Drop the device tables (after the engine has copied them)."""
        for k in ("nb6_t", "coef6_t", "cw_t", "mask6_t", "vflags_t", "vparams_t", "nb_edge_t", "coef_edge_t"):
            setattr(self, k, None)

    def host_tables(self):
        """The tables as numpy arrays (the names :class:`CompiledInstance` uses)."""
        g = lambda t: None if t is None else t.cpu().numpy()
        return dict(nb6=g(self.nb6_t), coef6=g(self.coef6_t), vflags=g(self.vflags_t), vparams=g(self.vparams_t),
                    cw=g(self.cw_t) if self.cw is not None else None,
                    mask6=g(self.mask6_t) if self.cw is not None else None,
                    nb_edge=g(self.nb_edge_t), coef_edge=g(self.coef_edge_t))


def compile_reference_inputs(n_voxel, P_2d, geometry_data, simulation_parameters, arrhythmia_parameters, *,
                             reorder=True, stream=None, **kw):
    """The drop-in's own inputs (``n_voxel``, ``P_2d`` (n, 21), ``geometry_data``
    with ``neighbor_id_2d`` (n, 18) and ``Delta``, optionally ``voxel`` (n, 3) in
    mm for the row order, and the two parameter dicts of
    simulation/simulation_gpu.py:261) -> a :class:`DeviceInstance` whose
    operator tables are compiled on the GPU from the uploaded P_2d and
    neighbour table.  Same tables, order and scalars as
    :func:`pyheartsim_b200.instance.compile_instance` (the host compiler)."""
    torch = _torch()
    n = int(n_voxel)
    dev = torch.device("cuda", torch.cuda.current_device())
    P = torch.as_tensor(np.ascontiguousarray(np.asarray(P_2d, dtype=np.float64)), device=dev)
    nb18 = torch.as_tensor(np.ascontiguousarray(np.asarray(geometry_data['neighbor_id_2d'], dtype=np.int32)),
                           device=dev)
    if P.shape != (n, 21) or nb18.shape != (n, 18):
        raise ValueError("P_2d must be (n_voxel, 21) and neighbor_id_2d (n_voxel, 18)")
    order = None
    vox = geometry_data.get('voxel') if hasattr(geometry_data, 'get') else None
    if reorder and vox is not None and np.shape(vox) == (n, 3):
        ijk = torch.round(torch.as_tensor(np.asarray(vox, dtype=np.float64), device=dev)
                          / float(geometry_data['Delta'])).to(torch.int32)
        _, order = lattice_neighbors(ijk, order=True, stream=stream)
    return _compile_tables(n, P, nb18, order, float(geometry_data['Delta']), simulation_parameters,
                           arrhythmia_parameters, stream, dev, **kw)


def compile_instance(voxel, Delta, parameter, D0, simulation_parameters, arrhythmia_parameters, *,
                     reorder=True, stream=None, **kw):
    """Voxel coordinates (n, 3) in mm and per-voxel parameters (the reference's
    ``parameter`` dict of P_2d columns 15..20) -> a :class:`DeviceInstance`,
    built on the GPU: neighbour table, P_2d, operator tables and row order.
    Keyword arguments as :func:`pyheartsim_b200.instance.compile_instance`
    (``full_cycles``, ``tol``, ``restart``, ``pacing_duration``, ...)."""
    torch = _torch()
    vox = np.asarray(voxel, dtype=np.float64)
    n = vox.shape[0]
    dev = torch.device("cuda", torch.cuda.current_device())
    ijk = torch.round(torch.as_tensor(vox, device=dev) / float(Delta)).to(torch.int32)
    nb18, order = lattice_neighbors(ijk, order=bool(reorder), stream=stream)
    P = equation_parts(simulation_parameters, nb18, D0, parameter, stream=stream)
    return _compile_tables(n, P, nb18, order, float(Delta), simulation_parameters, arrhythmia_parameters, stream,
                           dev, **kw)


def _compile_tables(n, P, nb18, order, Delta, simulation_parameters, arrhythmia_parameters, stream, dev, **kw):
    """Operator tables of an instance from device P_2d, neighbour table and row
    order (``phs_operator_flags``, ``phs_operator_tables``)."""
    torch = _torch()
    sc, s1, s2 = instance_scalars(simulation_parameters, arrhythmia_parameters, **kw)
    node_flag = np.asarray(arrhythmia_parameters['node_flag'])
    sc["tblock_steps"] = tblock_steps(sc["n_steps"], sc["dt"]) if np.any(node_flag == 3) else 0

    L = _lib.lib()
    st = _stream(torch, stream)
    fl = (ctypes.c_int32 * 3)()
    _lib.check(L.phs_operator_flags(n, _ptr(P), fl, st), "phs_operator_flags")
    face, edge, uniform = bool(fl[0]), bool(fl[1]), bool(fl[2])
    e = lambda shape, dt: torch.empty(shape, dtype=dt, device=dev)
    t = dict(inv=e(n, torch.int32), nb6=e((n, 6), torch.int32), coef6=e((n, 6), torch.float64),
             cw=e(n, torch.float64), mask6=e(n, torch.uint8), vflags=e(n, torch.uint8),
             vparams=None if uniform else e((n, 5), torch.float64),
             nb_edge=e((n, 12), torch.int32) if edge else None, coef_edge=e((n, 6), torch.float64) if edge else None)
    nf = torch.as_tensor(np.ascontiguousarray(node_flag, dtype=np.int32), device=dev)
    s1_t = torch.as_tensor(s1, device=dev) if s1.size else None
    s2_t = torch.as_tensor(s2, device=dev) if s2.size else None
    iso_word = e(1, torch.int32)
    a = _lib.OperatorTablesArgs()
    a.n_voxel = n
    a.Delta = float(Delta)
    a.P, a.nb18, a.node_flag, a.order = _ptr(P), _ptr(nb18), _ptr(nf), _ptr(order)
    for k in ("inv", "nb6", "coef6", "cw", "mask6", "vflags", "vparams", "nb_edge", "coef_edge"):
        setattr(a, k, _ptr(t[k]))
    a.s1, a.n_s1 = _ptr(s1_t), int(s1.size)
    a.s2, a.n_s2 = _ptr(s2_t), int(s2.size)
    a.iso_word = _ptr(iso_word)
    a.face_cross, a.edge = int(face), int(edge)
    a.stream = st
    _lib.check(L.phs_operator_tables(ctypes.byref(a)), "phs_operator_tables")
    iso = bool(a.iso)
    params = P[0, 15:20].cpu().numpy().copy()
    od = order.cpu().numpy().astype(np.int64) if order is not None else None
    if od is not None and np.array_equal(od, np.arange(n)):
        od = None
    inv = t["inv"].cpu().numpy().astype(np.int64) if od is not None else None
    inst = DeviceInstance(
        n_voxel=n, params=params, Delta=float(Delta), order=od, inv=inv, **sc,
        nb6_t=t["nb6"], coef6_t=t["coef6"], cw_t=t["cw"], mask6_t=t["mask6"], vflags_t=t["vflags"],
        vparams_t=t["vparams"], nb_edge_t=t["nb_edge"], coef_edge_t=t["coef_edge"],
        # presence markers read by the byte model and the serving footprint
        cw=True if iso else None, coef_edge=True if edge else None, vparams=None if uniform else True)
    return inst
