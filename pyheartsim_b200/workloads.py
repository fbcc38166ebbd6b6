"""Seeded workloads of the benchmark configurations, as compiled instances.

``batched_shells`` is the batched configuration: ``count`` ellipsoidal shells
(Delta 0.4 mm, wall 3 voxels, vein holes) with voxel counts log-uniform in
[n_min, n_max], Gaussian-blob scar (coverage ~U(0, 0.3): c = 0 inside, 0.1 on
the border ring), one focal pacing site each (a ball of radius 3 voxels around
a random healthy voxel), even instances Mitchell-Schaeffer (dt 0.05 ms), odd
instances Aliev-Panfilov (dt 0.02 ms physical = 0.02/6 model), 500 ms each.
Instances are generated in a process pool (spawn) so the host work does not
dominate start-up.
"""
import multiprocessing as mp
import os
from concurrent.futures import ProcessPoolExecutor

import numpy as np

from . import instance as _instance
from . import synthetic
from .geometry import lattice_neighbors

_BASE_COUNT = {}


def _shell_scaled(n_target, seed, Delta=0.4, wall=3):
    base = (25.0, 20.0, 18.0)
    if (Delta, wall) not in _BASE_COUNT:
        _BASE_COUNT[(Delta, wall)] = synthetic.shell(base, Delta, wall, 4, 5.0, 0).shape[0]
    s = float(np.sqrt(n_target / _BASE_COUNT[(Delta, wall)]))
    return synthetic.shell(tuple(np.asarray(base) * s), Delta, wall, 4, 5.0 * s, seed)


# Focal stimulus of the batched shells, per model: (ball radius in voxels,
# duration in physical ms).  Mitchell-Schaeffer (c = 1) fires from a 3-voxel
# ball and 2 ms; Aliev-Panfilov with the reference's diffusion (c = 1.6 x 6 in
# model units) drains a small stimulated region before it reaches threshold --
# balls of 3 and 5 voxels at 2 or 5 ms stay below u = 2e-4 -- so its focal site
# is an 8-voxel ball held for the reference's 5 ms (which fires and propagates).
FOCAL = {0: (3, 2.0), 1: (8, 5.0)}


def _focal(ijk, c_scale, rng, model):
    healthy = np.where(c_scale == 1.0)[0]
    centre = ijk[healthy[int(rng.integers(0, healthy.size))]]
    r = FOCAL[model][0]
    return np.where(np.sum((ijk - centre) ** 2, axis=1) <= r * r)[0]


def shell_inputs(i, n_target, seed, t_phys=500.0, scar_max=0.3, pacing_ms=None, fibres=False):
    """Reference-style inputs of shell ``i``: ((n_voxel, P_2d, geometry_data,
    simulation_parameters, arrhythmia_parameters), meta); ``fibres``:
    rule-based fibre field, anisotropic D0.  ``pacing_ms``: stimulus duration
    (physical ms; default per model, :data:`FOCAL`)."""
    rng = np.random.default_rng(seed * 1000 + i)
    ijk = _shell_scaled(n_target, seed * 1000 + i)
    nb = lattice_neighbors(ijk)
    cov = float(rng.uniform(0.0, scar_max))
    c_scale = synthetic.scar(ijk, nb, cov, rng)
    model = i % 2
    s1 = _focal(ijk, c_scale, rng, model)
    pacing_ms = FOCAL[model][1] if pacing_ms is None else pacing_ms
    dt_phys = 0.05 if model == 0 else 0.02
    D0 = synthetic.fibre_tensors(ijk) if fibres else None
    n, P, geom, sp, ap = synthetic.make_case(ijk, 0.4, model, dt_phys, t_phys, s1, flag=4, c_scale=c_scale, D0=D0)
    return (n, P, geom, sp, ap), {"index": i, "n": n, "model": model, "scar": cov, "pacing_ms": pacing_ms,
                                  "fibres": bool(fibres)}


def shell_case(i, n_target, seed, t_phys=500.0, scar_max=0.3, fast=True, tol=1e-5, restart=20,
               save_h=False, pacing_ms=None, fibres=False):
    """Reference-style inputs + the compiled instance of shell ``i`` (``fibres``:
    rule-based fibre field, anisotropic D0)."""
    (n, P, geom, sp, ap), meta = shell_inputs(i, n_target, seed, t_phys, scar_max, pacing_ms, fibres)
    inst = _instance.compile_instance(n, P, geom, sp, ap, full_cycles=not fast, tol=tol, atol=1e-5,
                                      restart=restart if fast else 50,
                                      pacing_duration=meta["pacing_ms"] / sp['time_scale'], save_h=save_h)
    return inst, (n, P, geom, sp, ap), meta


def shell_payload(i, n_target, seed, t_phys=500.0, scar_max=0.3, pacing_ms=None):
    """What a request for shell ``i`` carries, before any table is built: the
    voxel coordinates (mm), the reference's per-voxel parameter dict (scar in
    ``c_voxel``), the two parameter dicts and the pacing duration -- the same
    geometry, scar and pacing site as :func:`shell_inputs`, made without a
    neighbour table (the scar ring comes from a dense occupancy grid)."""
    rng = np.random.default_rng(seed * 1000 + i)
    ijk = _shell_scaled(n_target, seed * 1000 + i)
    cov = float(rng.uniform(0.0, scar_max))
    c_scale = synthetic.scar(ijk, None, cov, rng)
    model = i % 2
    s1 = _focal(ijk, c_scale, rng, model)
    pacing_ms = FOCAL[model][1] if pacing_ms is None else pacing_ms
    dt_phys = 0.05 if model == 0 else 0.02
    n = ijk.shape[0]
    sp, ap, par = synthetic.case_parameters(n, model, dt_phys, t_phys, s1, flag=4, c_scale=c_scale)
    return {"voxel": ijk * 0.4, "parameter": par, "sp": sp, "ap": ap, "pacing_ms": pacing_ms,
            "meta": {"index": i, "n": n, "model": model, "scar": cov, "pacing_ms": pacing_ms, "fibres": False}}


def compile_payload(payload, tol=1e-5, restart=20, save_h=False, stream=None, D0=None):
    """Device instance of a :func:`shell_payload` (neighbour table, P_2d and
    operator tables built on the GPU)."""
    from . import geometry_gpu
    sp = payload["sp"]
    return geometry_gpu.compile_instance(payload["voxel"], 0.4, payload["parameter"], D0, sp, payload["ap"],
                                         full_cycles=False, tol=tol, atol=1e-5, restart=restart,
                                         pacing_duration=payload["pacing_ms"] / sp['time_scale'], save_h=save_h,
                                         stream=stream)


def shell_case_device(i, n_target, seed, t_phys=500.0, scar_max=0.3, tol=1e-5, restart=20, save_h=False,
                      pacing_ms=None, fibres=False, stream=None):
    """The instance of :func:`shell_case` (same geometry, scar, pacing site and
    tables), built on the GPU: the neighbour table, P_2d and the operator
    tables come from the device geometry path."""
    pl = shell_payload(i, n_target, seed, t_phys, scar_max, pacing_ms)
    D0 = synthetic.fibre_tensors(np.rint(pl["voxel"] / 0.4).astype(np.int64)) if fibres else None
    inst = compile_payload(pl, tol=tol, restart=restart, save_h=save_h, stream=stream, D0=D0)
    meta = dict(pl["meta"], fibres=bool(fibres))
    return inst, meta


def _build_one(args):
    i, n_target, seed, kw = args
    inst, _, meta = shell_case(i, n_target, seed, **kw)
    return inst, meta


def _inputs_one(args):
    i, n_target, seed, kw = args
    return shell_inputs(i, n_target, seed, **kw)


def batched_inputs(count=64, n_min=50_000, n_max=400_000, seed=0, workers=None, **kw):
    """List of (reference-style inputs, meta) of the batched configuration,
    uncompiled (for the drop-in's end-to-end path)."""
    sizes = batch_sizes(count, n_min, n_max, seed)
    jobs = [(i, int(sizes[i]), seed, kw) for i in range(count)]
    workers = workers or min(count, max(1, (os.cpu_count() or 2) - 1), 32)
    if workers <= 1 or count <= 1:
        return [_inputs_one(j) for j in jobs]
    ctx = mp.get_context("spawn")
    with ProcessPoolExecutor(max_workers=workers, mp_context=ctx) as ex:
        return list(ex.map(_inputs_one, jobs))


def batch_sizes(count, n_min, n_max, seed):
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(n_min), np.log(n_max), size=count)).astype(np.int64)


def batched_shells(count=64, n_min=50_000, n_max=400_000, seed=0, workers=None, **kw):
    """List of (CompiledInstance, meta) for the batched configuration."""
    sizes = batch_sizes(count, n_min, n_max, seed)
    jobs = [(i, int(sizes[i]), seed, kw) for i in range(count)]
    workers = workers or min(count, max(1, (os.cpu_count() or 2) - 1), 32)
    if workers <= 1 or count <= 1:
        return [_build_one(j) for j in jobs]
    ctx = mp.get_context("spawn")
    with ProcessPoolExecutor(max_workers=workers, mp_context=ctx) as ex:
        return list(ex.map(_build_one, jobs))


# ----------------------------------------------------------------- named accuracy configurations

def sheet_c1(nx=200, ny=200, t_phys=500.0):
    """The plain FP64 sheet: nx x ny voxels (Delta 0.4 mm, c = 1, isotropic),
    Mitchell-Schaeffer (tau_in 0.3, tau_out 6, tau_open 120, tau_close 150,
    v_gate 0.13), dt 0.05 ms, a 5 x 5 corner stimulus at t = 0 lasting 1 ms
    (arrhythmia_flag 4), ``t_phys`` ms (10,000 steps at 500 ms), and 16
    electrodes on a 4 x 4 grid 1 mm above the sheet.
    Returns ((n, P_2d, geometry_data, simulation_parameters,
    arrhythmia_parameters), pacing_ms, electrode_xyz)."""
    ijk = synthetic.sheet(nx, ny)
    s1 = np.where((ijk[:, 0] < 5) & (ijk[:, 1] < 5))[0]
    case = synthetic.make_case(ijk, 0.4, 0, 0.05, t_phys, s1, flag=4)
    return case, 1.0, synthetic.electrodes_grid(nx, ny, 0.4)


# Pacing of the rotor shell per wall thickness: (S1 depth in mm, S1-S2 coupling
# interval in physical ms).  Chosen by sweeps of the FP32 engine: the S1 cap
# must fire on its own (1.2 mm fires through a 3-voxel wall but not through an
# 8-voxel one, which drains it; 2.4 mm fires), and S2 must land on the S1 wave's
# refractory tail.  Wall 3 with a 1.2 mm cap sustains re-entry to the end of
# the 1000 ms run (up to 6 activations per voxel) for S1-S2 of 220-240 ms and
# not from 250 ms; wall 8 with a 2.4 mm cap for 220 ms only (200 ms: S2 does not
# take; 240-300 ms: one extra wave that dies by 425 ms).
C2_PACING = {3: (1.2, 240.0), 8: (2.4, 220.0)}


def atrium_c2(wall=3, seed=0, t_phys=1000.0, s1_s2=None, n_electrodes=64, s1_mm=None):
    """The rotor shell: ellipsoidal shell with semi-axes 25/20/18 mm (Delta 0.4
    mm, ``wall`` voxels thick: 91,292 voxels at wall 3, 218,403 at wall 8) with
    four r = 5 mm vein holes along seeded radial directions; Aliev-Panfilov
    (k 8, a 0.15, eps0 0.002, mu1 0.2, mu2 0.3) with the reference's time
    scaling (time_scale 6, c = 1.6 x 6, configuration.py:141-157); dt 0.02 ms
    physical (0.02/6 model), ``t_phys`` ms (50,000 steps at 1000 ms).  S1: the
    cap of voxels within ``s1_mm`` of the lowest x, at t = 0; S2: the quadrant
    x < 0, y > 0 (the shell is centred on the origin) ``s1_s2`` ms later
    (arrhythmia_flag 1, the reference's 5 ms stimuli); defaults per wall from
    :data:`C2_PACING`; 64 electrodes 2 mm off the surface at seeded voxels.
    Returns ((n, P_2d, geometry_data, simulation_parameters,
    arrhythmia_parameters), pacing_ms (None: the reference's default),
    electrode_xyz)."""
    d_mm, d_s12 = C2_PACING.get(wall, C2_PACING[3])
    s1_s2 = d_s12 if s1_s2 is None else s1_s2
    s1_mm = d_mm if s1_mm is None else s1_mm
    ijk = synthetic.shell((25.0, 20.0, 18.0), 0.4, wall, 4, 5.0, seed)
    layers = int(round(s1_mm / 0.4))
    s1 = np.where(ijk[:, 0] < ijk[:, 0].min() + layers)[0]
    s2 = np.where((ijk[:, 0] < 0) & (ijk[:, 1] > 0))[0]
    case = synthetic.make_case(ijk, 0.4, 1, 0.02, t_phys, s1, s2_ids=s2, flag=1, s1_t=0.0, s1_s2=float(s1_s2))
    rng = np.random.default_rng(seed + 64)
    return case, None, synthetic.electrodes_off_surface(ijk, 0.4, n_electrodes, rng, offset=2.0)
