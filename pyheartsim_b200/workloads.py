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


def shell_case(i, n_target, seed, t_phys=500.0, scar_max=0.3, fast=True, tol=1e-5, restart=20,
               save_h=False, pacing_ms=2.0, fibres=False):
    """Reference-style inputs + the compiled instance of shell ``i`` (``fibres``:
    rule-based fibre field, anisotropic D0)."""
    rng = np.random.default_rng(seed * 1000 + i)
    ijk = _shell_scaled(n_target, seed * 1000 + i)
    nb = lattice_neighbors(ijk)
    cov = float(rng.uniform(0.0, scar_max))
    c_scale = synthetic.scar(ijk, nb, cov, rng)
    healthy = np.where(c_scale == 1.0)[0]
    centre = ijk[healthy[int(rng.integers(0, healthy.size))]]
    s1 = np.where(np.sum((ijk - centre) ** 2, axis=1) <= 9)[0]
    model = i % 2
    dt_phys = 0.05 if model == 0 else 0.02
    D0 = synthetic.fibre_tensors(ijk) if fibres else None
    n, P, geom, sp, ap = synthetic.make_case(ijk, 0.4, model, dt_phys, t_phys, s1, flag=4, c_scale=c_scale, D0=D0)
    inst = _instance.compile_instance(n, P, geom, sp, ap, full_cycles=not fast, tol=tol, atol=1e-5,
                                      restart=restart if fast else 50, pacing_duration=pacing_ms / sp['time_scale'],
                                      save_h=save_h)
    return inst, (n, P, geom, sp, ap), {"index": i, "n": n, "model": model, "scar": cov,
                                        "pacing_ms": pacing_ms, "fibres": bool(fibres)}


def shell_case_device(i, n_target, seed, t_phys=500.0, scar_max=0.3, tol=1e-5, restart=20, save_h=False,
                      pacing_ms=2.0, fibres=False, stream=None):
    """The instance of :func:`shell_case` (same geometry, scar, pacing site and
    tables), built on the GPU: the neighbour table, P_2d and the operator
    tables come from the device geometry path; only the face neighbours the
    scar generator needs come back to the host."""
    from . import geometry_gpu
    rng = np.random.default_rng(seed * 1000 + i)
    ijk = _shell_scaled(n_target, seed * 1000 + i)
    nb18, _ = geometry_gpu.lattice_neighbors(ijk, order=False, stream=stream)
    nb6 = nb18[:, :6].cpu().numpy()
    cov = float(rng.uniform(0.0, scar_max))
    c_scale = synthetic.scar(ijk, nb6, cov, rng)
    healthy = np.where(c_scale == 1.0)[0]
    centre = ijk[healthy[int(rng.integers(0, healthy.size))]]
    s1 = np.where(np.sum((ijk - centre) ** 2, axis=1) <= 9)[0]
    model = i % 2
    dt_phys = 0.05 if model == 0 else 0.02
    n = ijk.shape[0]
    sp, ap, par = synthetic.case_parameters(n, model, dt_phys, t_phys, s1, flag=4, c_scale=c_scale)
    D0 = synthetic.fibre_tensors(ijk) if fibres else None
    inst = geometry_gpu.compile_instance(ijk * 0.4, 0.4, par, D0, sp, ap, full_cycles=False, tol=tol, atol=1e-5,
                                         restart=restart, pacing_duration=pacing_ms / sp['time_scale'],
                                         save_h=save_h, stream=stream)
    return inst, {"index": i, "n": n, "model": model, "scar": cov, "pacing_ms": pacing_ms, "fibres": bool(fibres)}


def _build_one(args):
    i, n_target, seed, kw = args
    inst, _, meta = shell_case(i, n_target, seed, **kw)
    return inst, meta


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
