"""Accuracy of the FP32 early-exit path against the plain FP64 path.

The plain FP64 path is the reference's scheme (GMRES(50) full cycles, FP64
state; within 1e-9 of the FP64 oracle on every tested case), so it serves as
the reference here.  Both runs keep a Vm history sampled every step on the
device (``sample_stride`` 1), from which ``phs_activation_times`` extracts
every upward crossing of Vm = 0.5 per voxel: the first is the activation time
(LAT) and the later ones are re-activations (re-entry, rotors), all in units
of dt.  The 1 kHz history (every ``stride``-th step) is also returned for the
electrograms.
"""
import time

import numpy as np

from . import _lib
from . import instance as _instance
from .engine import BatchedEngine

MAX_ACTIVATIONS = 32


def run_with_activations(case, pacing_duration, fast, tol=1e-7, max_activations=MAX_ACTIVATIONS):
    """Run one instance to its end with a per-step device history.

    ``case`` is the reference's (n_voxel, P_2d, geometry_data,
    simulation_parameters, arrhythmia_parameters).  ``fast``: FP32 state with
    the Givens early exit at ``tol`` from the extrapolated guess (restart 20);
    else the plain FP64 path (GMRES(50) full cycles).  Returns a dict with the
    activation samples ``times`` (n, max_activations; -1 past ``counts``),
    ``counts``, the 1 kHz history ``u_1khz`` (S, n) in the caller's order, the
    final state and the wall time."""
    n, P, geom, sp, ap = case
    kw = dict(full_cycles=not fast, tol=tol if fast else 1e-5, atol=1e-5, restart=20 if fast else 50,
              pacing_duration=pacing_duration)
    inst = _instance.compile_instance(n, P, geom, dict(sp), dict(ap), **kw)
    stride, S = inst.sample_stride, inst.n_samples
    inst.sample_stride, inst.n_samples = 1, int(inst.n_steps)
    eng = BatchedEngine(_lib.PREC_F32 if fast else _lib.PREC_F64)
    try:
        slot = eng.add(inst)
        t0 = time.perf_counter()
        while not eng.finished(slot):
            eng.advance(5000)
        wall = time.perf_counter() - t0
        info = eng.info(slot)
        times, counts = eng.activation_times(slot, max_activations)
        # the reference's 1 kHz samples: steps 0, stride, 2 stride, ...
        idx = np.arange(0, int(inst.n_steps), max(stride, 1))[:S]
        u = np.stack([eng.history(slot, int(k), 1)[0] for k in idx])
    finally:
        eng.close()
    return {"times": times, "counts": counts, "u_1khz": u, "wall_s": wall, "steps": int(info["step"]),
            "status": int(info["status"]), "arnoldi_per_step": info["arnoldi_steps"] / max(info["step"], 1),
            "n": int(n)}


def compare_activations(ref, test, max_activations=MAX_ACTIVATIONS):
    """Activation-time errors of ``test`` against ``ref`` (outputs of
    :func:`run_with_activations`), in steps (units of dt).

    Returns the first-activation error (max over voxels activated in both runs,
    and the count activated in only one), and per re-activation index i the
    voxels with at least i+1 activations in both, their max |dLAT|, and the
    voxels with i+1 activations in one run only.  ``nearest_*`` pair each
    reference activation with the test run's nearest crossing of the same
    voxel instead of the one with the same count."""
    cr, ct = ref["counts"], test["counts"]
    tr, tt = ref["times"].astype(np.int64), test["times"].astype(np.int64)
    out = {"voxels": int(cr.size), "activation_count_equal_frac": float(np.mean(cr == ct)),
           "max_activations_ref": int(cr.max()), "max_activations_test": int(ct.max())}
    per = []
    valid_t = tt >= 0
    for i in range(min(max_activations, int(max(cr.max(), ct.max())))):
        both = (cr > i) & (ct > i)
        one = int(((cr > i) != (ct > i)).sum())
        d = np.abs(tr[both, i] - tt[both, i])
        # the same activation found by time instead of by count: the test
        # run's nearest crossing of that voxel (an extra or missing crossing
        # elsewhere in the sequence does not shift the pairing)
        has = cr > i
        near = np.where(valid_t[has], np.abs(tt[has] - tr[has, i][:, None]), np.iinfo(np.int64).max).min(axis=1)
        near = near[near < np.iinfo(np.int64).max]
        per.append({"index": i, "voxels_both": int(both.sum()), "voxels_one_run_only": one,
                    "max_dlat_steps": int(d.max()) if d.size else None,
                    "p99_dlat_steps": float(np.percentile(d, 99)) if d.size else None,
                    "frac_within_1_step": float(np.mean(d <= 1)) if d.size else None,
                    "nearest_max_dlat_steps": int(near.max()) if near.size else None,
                    "nearest_p99_dlat_steps": float(np.percentile(near, 99)) if near.size else None,
                    "nearest_frac_within_1_step": float(np.mean(near <= 1)) if near.size else None})
    out["first"] = per[0] if per else None
    out["reactivations"] = per[1:]
    return out


def electrogram_errors(ref_u, test_u, electrodes, geom, c_voxel):
    """Electrogram relative L2 errors against the FP64 electrogram of the
    reference history: the FP32 history through the FP64 contraction and
    through BF16x3, and the reference history through BF16x3 (the
    contraction's own error)."""
    from .simulation import unipolar_electrogram_gpu as egm
    args = (geom['voxel'], None, c_voxel)
    tail = (geom['Delta'], geom['neighbor_id_2d'])
    e_ref = egm.compute(electrodes, *args, ref_u, *tail)
    rel = lambda a: float(np.linalg.norm(a - e_ref) / np.linalg.norm(e_ref))
    return {"electrodes": int(electrodes.shape[0]), "samples": int(ref_u.shape[0]),
            "fp32_history_fp64_egm": rel(egm.compute(electrodes, *args, test_u.astype(np.float64), *tail)),
            "fp32_history_bf16x3_egm": rel(egm.compute(electrodes, *args, test_u.astype(np.float64), *tail,
                                                       mode="bf16x3")),
            "fp64_history_bf16x3_egm": rel(egm.compute(electrodes, *args, ref_u, *tail, mode="bf16x3"))}


def compare_case(case, pacing_duration, electrodes=None, tol=1e-7):
    """Plain FP64 vs FP32 early exit on one configuration: activation errors,
    max |dVm| over the 1 kHz samples, electrogram errors, wall times."""
    ref = run_with_activations(case, pacing_duration, fast=False)
    test = run_with_activations(case, pacing_duration, fast=True, tol=tol)
    out = compare_activations(ref, test)
    out["max_abs_dvm_1khz"] = float(np.abs(ref["u_1khz"] - test["u_1khz"].astype(np.float64)).max())
    out["plain_fp64_s"] = ref["wall_s"]
    out["fast_fp32_s"] = test["wall_s"]
    out["steps"] = ref["steps"]
    out["arnoldi_per_step_fast"] = test["arnoldi_per_step"]
    out["status"] = [ref["status"], test["status"]]
    if electrodes is not None:
        out["electrogram"] = electrogram_errors(ref["u_1khz"], test["u_1khz"], electrodes, case[2], case[1][:, 20])
    return out
