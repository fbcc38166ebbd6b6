"""Stimulus schedule of the reference, compiled once per run.

The reference evaluates ``apply_pacing`` on the host before every step and
uploads a full J vector (simulation/simulation_gpu.py:373-377).  The windows
only depend on the step index, so they are evaluated here for all steps at
once -- with the reference's own FP64 expressions and inclusive bounds
(simulation/pacing.py:136-170) -- into one byte per step (bit 0: S1 window
open, bit 1: S2 window open).  The device combines that byte with a per-voxel
membership byte, so no stimulus vector crosses PCIe during a run.
"""
import numpy as np

S1_ON = 1
S2_ON = 2


def assign_pacing_parameters(arrhythmia_parameters, arrhythmia_flag, simulation_parameters,
                             pacing_duration=None):
    """(s1_ids, s2_ids, s1_t, J_magnitude, pacing_duration, s2_t) as in
    simulation/pacing.py:102-134.  ``pacing_duration`` overrides the
    reference's hard-coded 5 ms (5/time_scale for Aliev-Panfilov)."""
    s1 = arrhythmia_parameters['s1_pacing_voxel_id']
    s1_t = arrhythmia_parameters['s1_t']
    s2_t = s1_t + arrhythmia_parameters['s1_s2_delta_t']
    s2 = []
    if arrhythmia_flag in (1, 2, 3, 4, 5, 6):
        s2 = arrhythmia_parameters['s2_pacing_voxel_id']
    if pacing_duration is None:
        if simulation_parameters['heart_model_flag'] == 0:
            pacing_duration = 5
        else:
            pacing_duration = 5 / simulation_parameters['time_scale']
    return s1, s2, s1_t, 1, pacing_duration, s2_t


def _window(t, t0, dur):
    return (t >= t0) & (t <= t0 + dur)


def schedule(n_steps, dt, arrhythmia_parameters, simulation_parameters, arrhythmia_flag,
             s1_t, pacing_duration, s2_t):
    """uint8[n_steps]: bit 0 = S1 paced at model_time = step*dt, bit 1 = S2.

    Same branch structure as simulation/pacing.py:136-170, including the
    ``elif`` that ties flags 1-4 to the flag-6 test and the repeated
    subtraction of the cycle length for flag 0 (evaluated elementwise, so each
    step sees exactly the reference's sequence of FP64 operations).
    """
    t = np.arange(n_steps, dtype=np.float64) * dt
    s1 = np.zeros(n_steps, dtype=bool)
    s2 = np.zeros(n_steps, dtype=bool)
    ts = simulation_parameters['time_scale']
    if arrhythmia_flag == 0:
        start = arrhythmia_parameters['pacing_start_time']
        cyc = arrhythmia_parameters['pacing_cycle_length']
        tt = t.copy()
        while True:
            m = (tt - start) > cyc
            if not m.any():
                break
            if not cyc > 0:
                raise ValueError("pacing_cycle_length must be > 0 for arrhythmia_flag 0 "
                                 "(the reference loops forever here)")
            tt[m] = tt[m] - cyc
        s1 |= _window(tt, start, pacing_duration)
    if arrhythmia_flag == 5:
        f1, f2 = 0 / ts, 300 / ts
        s1 |= _window(t, f1, pacing_duration)
        s2 |= _window(t, f2, pacing_duration)
    if arrhythmia_flag == 6:
        f1, f2 = 0 / ts, 50 / ts
        s1 |= _window(t, f1, pacing_duration)
        s2 |= _window(t, f2, pacing_duration)
    elif arrhythmia_flag in (1, 2, 3, 4):
        s1 |= _window(t, s1_t, pacing_duration)
    if arrhythmia_flag in (1, 2, 3):
        s2 |= _window(t, s2_t, pacing_duration)
    return (s1.astype(np.uint8) * S1_ON) | (s2.astype(np.uint8) * S2_ON)
