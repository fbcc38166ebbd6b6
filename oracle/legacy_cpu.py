"""CPU baseline: port of the reference's legacy CPU time stepper.

TEST/BENCH INFRASTRUCTURE ONLY -- imported by ``bench.py``'s CPU-baseline leg
and its ``--impl reference`` arm (and tests), never by the product package.

Restates legacy/compute_simulation_cpu.py (jiyuehe/PyHeartSim), whose own
``execute()`` cannot run as shipped (it imports a missing ``modules.pacing`` and
unpacks 12 values from a 7-value function):

* ``reaction_step_rk4``   legacy/compute_simulation_cpu.py:144-209 -- Numba
                          ``njit(parallel=True)``, nine ``prange`` passes, FP64
* ``cn_step``             legacy/compute_simulation_cpu.py:113-142 -- rebuilds
                          A = I - dt/2 L every step, b = u* + dt/2 L u*, SciPy
                          BiCGSTAB with atol 1e-6, maxiter 1000
* the step loop           legacy/compute_simulation_cpu.py:271-305 with the
                          pacing of simulation/pacing.py:136-170
The Laplacian is the reference's (simulation_fp64.laplacian).
"""
import os

import numpy as np
import scipy.sparse as sp
from scipy.sparse.linalg import bicgstab

from . import simulation_fp64

try:
    from numba import njit, prange
    HAVE_NUMBA = True
except Exception:  # pragma: no cover - numba is part of the image
    HAVE_NUMBA = False


if HAVE_NUMBA:
    @njit(cache=True)
    def _reaction_one(model, u, h, P, J, n):
        if model == 0:
            du = (h[n] * (u[n] ** 2) * (1 - u[n])) / P[n, 17] - u[n] / P[n, 18] + J[n]
            if u[n] < P[n, 19]:
                dh = (1 - h[n]) / P[n, 15]
            else:
                dh = -h[n] / P[n, 16]
        else:
            du = -P[n, 15] * u[n] * (u[n] - P[n, 16]) * (u[n] - 1) - u[n] * h[n] + J[n]
            dh = (P[n, 17] + P[n, 18] * h[n] / (u[n] + P[n, 19])) * (-h[n] - P[n, 15] * u[n] * (u[n] - P[n, 16] - 1))
        return du, dh

    @njit(parallel=True, cache=True)
    def reaction_step_rk4(model, u0, h0, P, J, dt):
        n = u0.shape[0]
        un = np.empty_like(u0)
        hn = np.empty_like(h0)
        k1u = np.zeros(n); k1h = np.zeros(n); k2u = np.zeros(n); k2h = np.zeros(n)
        k3u = np.zeros(n); k3h = np.zeros(n); k4u = np.zeros(n); k4h = np.zeros(n)
        ut = np.empty_like(u0)
        ht = np.empty_like(h0)
        for i in prange(n):
            k1u[i], k1h[i] = _reaction_one(model, u0, h0, P, J, i)
        for i in prange(n):
            ut[i] = u0[i] + 0.5 * dt * k1u[i]
            ht[i] = h0[i] + 0.5 * dt * k1h[i]
        for i in prange(n):
            k2u[i], k2h[i] = _reaction_one(model, ut, ht, P, J, i)
        for i in prange(n):
            ut[i] = u0[i] + 0.5 * dt * k2u[i]
            ht[i] = h0[i] + 0.5 * dt * k2h[i]
        for i in prange(n):
            k3u[i], k3h[i] = _reaction_one(model, ut, ht, P, J, i)
        for i in prange(n):
            ut[i] = u0[i] + dt * k3u[i]
            ht[i] = h0[i] + dt * k3h[i]
        for i in prange(n):
            k4u[i], k4h[i] = _reaction_one(model, ut, ht, P, J, i)
        for i in prange(n):
            un[i] = u0[i] + (dt / 6.0) * (k1u[i] + 2 * k2u[i] + 2 * k3u[i] + k4u[i])
            hn[i] = h0[i] + (dt / 6.0) * (k1h[i] + 2 * k2h[i] + 2 * k3h[i] + k4h[i])
        return un, hn
else:  # pragma: no cover
    def reaction_step_rk4(model, u0, h0, P, J, dt):
        return simulation_fp64.rk4(model, u0, h0, P, J, dt)


def cn_step(u_star, L, dt, tol=1e-6):
    """legacy/compute_simulation_cpu.py:113-142."""
    n = u_star.shape[0]
    I = sp.identity(n, format='csr')
    A = I - (dt / 2.0) * L
    b = u_star + (dt / 2.0) * (L @ u_star)
    u_next, info = bicgstab(A, b, x0=u_star, atol=tol, maxiter=1000)
    return u_next


class LegacyRun:
    """The legacy CPU stepper on one instance (reference argument dicts)."""

    def __init__(self, n_voxel, P_2d, geometry_data, simulation_parameters, arrhythmia_parameters,
                 pacing_duration=None):
        self.n = n_voxel
        self.P = np.ascontiguousarray(np.asarray(P_2d, dtype=np.float64))
        nf = np.asarray(arrhythmia_parameters['node_flag'])
        Pp = self.P.copy()
        Pp[nf == 4, 20] = 0.0
        self.L = simulation_fp64.laplacian(Pp, geometry_data['neighbor_id_2d'], geometry_data['Delta'])
        self.sp = simulation_parameters
        self.ap = arrhythmia_parameters
        self.model = int(simulation_parameters['heart_model_flag'])
        self.dt = simulation_parameters['dt']
        self.flag = simulation_parameters['arrhythmia_flag']
        _, s1, s2, self.s1_t, self.jmag, self.pdur, self.s2_t = simulation_fp64.assign_pacing_parameters(
            arrhythmia_parameters, self.flag, n_voxel, simulation_parameters, pacing_duration)
        self.s1 = np.atleast_1d(np.asarray(s1, dtype=np.int64))
        self.s2 = np.atleast_1d(np.asarray(s2, dtype=np.int64)) if np.size(s2) else np.zeros(0, np.int64)
        self.u = np.zeros(n_voxel)
        self.h = np.ones(n_voxel) if self.model == 0 else np.zeros(n_voxel)
        self.step_index = 0

    def step(self):
        mt = self.step_index * self.dt
        a, b = simulation_fp64.pacing_windows(self.ap, self.sp, self.flag, mt, self.s1_t, self.pdur, self.s2_t)
        J = np.zeros(self.n)
        if a:
            J[self.s1] = self.jmag
        if b:
            J[self.s2] = self.jmag
        us, self.h = reaction_step_rk4(self.model, self.u, self.h, self.P, J, self.dt)
        self.u = cn_step(us, self.L, self.dt)
        self.step_index += 1


def threads():
    try:
        import numba
        return int(numba.get_num_threads())
    except Exception:  # pragma: no cover
        return os.cpu_count() or 1
