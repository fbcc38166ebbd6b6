"""FP64 CPU oracle of PyHeartSim's time-stepping path.

TEST INFRASTRUCTURE ONLY.  Imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` -- as the checker, never as the thing
measured or shipped.  The product package ``pyheartsim_b200`` never imports it.

A plain NumPy/SciPy restatement, in FP64, of the reference's
``simulation/simulation_gpu.py::compute`` (jiyuehe/PyHeartSim):

* P_2d assembly             simulation/equation_parts.py:36-114 (vectorised)
* diffusion matrix L        simulation/simulation_gpu.py:138-225 (COO -> CSR,
                            explicit zeros at column 0 for absent neighbours)
* pacing schedule           simulation/pacing.py:102-170
* RK4 reaction              simulation/simulation_gpu.py:27-43, 71-130
* CN step + GMRES(50)       simulation/simulation_gpu.py:227-259 with CuPy's
                            documented full-cycle GMRES semantics
* driver loop               simulation/simulation_gpu.py:261-409 (step count,
                            1 kHz sampling after the step, temporary block)

Parity is pinned: ``tests/test_oracle_golden.py`` checks this module against
``tests/golden/*.npz``, produced by running the reference's own code
(``tests/golden/make_golden.py``) in FP64 and FP32.
"""
import numpy as np
import scipy.sparse as sp

# ----------------------------------------------------------------- model inputs


def load_fiber(n_voxel):
    """Identity diffusion tensors (simulation/equation_parts.py:17-34, fiber_flag 0)."""
    return [np.eye(3) for _ in range(n_voxel)]


def heart_model_equation_parts(simulation_parameters, n_voxel, D0, neighbor_id_2d, parameter):
    """P_2d (n, 21), simulation/equation_parts.py:36-114."""
    D = np.asarray(D0, dtype=np.float64).reshape(n_voxel, 3, 3)
    D11, D12, D13 = D[:, 0, 0], D[:, 0, 1], D[:, 0, 2]
    D21, D22, D23 = D[:, 1, 0], D[:, 1, 1], D[:, 1, 2]
    D31, D32, D33 = D[:, 2, 0], D[:, 2, 1], D[:, 2, 2]
    nb = np.asarray(neighbor_id_2d)
    d = np.sign(nb + 1)
    nb2 = nb.copy()
    nb2[nb2 == -1] = 0
    P = np.zeros((n_voxel, 21))
    P[:, 0] = 4 * d[:, 0] * D11
    P[:, 1] = 4 * d[:, 1] * D11
    P[:, 2] = 4 * d[:, 2] * D22
    P[:, 3] = 4 * d[:, 3] * D22
    P[:, 4] = 4 * d[:, 4] * D33
    P[:, 5] = 4 * d[:, 5] * D33

    def cross(Da, Db, Dc):
        return (d[:, 0] * d[:, 1] * (Da[nb2[:, 0]] - Da[nb2[:, 1]]) +
                d[:, 2] * d[:, 3] * (Db[nb2[:, 2]] - Db[nb2[:, 3]]) +
                d[:, 4] * d[:, 5] * (Dc[nb2[:, 4]] - Dc[nb2[:, 5]]))

    P[:, 6] = d[:, 0] * d[:, 1] * cross(D11, D21, D31)
    P[:, 7] = d[:, 2] * d[:, 3] * cross(D12, D22, D32)
    P[:, 8] = d[:, 4] * d[:, 5] * cross(D13, D23, D33)
    P[:, 9] = 2 * d[:, 6] * d[:, 8] * D12
    P[:, 10] = 2 * d[:, 7] * d[:, 9] * D12
    P[:, 11] = 2 * d[:, 14] * d[:, 16] * D13
    P[:, 12] = 2 * d[:, 15] * d[:, 17] * D13
    P[:, 13] = 2 * d[:, 10] * d[:, 12] * D23
    P[:, 14] = 2 * d[:, 11] * d[:, 13] * D23
    if simulation_parameters['heart_model_flag'] == 0:
        keys = ('tau_open_voxel', 'tau_close_voxel', 'tau_in_voxel', 'tau_out_voxel', 'v_gate_voxel')
    else:
        keys = ('k_voxel', 'a_voxel', 'epsilon_0_voxel', 'mu1_voxel', 'mu2_voxel')
    for c, k in zip(range(15, 20), keys):
        P[:, c] = parameter[k]
    P[:, 20] = parameter['c_voxel']
    return P


# ----------------------------------------------------------------- operator


_CROSS = ((6, 8, 9), (9, 7, 10), (14, 16, 11), (17, 15, 12), (10, 12, 13), (13, 11, 14))


def laplacian(P_2d, neighbor_id_2d, Delta):
    """Diffusion matrix L as scipy CSR, simulation/simulation_gpu.py:138-225.

    Same entries in the same COO order; absent neighbours (-1) are remapped to
    column 0 first (simulation_gpu.py:296-297), so their zero coefficients land
    on column 0 as explicit zeros and duplicates are summed by ``tocsr``.
    """
    P = np.asarray(P_2d, dtype=np.float64)
    n = P.shape[0]
    nb2 = np.asarray(neighbor_id_2d).copy()
    nb2[nb2 == -1] = 0
    Dc = P[:, 20] / (4 * Delta ** 2)
    rows = [np.arange(n)]
    cols = [np.arange(n)]
    vals = [Dc * -(P[:, 0] + P[:, 1] + P[:, 2] + P[:, 3] + P[:, 4] + P[:, 5])]
    ar = np.arange(n)
    for k in range(6):
        rows.append(ar); cols.append(nb2[:, k]); vals.append(Dc * P[:, k])
    for a, b, c in ((0, 1, 6), (2, 3, 7), (4, 5, 8)):
        rows.append(ar); cols.append(nb2[:, a]); vals.append(Dc * P[:, c])
        rows.append(ar); cols.append(nb2[:, b]); vals.append(-Dc * P[:, c])
    for a, b, c in _CROSS:
        rows.append(ar); cols.append(nb2[:, a]); vals.append(Dc * P[:, c])
        rows.append(ar); cols.append(nb2[:, b]); vals.append(-Dc * P[:, c])
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    v = np.concatenate(vals)
    # the reference appends per row (row-major COO); order rows stably
    o = np.argsort(r, kind='stable')
    return sp.coo_matrix((v[o], (r[o], c[o])), shape=(n, n)).tocsr()


# ----------------------------------------------------------------- pacing


def assign_pacing_parameters(arrhythmia_parameters, arrhythmia_flag, n_voxel, simulation_parameters,
                             pacing_duration=None):
    """simulation/pacing.py:102-134 (the do_flag == 0 branch).

    ``pacing_duration`` overrides the hard-coded 5 ms (5/time_scale for AP) when
    given; the reference has no such argument.
    """
    s1 = arrhythmia_parameters['s1_pacing_voxel_id']
    s1_t = arrhythmia_parameters['s1_t']
    s2_t = s1_t + arrhythmia_parameters['s1_s2_delta_t']
    s2 = []
    if arrhythmia_flag in (1, 2, 3, 4, 5, 6):
        s2 = arrhythmia_parameters['s2_pacing_voxel_id']
    if pacing_duration is None:
        pacing_duration = 5 if simulation_parameters['heart_model_flag'] == 0 else \
            5 / simulation_parameters['time_scale']
    return np.zeros(n_voxel), s1, s2, s1_t, 1, pacing_duration, s2_t


def pacing_windows(arrhythmia_parameters, simulation_parameters, arrhythmia_flag, model_time,
                   s1_t, pacing_duration, s2_t):
    """Which sets are paced at ``model_time``: (s1_on, s2_on), simulation/pacing.py:136-170."""
    s1_on = s2_on = False
    if arrhythmia_flag == 0:
        t = model_time
        start = arrhythmia_parameters['pacing_start_time']
        cyc = arrhythmia_parameters['pacing_cycle_length']
        while t - start > cyc:
            t = t - cyc
        if t >= start and t <= start + pacing_duration:
            s1_on = True
    if arrhythmia_flag == 5:
        f1 = 0 / simulation_parameters['time_scale']
        f2 = 300 / simulation_parameters['time_scale']
        if model_time >= f1 and model_time <= f1 + pacing_duration:
            s1_on = True
        if model_time >= f2 and model_time <= f2 + pacing_duration:
            s2_on = True
    if arrhythmia_flag == 6:
        f1 = 0 / simulation_parameters['time_scale']
        f2 = 50 / simulation_parameters['time_scale']
        if model_time >= f1 and model_time <= f1 + pacing_duration:
            s1_on = True
        if model_time >= f2 and model_time <= f2 + pacing_duration:
            s2_on = True
    elif arrhythmia_flag in (1, 2, 3, 4):
        if model_time >= s1_t and model_time <= s1_t + pacing_duration:
            s1_on = True
    if arrhythmia_flag in (1, 2, 3) and model_time >= s2_t and model_time <= s2_t + pacing_duration:
        s2_on = True
    return s1_on, s2_on


# ----------------------------------------------------------------- reaction


def reaction(model, u, h, P, J):
    """simulation/simulation_gpu.py:27-43 (vectorised over voxels)."""
    if model == 0:
        du = (h * (u ** 2) * (1 - u)) / P[:, 17] - u / P[:, 18] + J
        dh = np.where(u < P[:, 19], (1 - h) / P[:, 15], -h / P[:, 16])
    else:
        du = -P[:, 15] * u * (u - P[:, 16]) * (u - 1) - u * h + J
        dh = (P[:, 17] + P[:, 18] * h / (u + P[:, 19])) * (-h - P[:, 15] * u * (u - P[:, 16] - 1))
    return du, dh


def rk4(model, u, h, P, J, dt):
    """simulation/simulation_gpu.py:71-130."""
    k1u, k1h = reaction(model, u, h, P, J)
    k2u, k2h = reaction(model, u + 0.5 * dt * k1u, h + 0.5 * dt * k1h, P, J)
    k3u, k3h = reaction(model, u + 0.5 * dt * k2u, h + 0.5 * dt * k2h, P, J)
    k4u, k4h = reaction(model, u + dt * k3u, h + dt * k3h, P, J)
    us = u + (dt / 6.0) * (k1u + 2.0 * k2u + 2.0 * k3u + k4u)
    hs = h + (dt / 6.0) * (k1h + 2.0 * k2h + 2.0 * k3h + k4h)
    return us, hs


# ----------------------------------------------------------------- GMRES


def gmres(A, b, x0, tol=1e-5, atol=None, restart=50, maxiter=None, stats=None):
    """Restarted GMRES with CuPy's semantics (the solver called at
    simulation/simulation_gpu.py:253): atol_eff = max(atol, tol*||b||);
    ||b|| == 0 returns b; a true-residual test at each cycle start; full
    cycles of classical Gram-Schmidt; Hessenberg least squares with lstsq.
    Returns (x, info)."""
    n = b.shape[0]
    b = np.asarray(b, dtype=np.float64)
    x = np.array(x0, dtype=np.float64, copy=True)
    b_norm = np.linalg.norm(b)
    if b_norm == 0:
        return b.copy(), 0
    atol = tol * b_norm if atol is None else max(float(atol), tol * b_norm)
    maxiter = n * 10 if maxiter is None else maxiter
    m = min(restart, n)
    V = np.empty((n, m), order='F')
    H = np.zeros((m + 1, m), order='F')
    e = np.zeros(m + 1)
    iters = 0
    while True:
        r = b - A @ x
        r_norm = np.linalg.norm(r)
        if r_norm <= atol or iters >= maxiter:
            break
        V[:, 0] = r / r_norm
        e[:] = 0
        e[0] = r_norm
        v = V[:, 0]
        for j in range(m):
            u = A @ v
            h = V[:, :j + 1].T @ u
            u = u - V[:, :j + 1] @ h
            H[:j + 1, j] = h
            H[j + 1, j] = np.linalg.norm(u)
            if j + 1 < m:
                v = u / H[j + 1, j]
                V[:, j + 1] = v
        y = np.linalg.lstsq(H, e, rcond=None)[0]
        x += V @ y
        iters += m
        if stats is not None:
            stats['arnoldi'] = stats.get('arnoldi', 0) + m
    info = iters if (iters == maxiter and not r_norm <= atol) else 0
    return x, info


# ----------------------------------------------------------------- driver


def step_schedule(simulation_parameters):
    """(steps, samples, stride) of simulation/simulation_gpu.py:286-290, 355-356."""
    t_final = float(simulation_parameters['t_final'])
    dt = simulation_parameters['dt']
    if simulation_parameters['heart_model_flag'] == 0:
        n_samples = int(np.round(t_final))
    else:
        n_samples = int(np.round(t_final * simulation_parameters['time_scale']))
    steps = int(np.round(t_final / dt))
    stride = int(1 / (dt * simulation_parameters['time_scale']))
    return steps, n_samples, stride


def compute(n_voxel, P_2d, geometry_data, simulation_parameters, arrhythmia_parameters,
            max_steps=None, pacing_duration=None, tol=1e-5, restart=50, record_lat=False,
            stats=None):
    """FP64 restatement of simulation/simulation_gpu.py:261-409.

    Returns (u_hist, h_hist, physical_time) like the reference, plus the
    activation step table (first step after which u >= 0.5, -1 if none) when
    ``record_lat``.  ``max_steps`` truncates the run (sampling unchanged).
    """
    node_flag = np.asarray(arrhythmia_parameters['node_flag'])
    temp_ids = np.where(node_flag == 3)[0]
    perm_ids = np.where(node_flag == 4)[0]
    nb = np.asarray(geometry_data['neighbor_id_2d'])
    Delta = geometry_data['Delta']
    t_final = float(simulation_parameters['t_final'])
    dt = simulation_parameters['dt']
    flag = simulation_parameters['arrhythmia_flag']
    model = simulation_parameters['heart_model_flag']
    _, s1, s2, s1_t, Jmag, pdur, s2_t = assign_pacing_parameters(
        arrhythmia_parameters, flag, n_voxel, simulation_parameters, pacing_duration)
    u = np.zeros(n_voxel)
    h = np.ones(n_voxel) if model == 0 else np.zeros(n_voxel)
    steps, n_samples, stride = step_schedule(simulation_parameters)
    if max_steps is not None:
        steps = min(steps, max_steps)
    U = np.zeros((n_samples, n_voxel))
    Hh = np.zeros((n_samples, n_voxel))
    T = np.zeros(n_samples)
    P = np.array(P_2d, dtype=np.float64, copy=True)
    Pp = P.copy()
    Pp[perm_ids, 20] = 0.0
    L = laplacian(Pp, nb, Delta)
    I = sp.identity(n_voxel, format='csr')
    A = I - (dt / 2.0) * L
    if len(temp_ids) > 0:
        Pt = Pp.copy()
        Pt[temp_ids, 20] = 0.0
        Lt = laplacian(Pt, nb, Delta)
        At = I - (dt / 2.0) * Lt
    else:
        Lt, At = L, A
    lat = np.full(n_voxel, -1, dtype=np.int64)
    id_save = 0
    s1 = np.atleast_1d(np.asarray(s1, dtype=np.int64)) if np.size(s1) else np.zeros(0, np.int64)
    s2 = np.atleast_1d(np.asarray(s2, dtype=np.int64)) if np.size(s2) else np.zeros(0, np.int64)
    for step in range(steps):
        mt = step * dt
        if mt >= 0 and mt < 350 * dt:
            aL, aA = Lt, At
        else:
            aL, aA = L, A
        s1_on, s2_on = pacing_windows(arrhythmia_parameters, simulation_parameters, flag, mt,
                                      s1_t, pdur, s2_t)
        J = np.zeros(n_voxel)
        if s1_on:
            J[s1] = Jmag
        if s2_on:
            J[s2] = Jmag
        us, hn = rk4(model, u, h, P, J, dt)
        b = us + (dt / 2.0) * (aL @ us)
        u, _ = gmres(aA, b, us, tol=tol, atol=1e-5, restart=restart, maxiter=10000, stats=stats)
        h = hn
        if record_lat:
            lat[(lat < 0) & (u >= 0.5)] = step
        if stride > 0:
            if step % stride == 0 and id_save < n_samples:
                U[id_save], Hh[id_save], T[id_save] = u, h, mt * simulation_parameters['time_scale']
                id_save += 1
        elif id_save < n_samples:
            U[id_save], Hh[id_save], T[id_save] = u, h, mt * simulation_parameters['time_scale']
            id_save += 1
    out = (U[:id_save], Hh[:id_save], T[:id_save])
    return out + (lat,) if record_lat else out
