"""Voxel geometry and model tables in the reference's formats.

* ``lattice_neighbors``: the (n, 18) neighbour table of
  utility/voxelization.py:102-152 (same column order, -1 for absent), built by
  hashing integer lattice coordinates instead of one KDTree query per neighbour;
* ``heart_model_equation_parts``: P_2d (n, 21) of
  simulation/equation_parts.py:36-114, vectorised;
* ``load_fiber``: identity D0 list of simulation/equation_parts.py:17-34.
"""
import numpy as np

# neighbour offsets in the reference's column order (utility/voxelization.py:107-132)
OFFSETS = np.array([
    [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
    [1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0],
    [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1],
    [1, 0, 1], [-1, 0, 1], [1, 0, -1], [-1, 0, -1],
], dtype=np.int64)


def lattice_neighbors(ijk):
    """(n, 18) int64 neighbour table of integer coordinates ``ijk`` (n, 3)."""
    ijk = np.asarray(np.rint(ijk), dtype=np.int64)
    n = ijk.shape[0]
    lo = ijk.min(axis=0) - 1
    span = ijk.max(axis=0) - lo + 2
    key = lambda p: ((p[:, 0] - lo[0]) * span[1] + (p[:, 1] - lo[1])) * span[2] + (p[:, 2] - lo[2])
    keys = key(ijk)
    order = np.argsort(keys, kind="stable")
    sk = keys[order]
    if n > 1 and np.any(sk[1:] == sk[:-1]):
        raise ValueError("duplicate voxel coordinates")
    nb = np.full((n, 18), -1, dtype=np.int64)
    for c, off in enumerate(OFFSETS):
        q = key(ijk + off)
        pos = np.searchsorted(sk, q)
        pos = np.minimum(pos, n - 1)
        hit = sk[pos] == q
        nb[hit, c] = order[pos[hit]]
    return nb


def load_fiber(n_voxel):
    """Identity diffusion tensor per voxel (simulation/equation_parts.py:17-34)."""
    return [np.eye(3) for _ in range(n_voxel)]


def heart_model_equation_parts(simulation_parameters, n_voxel, D0, neighbor_id_2d, parameter):
    """P_2d (n, 21), simulation/equation_parts.py:36-114."""
    if D0 is None:
        D = np.broadcast_to(np.eye(3), (n_voxel, 3, 3))
    else:
        D = np.asarray(D0, dtype=np.float64).reshape(n_voxel, 3, 3)
    nb = np.asarray(neighbor_id_2d)
    d = np.sign(nb + 1)
    nb2 = nb.copy()
    nb2[nb2 == -1] = 0
    P = np.zeros((n_voxel, 21))
    for k, (i, j) in enumerate(((0, 0), (0, 0), (1, 1), (1, 1), (2, 2), (2, 2))):
        P[:, k] = 4 * d[:, k] * D[:, i, j]

    def cross(col):
        return (d[:, 0] * d[:, 1] * (D[nb2[:, 0], 0, col] - D[nb2[:, 1], 0, col]) +
                d[:, 2] * d[:, 3] * (D[nb2[:, 2], 1, col] - D[nb2[:, 3], 1, col]) +
                d[:, 4] * d[:, 5] * (D[nb2[:, 4], 2, col] - D[nb2[:, 5], 2, col]))

    P[:, 6] = d[:, 0] * d[:, 1] * cross(0)
    P[:, 7] = d[:, 2] * d[:, 3] * cross(1)
    P[:, 8] = d[:, 4] * d[:, 5] * cross(2)
    P[:, 9] = 2 * d[:, 6] * d[:, 8] * D[:, 0, 1]
    P[:, 10] = 2 * d[:, 7] * d[:, 9] * D[:, 0, 1]
    P[:, 11] = 2 * d[:, 14] * d[:, 16] * D[:, 0, 2]
    P[:, 12] = 2 * d[:, 15] * d[:, 17] * D[:, 0, 2]
    P[:, 13] = 2 * d[:, 10] * d[:, 12] * D[:, 1, 2]
    P[:, 14] = 2 * d[:, 11] * d[:, 13] * D[:, 1, 2]
    if simulation_parameters['heart_model_flag'] == 0:
        keys = ('tau_open_voxel', 'tau_close_voxel', 'tau_in_voxel', 'tau_out_voxel', 'v_gate_voxel')
    else:
        keys = ('k_voxel', 'a_voxel', 'epsilon_0_voxel', 'mu1_voxel', 'mu2_voxel')
    for c, k in zip(range(15, 20), keys):
        P[:, c] = parameter[k]
    P[:, 20] = parameter['c_voxel']
    return P
