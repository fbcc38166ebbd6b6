"""FP64 CPU oracle of PyHeartSim's unipolar electrogram.

TEST INFRASTRUCTURE ONLY (imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py``; never by the product package).

Restates, in FP64, ``simulation/unipolar_electrogram_gpu.py::compute``
(jiyuehe/PyHeartSim):

* D-tensor split            simulation/unipolar_electrogram_equation_parts.py:17-39
* electrode distances       ...equation_parts.py:41-58  (l = |x_v - x_e|, l < 1 -> 1)
* gradients                 ...equation_parts.py:60-103 (central difference,
                            zero where either neighbour is missing)
* per-(voxel, electrode, t) sum of the kernel simulation/unipolar_electrogram_gpu.py:55-69
* normalisation             ...equation_parts.py:118-124 (1 / mean ptp)

``direct`` follows the reference term by term; ``leadfield`` folds everything
but V into one (n_v, n_e) matrix so that egm = V @ M (the at-scale oracle).
Parity is pinned against ``tests/golden/*.npz`` (reference run under the
Numba CUDA simulator).
"""
import numpy as np


def electrode_distances(electrode_xyz, voxel):
    """(l, lx, ly, lz), each (n_v, n_e); ...equation_parts.py:41-58."""
    lx = voxel[:, 0:1] - electrode_xyz[None, :, 0]
    ly = voxel[:, 1:2] - electrode_xyz[None, :, 1]
    lz = voxel[:, 2:3] - electrode_xyz[None, :, 2]
    l = np.sqrt(lx ** 2 + ly ** 2 + lz ** 2)
    l[l < 1] = 1
    return l, lx, ly, lz


def gradients(V, neighbor_id_2d, Delta):
    """(dvdx, dvdy, dvdz), each (T, n_v); ...equation_parts.py:60-103."""
    nb = np.asarray(neighbor_id_2d)
    out = []
    for a, b in ((0, 1), (2, 3), (4, 5)):
        p = nb[:, a].copy()
        m = nb[:, b].copy()
        p0, m0 = p == -1, m == -1
        p[p0] = 0
        m[m0] = 0
        g = (V[:, p] - V[:, m]) / (2 * Delta)
        g[:, p0] = 0
        g[:, m0] = 0
        out.append(g)
    return tuple(out)


def normalize(egm, typical_magnitude=1.0):
    """...equation_parts.py:118-124."""
    voltage = np.array([np.ptp(egm[:, e]) for e in range(egm.shape[1])])
    return egm * (typical_magnitude / np.mean(voltage))


def _dtensor(D0, n_v):
    if D0 is None:
        return np.broadcast_to(np.eye(3), (n_v, 3, 3))
    return np.asarray(D0, dtype=np.float64).reshape(n_v, 3, 3)


def direct(electrode_xyz, voxel, D0, c_voxel, V, Delta, neighbor_id_2d, normalise=True,
           chunk=4096):
    """Term-by-term FP64 sum of simulation/unipolar_electrogram_gpu.py:55-69."""
    V = np.asarray(V, dtype=np.float64)
    electrode_xyz = np.asarray(electrode_xyz, dtype=np.float64)
    voxel = np.asarray(voxel, dtype=np.float64)
    n_v = voxel.shape[0]
    D = _dtensor(D0, n_v)
    gx, gy, gz = gradients(V, neighbor_id_2d, Delta)
    c = np.asarray(c_voxel, dtype=np.float64)
    T = V.shape[0]
    egm = np.zeros((T, electrode_xyz.shape[0]))
    for v0 in range(0, n_v, chunk):
        sl = slice(v0, min(n_v, v0 + chunk))
        l, lx, ly, lz = electrode_distances(electrode_xyz, voxel[sl])
        Ds = D[sl]
        fx = Ds[:, 0, 0][None] * gx[:, sl] + Ds[:, 0, 1][None] * gy[:, sl] + Ds[:, 0, 2][None] * gz[:, sl]
        fy = Ds[:, 1, 0][None] * gx[:, sl] + Ds[:, 1, 1][None] * gy[:, sl] + Ds[:, 1, 2][None] * gz[:, sl]
        fz = Ds[:, 2, 0][None] * gx[:, sl] + Ds[:, 2, 1][None] * gy[:, sl] + Ds[:, 2, 2][None] * gz[:, sl]
        w = c[sl][:, None] / (l ** 3)
        egm += fx @ (w * lx) + fy @ (w * ly) + fz @ (w * lz)
    return normalize(egm) if normalise else egm


def leadfield(electrode_xyz, voxel, D0, c_voxel, Delta, neighbor_id_2d, chunk=8192):
    """M (n_v, n_e) with egm_raw = V @ M, FP64.

    g[v,e,:] = c_v / l^3 * D_v^T l_ve is the weight of grad V at voxel v;
    the central difference spreads it to the +d neighbour (+1/(2 Delta)) and
    the -d neighbour (-1/(2 Delta)) when both exist.
    """
    electrode_xyz = np.asarray(electrode_xyz, dtype=np.float64)
    voxel = np.asarray(voxel, dtype=np.float64)
    nb = np.asarray(neighbor_id_2d)
    n_v = voxel.shape[0]
    n_e = electrode_xyz.shape[0]
    D = _dtensor(D0, n_v)
    c = np.asarray(c_voxel, dtype=np.float64)
    M = np.zeros((n_v, n_e))
    for v0 in range(0, n_v, chunk):
        idx = np.arange(v0, min(n_v, v0 + chunk))
        l, lx, ly, lz = electrode_distances(electrode_xyz, voxel[idx])
        w = c[idx][:, None] / (l ** 3)
        Ds = D[idx]
        for d, (a, b) in enumerate(((0, 1), (2, 3), (4, 5))):
            g = w * (Ds[:, 0, d][:, None] * lx + Ds[:, 1, d][:, None] * ly + Ds[:, 2, d][:, None] * lz)
            p = nb[idx, a]
            m = nb[idx, b]
            ok = (p >= 0) & (m >= 0)
            g = g[ok] / (2 * Delta)
            np.add.at(M, p[ok], g)
            np.add.at(M, m[ok], -g)
    return M


def compute(electrode_xyz, voxel, D0, c_voxel, action_potential, Delta, neighbor_id_2d,
            batch_size=50):
    """Drop-in signature of simulation/unipolar_electrogram_gpu.py:71 (FP64 oracle)."""
    M = leadfield(electrode_xyz, voxel, D0, c_voxel, Delta, neighbor_id_2d)
    return normalize(np.asarray(action_potential, dtype=np.float64) @ M)
