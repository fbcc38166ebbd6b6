"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No patient meshes are available, so every workload is generated here from
``numpy.random.default_rng(seed)``:

* ``sheet``          2-D sheet of nx x ny voxels (reference geometry order);
* ``shell``          voxelised ellipsoidal shell with cylindrical vein holes;
* ``scar``           Gaussian-blob scar mask: c = 0 inside, c_border on a
                     one-voxel ring around it;
* ``make_case``      the reference's argument dicts for one simulation;
* ``electrodes_*``   electrode positions.
Voxels are ordered z-major, then y, then x (rows along x are contiguous),
which keeps +-x neighbours adjacent in memory.
"""
import numpy as np

from .geometry import heart_model_equation_parts, lattice_neighbors

MS_PARAMS = dict(tau_in=0.3, tau_out=6.0, tau_open=120.0, tau_close=150.0, v_gate=0.13)
AP_PARAMS = dict(k=8.0, a=0.15, epsilon_0=0.002, mu1=0.2, mu2=0.3)


def _order_zyx(ijk):
    o = np.lexsort((ijk[:, 0], ijk[:, 1], ijk[:, 2]))
    return ijk[o]


def sheet(nx, ny, order="reference"):
    """Integer coordinates of an nx x ny sheet.  ``reference`` order is x outer,
    y inner (tool/create_geometry.py:55-60); ``zyx`` is rows along x."""
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    ijk = np.stack([i.ravel(), j.ravel(), np.zeros(nx * ny, dtype=np.int64)], axis=1).astype(np.int64)
    return _order_zyx(ijk) if order == "zyx" else ijk


def shell(semi_axes=(25.0, 20.0, 18.0), Delta=0.4, wall=3, n_holes=4, hole_radius=5.0, seed=0):
    """Voxelised ellipsoidal shell: lattice points (spacing Delta, in mm) whose
    scaled radius lies in the outer `wall` voxels of the ellipsoid, minus
    `n_holes` cylinders of `hole_radius` mm along seeded radial directions.
    Returns integer coordinates (n, 3) ordered z, y, x."""
    a = np.asarray(semi_axes, dtype=np.float64)
    ext = np.ceil(a / Delta).astype(int) + 1
    rng = np.random.default_rng(seed)
    pts = []
    for kz in range(-ext[2], ext[2] + 1):
        z = kz * Delta
        ys = np.arange(-ext[1], ext[1] + 1)
        xs = np.arange(-ext[0], ext[0] + 1)
        X, Y = np.meshgrid(xs * Delta, ys * Delta, indexing="xy")
        r = np.sqrt((X / a[0]) ** 2 + (Y / a[1]) ** 2 + (z / a[2]) ** 2)
        # distance below the surface measured along the normal, approximately
        grad = np.sqrt((X / a[0] ** 2) ** 2 + (Y / a[1] ** 2) ** 2 + (z / a[2] ** 2) ** 2)
        depth = (1.0 - r) * r / np.maximum(grad, 1e-12)
        inside = (r <= 1.0) & (depth < wall * Delta)
        jj, ii = np.nonzero(inside)
        if ii.size:
            pts.append(np.stack([xs[ii], ys[jj], np.full(ii.size, kz)], axis=1))
    ijk = np.concatenate(pts).astype(np.int64)
    xyz = ijk * Delta
    keep = np.ones(ijk.shape[0], dtype=bool)
    for _ in range(n_holes):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        proj = xyz @ d
        perp = xyz - proj[:, None] * d[None, :]
        keep &= ~((np.linalg.norm(perp, axis=1) < hole_radius) & (proj > 0))
    return _order_zyx(ijk[keep])


def shell_for_size(n_target, seed=0, Delta=0.4, wall=3, base=(25.0, 20.0, 18.0), n_holes=4, hole_radius=5.0):
    """Shell scaled so that its voxel count is close to ``n_target``."""
    n0 = shell(base, Delta, wall, n_holes, hole_radius, seed).shape[0]
    s = np.sqrt(n_target / n0)
    for _ in range(3):
        ijk = shell(tuple(np.asarray(base) * s), Delta, wall, n_holes, hole_radius * s, seed)
        s *= np.sqrt(n_target / ijk.shape[0])
    return ijk


def scar(ijk, nb, coverage, rng, c_border=0.1, n_blobs=6, width=8.0):
    """Conductivity scale (n,): Gaussian-blob field thresholded to ``coverage``;
    0 inside, ``c_border`` on the one-voxel ring around the scar (face
    neighbours ``nb[:, :6]``; with ``nb`` None, the face neighbours are looked
    up in a dense occupancy grid of the lattice coordinates, same result), 1
    elsewhere."""
    n = ijk.shape[0]
    c = np.ones(n)
    if coverage <= 0:
        return c
    centers = ijk[rng.integers(0, n, size=n_blobs)].astype(np.float64)
    f = np.zeros(n)
    for cc in centers:
        f += np.exp(-np.sum((ijk - cc) ** 2, axis=1) / (2 * width ** 2))
    thr = np.quantile(f, 1.0 - coverage)
    core = f >= thr
    ring = np.zeros(n, dtype=bool)
    if nb is None:
        lo = ijk.min(axis=0) - 1
        g = ijk - lo
        grid = np.zeros(tuple(g.max(axis=0) + 2), dtype=bool)
        grid[g[core, 0], g[core, 1], g[core, 2]] = True
        for d in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
            q = g + np.asarray(d)
            ring |= grid[q[:, 0], q[:, 1], q[:, 2]]
    else:
        nbs = nb[:, :6]
        for k in range(6):
            q = nbs[:, k]
            ok = q >= 0
            ring[ok] |= core[q[ok]]
    ring &= ~core
    c[core] = 0.0
    c[ring] = c_border
    return c


def model_parameters(model, n, c_voxel):
    if model == 0:
        p = MS_PARAMS
        return {'tau_in_voxel': np.full(n, p['tau_in']), 'tau_out_voxel': np.full(n, p['tau_out']),
                'tau_open_voxel': np.full(n, p['tau_open']), 'tau_close_voxel': np.full(n, p['tau_close']),
                'v_gate_voxel': np.full(n, p['v_gate']), 'c_voxel': np.asarray(c_voxel, dtype=np.float64)}
    p = AP_PARAMS
    return {'k_voxel': np.full(n, p['k']), 'a_voxel': np.full(n, p['a']),
            'epsilon_0_voxel': np.full(n, p['epsilon_0']), 'mu1_voxel': np.full(n, p['mu1']),
            'mu2_voxel': np.full(n, p['mu2']), 'c_voxel': np.asarray(c_voxel, dtype=np.float64)}


def fibre_tensors(ijk, r=0.3, helix_deg=60.0):
    """Rule-based fibre field of a shell centred on the origin, as diffusion
    tensors D0 = r I + (1 - r) e e^T (the fiber_flag == 1 form of
    simulation/equation_parts.py:28-29).  The fibre e lies in the wall's tangent
    plane and turns with depth from +helix_deg (inner surface) to -helix_deg
    (outer), measured from the circumferential direction.  Returns (n, 3, 3)."""
    x = np.asarray(ijk, dtype=np.float64)
    rho = np.linalg.norm(x, axis=1)
    rad = x / np.maximum(rho, 1e-9)[:, None]
    circ = np.cross(np.array([0.0, 0.0, 1.0]), rad)
    small = np.linalg.norm(circ, axis=1) < 1e-6
    circ[small] = np.array([1.0, 0.0, 0.0])
    circ /= np.linalg.norm(circ, axis=1)[:, None]
    lng = np.cross(rad, circ)
    # depth through the wall from the radius, 0 inside .. 1 outside
    t = (rho - rho.min()) / max(rho.max() - rho.min(), 1e-9)
    a = np.deg2rad(helix_deg) * (1.0 - 2.0 * t)
    e = np.cos(a)[:, None] * circ + np.sin(a)[:, None] * lng
    return r * np.eye(3)[None] + (1.0 - r) * e[:, :, None] * e[:, None, :]


def make_case(ijk, Delta, model, dt_phys, t_phys, s1_ids, *, c_phys=None, s2_ids=None, flag=4,
              s1_t=0.0, s1_s2=0.0, start=10.0, cycle=300.0, node_flag=None, c_scale=None, D0=None):
    """The reference's (n_voxel, P_2d, geometry_data, simulation_parameters,
    arrhythmia_parameters) for one simulation, with the reference's time scaling
    for Aliev-Panfilov (configuration.py:145-157: dt, t_final and pacing times
    divided by 6, c multiplied by 6).  ``D0``: (n, 3, 3) diffusion tensors
    (default identity, the reference's load_fiber)."""
    n = ijk.shape[0]
    nb = lattice_neighbors(ijk)
    sp, ap, par = case_parameters(n, model, dt_phys, t_phys, s1_ids, c_phys=c_phys, s2_ids=s2_ids, flag=flag,
                                  s1_t=s1_t, s1_s2=s1_s2, start=start, cycle=cycle, node_flag=node_flag,
                                  c_scale=c_scale)
    P = heart_model_equation_parts(sp, n, D0, nb, par)
    geom = {'neighbor_id_2d': nb, 'Delta': Delta, 'voxel': ijk * Delta}
    return n, P, geom, sp, ap


def case_parameters(n, model, dt_phys, t_phys, s1_ids, *, c_phys=None, s2_ids=None, flag=4, s1_t=0.0, s1_s2=0.0,
                    start=10.0, cycle=300.0, node_flag=None, c_scale=None):
    """(simulation_parameters, arrhythmia_parameters, parameter) of make_case,
    without the geometry tables (for builders that make those on the device)."""
    ts = 1 if model == 0 else 6
    if c_phys is None:
        c_phys = 1.0 if model == 0 else 1.6
    c = np.full(n, c_phys * ts)
    if c_scale is not None:
        c = c * c_scale
    sp = {'t_final': t_phys / ts, 'dt': dt_phys / ts, 'heart_model_flag': model, 'arrhythmia_flag': flag,
          'time_scale': ts}
    ap = {'pacing_start_time': start / ts, 'pacing_cycle_length': cycle / ts,
          's1_pacing_voxel_id': np.asarray(s1_ids, dtype=np.int64),
          's2_pacing_voxel_id': np.asarray(s2_ids if s2_ids is not None else [], dtype=np.int64),
          's1_t': s1_t / ts, 's1_s2_delta_t': s1_s2 / ts,
          'node_flag': np.zeros(n, dtype=np.int64) if node_flag is None else node_flag}
    par = model_parameters(model, n, c)
    return sp, ap, par


def electrodes_grid(nx, ny, Delta, nside=4, z=1.0):
    """nside x nside electrodes at 1/8, 3/8, ... of a sheet, height z (mm)."""
    fr = (np.arange(nside) * 2 + 1) / (2 * nside)
    X, Y = np.meshgrid(fr * (nx - 1) * Delta, fr * (ny - 1) * Delta, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), np.full(X.size, z)], axis=1)


def electrodes_off_surface(ijk, Delta, n_e, rng, offset=2.0):
    """n_e electrodes at seeded surface voxels, ``offset`` mm along the outward
    direction from the centroid."""
    xyz = ijk * Delta
    ctr = xyz.mean(axis=0)
    idx = rng.choice(xyz.shape[0], size=n_e, replace=xyz.shape[0] < n_e)
    d = xyz[idx] - ctr
    d /= np.maximum(np.linalg.norm(d, axis=1, keepdims=True), 1e-12)
    return xyz[idx] + offset * d


def small_shell_case(seed=1, t_phys=40.0, dt=0.05, scar_cov=0.15, fibres=False):
    """A small scarred Mitchell-Schaeffer shell (semi-axes 9/8/7 mm, wall 3
    voxels, two vein holes, ~12k voxels) paced at one seeded healthy site:
    ((n, P_2d, geometry_data, simulation_parameters, arrhythmia_parameters),
    pacing_ms).  ``fibres``: rule-based fibre field (anisotropic D0)."""
    ijk = shell((9.0, 8.0, 7.0), 0.4, 3, 2, 2.0, seed)
    rng = np.random.default_rng(seed)
    nb = lattice_neighbors(ijk)
    c = scar(ijk, nb, scar_cov, rng)
    healthy = np.where(c == 1.0)[0]
    centre = ijk[healthy[int(rng.integers(0, healthy.size))]]
    s1 = np.where(np.sum((ijk - centre) ** 2, axis=1) <= 9)[0]
    D0 = fibre_tensors(ijk) if fibres else None
    return make_case(ijk, 0.4, 0, dt, t_phys, s1, flag=4, c_scale=c, D0=D0), 2.0
