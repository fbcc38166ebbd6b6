"""Generate ``tests/golden/c1_sheet_oracle.npz``: the FP64 oracle's run of the
plain sheet configuration at its full size.

Test infrastructure only.  The configuration (``workloads.sheet_c1``): a
200 x 200 Mitchell-Schaeffer sheet, dt 0.05 ms, a 1 ms corner stimulus,
500 ms = 10,000 steps, 16 electrodes on a 4 x 4 grid 1 mm above the sheet.
The reference's own code cannot run this size here (its kernels run under
the Numba CUDA simulator at seconds per step), so the fixture comes from the
FP64 oracle (``oracle/simulation_fp64.py``, ``oracle/egm_fp64.py``), which is
itself pinned to the reference's own runs by ``tests/test_oracle_golden.py``.
About 10 minutes on 8 cores.

The full (500, 40000) history does not fit a small fixture, so the file
keeps what the GPU test compares:

* ``lat``           activation step of every voxel (first step after which
                    u >= 0.5, -1 if none);
* ``u_at``          u at the samples ``sample_ids`` (all voxels);
* ``u_sum``, ``u_sq`` per-sample sum and sum of squares of u (all 500 samples);
* ``egm``           the normalised FP64 electrogram (500, 16);
* ``physical_time`` the sample times.

Run:  python tests/golden/make_golden_c1.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SAMPLE_IDS = np.array([20, 100, 250, 499])


def main():
    from oracle import egm_fp64, simulation_fp64
    from pyheartsim_b200 import workloads
    (n, P, geom, sp, ap), pdur, el = workloads.sheet_c1()
    t0 = time.perf_counter()
    u, h, t, lat = simulation_fp64.compute(n, P, geom, dict(sp), dict(ap), pacing_duration=pdur, record_lat=True)
    t_sim = time.perf_counter() - t0
    egm = egm_fp64.compute(el, geom['voxel'], None, P[:, 20], u, geom['Delta'], geom['neighbor_id_2d'])
    np.savez_compressed(os.path.join(HERE, "c1_sheet_oracle.npz"), lat=lat.astype(np.int32),
                        sample_ids=SAMPLE_IDS, u_at=u[SAMPLE_IDS], u_sum=u.sum(axis=1), u_sq=(u * u).sum(axis=1),
                        egm=egm, physical_time=t, electrodes=el)
    print(f"c1: {n} voxels, {u.shape[0]} samples, oracle {t_sim:.0f} s, activated {int((lat >= 0).sum())}, "
          f"last activation step {int(lat.max())}")


if __name__ == "__main__":
    main()
