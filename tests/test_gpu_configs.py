"""The named accuracy configurations on the GPU.

* sheet (c1): the plain FP64 drop-in over the whole 500 ms run (10,000 steps,
  40,000 voxels) and its 16-electrode electrogram against the FP64 oracle's
  run of the same configuration (tests/golden/c1_sheet_oracle.npz,
  tests/golden/make_golden_c1.py);
* rotor shell (c2): the full geometry (91,292 voxels, Aliev-Panfilov, S1 plane
  + S2 quadrant) over the first 40 ms, the FP32 early-exit path against the
  plain FP64 path;
* batched shells (c3): one Mitchell-Schaeffer and one Aliev-Panfilov instance
  of the benchmark batch at their full size over the first 40 ms, FP32 against
  plain FP64.
The full-length c2 and c3 comparisons run in bench.py's accuracy leg.
"""
import numpy as np
import pytest

from pyheartsim_b200 import workloads
from pyheartsim_b200.simulation import simulation_gpu, unipolar_electrogram_gpu
from tests import golden_cases

pytestmark = pytest.mark.gpu

PLAIN_ATOL = 1e-9          # plain FP64 path vs the FP64 oracle, |dVm|
EGM_RTOL = 1e-10           # FP64 electrogram, relative L2
FAST_LAT_STEPS = 1         # FP32 early-exit path: activation steps within 1 dt
FAST_DVM = 1e-3            # FP32 early-exit path: max |dVm| over the first 40 ms


def test_c1_sheet_full_run_matches_oracle(cuda_device):
    (n, P, geom, sp, ap), pdur, el = workloads.sheet_c1()
    g = np.load(f"{golden_cases.GOLDEN}/c1_sheet_oracle.npz")
    u, h, t, lat = simulation_gpu.compute(n, P, geom, dict(sp), dict(ap), pacing_duration=pdur, return_lat=True)
    assert u.shape == (500, 40000) and u.dtype == np.float64
    np.testing.assert_array_equal(t, g["physical_time"])
    np.testing.assert_array_equal(lat, g["lat"])                      # activation step of every voxel
    np.testing.assert_allclose(u[g["sample_ids"]], g["u_at"], rtol=0, atol=PLAIN_ATOL)
    # every sample through its sum and sum of squares (n x the per-voxel bound)
    np.testing.assert_allclose(u.sum(axis=1), g["u_sum"], rtol=0, atol=n * PLAIN_ATOL)
    np.testing.assert_allclose((u * u).sum(axis=1), g["u_sq"], rtol=0, atol=2 * n * PLAIN_ATOL)
    egm = unipolar_electrogram_gpu.compute(el, geom['voxel'], None, P[:, 20], u, geom['Delta'],
                                           geom['neighbor_id_2d'])
    rel = np.linalg.norm(egm - g["egm"]) / np.linalg.norm(g["egm"])
    assert rel < EGM_RTOL, rel


def _fast_vs_plain(case, pdur):
    n, P, geom, sp, ap = case
    u64, _, _, lat64, info = simulation_gpu.compute(n, P, geom, dict(sp), dict(ap), pacing_duration=pdur,
                                                    return_lat=True, return_info=True)
    u32, _, _, lat32 = simulation_gpu.compute(n, P, geom, dict(sp), dict(ap), pacing_duration=pdur,
                                              dtype=np.float32, fast=True, tol=1e-7, return_lat=True)
    # a voxel may cross Vm = 0.5 in one run's last step and one step after the
    # end in the other; any other voxel activates in both runs or in neither
    one = (lat64 >= 0) != (lat32 >= 0)
    last = info["steps"] - FAST_LAT_STEPS
    assert np.all(np.maximum(lat64[one], lat32[one]) >= last), "a voxel activated in one precision only"
    both = (lat64 >= 0) & (lat32 >= 0)
    assert both.sum() > n // 20, "the case must propagate"
    dlat = int(np.abs(lat64[both].astype(np.int64) - lat32[both]).max())
    dvm = float(np.abs(u64 - u32).max())
    assert dlat <= FAST_LAT_STEPS, dlat
    assert dvm < FAST_DVM, dvm


def test_c2_rotor_shell_full_geometry_first_40ms(cuda_device):
    (n, P, geom, sp, ap), pdur, _ = workloads.atrium_c2(wall=3, t_phys=40.0)
    assert n == 91292
    _fast_vs_plain((n, P, geom, sp, ap), pdur)


@pytest.mark.parametrize("i", [0, 1])
def test_c3_batch_instances_first_40ms(i, cuda_device):
    """Instance i of the benchmark batch (seed 0): 0 is Mitchell-Schaeffer, 1
    Aliev-Panfilov, at their full sizes."""
    sizes = workloads.batch_sizes(64, 50_000, 400_000, 0)
    _, case, meta = workloads.shell_case(i, int(sizes[i]), 0, t_phys=40.0)
    assert meta["model"] == i % 2
    _fast_vs_plain(case, meta["pacing_ms"] / case[3]["time_scale"])
