"""Electrode LAT and conduction velocity on the GPU against the reference's
own outputs (tests/golden/analysis_*.npz) and the oracle."""
import numpy as np
import pytest

from oracle import analysis as oracle_analysis
from pyheartsim_b200 import analysis
from tests import golden_cases

pytestmark = pytest.mark.gpu

CV_RTOL = 1e-9     # SVD plane fit vs numpy's LAPACK lstsq, FP64


@pytest.mark.parametrize("name", golden_cases.analysis_names())
def test_lat_and_cv_match_reference(name, cuda_device):
    g = np.load(f"{golden_cases.GOLDEN}/{name}.npz")
    lat = analysis.compute_electrode_lat(g["egm"])
    np.testing.assert_array_equal(lat, g["lat_electrode"])            # integer: bit-exact
    vec, mag, mean = analysis.compute({"electrogram_unipolar": g["egm"]},
                                      {"voxel": g["voxel"], "voxel_id_of_simulation_electrode": g["electrode_ids"]})
    np.testing.assert_array_equal(np.isnan(mag), np.isnan(g["cv_magnitudes"]))
    np.testing.assert_allclose(vec, g["cv_vectors"], rtol=CV_RTOL, atol=0)
    np.testing.assert_allclose(mag, g["cv_magnitudes"], rtol=CV_RTOL, atol=0)
    assert abs(mean - float(g["cv_mean"])) <= CV_RTOL * abs(float(g["cv_mean"]))


def test_lat_float32_ties_and_nan_follow_numpy(cuda_device):
    rng = np.random.default_rng(5)
    egm = rng.integers(-3, 4, size=(50, 70)).astype(np.float32)    # many ties
    egm[10, 5] = np.nan
    egm[20:, 6] = np.nan
    np.testing.assert_array_equal(analysis.compute_electrode_lat(egm), oracle_analysis.compute_electrode_lat(egm))


def test_cv_random_points_match_oracle(cuda_device):
    rng = np.random.default_rng(9)
    xyz = rng.uniform(0, 25, size=(500, 3))
    lat = np.linalg.norm(xyz - xyz[0], axis=1) / 0.7 + rng.normal(0, 0.5, 500)
    v, m, mean = analysis.conduction_velocity(xyz, lat)
    vo, mo, meano = oracle_analysis.conduction_velocity(xyz, lat)
    np.testing.assert_array_equal(np.isnan(m), np.isnan(mo))
    np.testing.assert_allclose(v, vo, rtol=CV_RTOL, atol=0)
    np.testing.assert_allclose(m, mo, rtol=CV_RTOL, atol=0)


def test_result_file_from_the_device_history(tmp_path, cuda_device):
    """Run an instance, compute its electrogram and electrode LAT on the device,
    stream the reference's result file from the device history, read it back."""
    from pyheartsim_b200 import instance, results
    from pyheartsim_b200.engine import BatchedEngine
    from pyheartsim_b200.simulation import unipolar_electrogram_gpu
    from tests import gpu_cases
    (n, P, geom, sp, ap), pdur = gpu_cases.small_shell_ms(t_phys=30.0)
    inst = instance.compile_instance(n, P, geom, dict(sp), dict(ap), full_cycles=False, tol=1e-7, restart=20,
                                     pacing_duration=pdur)
    eng = BatchedEngine()
    s = eng.add(inst)
    while not eng.finished(s):
        eng.advance(100)
    u, h = eng.history(s, with_h=True)
    ids = np.arange(0, n, 97)
    egm = unipolar_electrogram_gpu.compute(geom["voxel"][ids] + 1.5, geom["voxel"], None, P[:, 20], u.astype(np.float64),
                                           geom["Delta"], geom["neighbor_id_2d"])
    lat = analysis.compute_electrode_lat(egm)
    t = inst.sample_times(u.shape[0])
    path = results.save_simulation_results(tmp_path / "shell_simulation_results", eng, s, geometry_flag=1,
                                           electrogram=egm, save_all=True, physical_time=t, lat_electrode=lat,
                                           chunk=7)
    eng.close()
    f = np.load(path)
    assert f.files == ["geometry_flag", "electrogram_unipolar", "action_potential", "h", "physical_time",
                       "lat_electrode"]
    np.testing.assert_array_equal(f["action_potential"], u)
    np.testing.assert_array_equal(f["h"], h)
    np.testing.assert_array_equal(f["electrogram_unipolar"], egm)
    np.testing.assert_array_equal(f["lat_electrode"], lat)
    np.testing.assert_array_equal(f["physical_time"], t)


INTERP_ATOL = 1e-12   # barycentric sums: the same operations as scipy, a different simplex on shared facets


@pytest.mark.parametrize("k", range(4))
def test_interpolate_lat_matches_reference(k, cuda_device):
    """utility/lat_map.py:29-46 on the device against the reference's own
    interpolate_lat: 3-D shell, flat sheet (constant z dropped), sparse 3-D
    points, and a 4 x 4 electrode grid above a sheet (nearest fallback on the
    border)."""
    name, vox, el, lat_e, lat_v = golden_cases.interp_cases()[k]
    out = analysis.interpolate_lat(vox, el, lat_e)
    assert out.dtype == np.float64 and out.shape == lat_v.shape
    np.testing.assert_array_equal(np.isnan(out), np.isnan(lat_v))
    np.testing.assert_allclose(out, lat_v, rtol=0, atol=INTERP_ATOL)


def test_interpolate_lat_random_3d_matches_oracle(cuda_device):
    rng = np.random.default_rng(21)
    el = rng.uniform(0, 20, size=(300, 3))
    vox = rng.uniform(-2, 22, size=(20000, 3))
    lat = rng.uniform(0, 80, size=300)
    out = analysis.interpolate_lat(vox, el, lat)
    ref = oracle_analysis.interpolate_lat(vox, el, lat)
    np.testing.assert_array_equal(np.isnan(out), np.isnan(ref))
    np.testing.assert_allclose(out, ref, rtol=0, atol=INTERP_ATOL)
