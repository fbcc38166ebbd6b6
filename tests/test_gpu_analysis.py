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
