"""The analysis oracle (electrode LAT, conduction velocity) against the
reference's own outputs (tests/golden/analysis_*.npz)."""
import numpy as np
import pytest

from oracle import analysis
from tests import golden_cases


@pytest.mark.parametrize("name", golden_cases.analysis_names())
def test_oracle_matches_reference_analysis(name):
    g = np.load(f"{golden_cases.GOLDEN}/{name}.npz")
    lat = analysis.compute_electrode_lat(g["egm"])
    np.testing.assert_array_equal(lat, g["lat_electrode"])
    vec, mag, mean = analysis.compute({"electrogram_unipolar": g["egm"]},
                                      {"voxel": g["voxel"], "voxel_id_of_simulation_electrode": g["electrode_ids"]})
    np.testing.assert_array_equal(np.isnan(mag), np.isnan(g["cv_magnitudes"]))
    np.testing.assert_allclose(vec, g["cv_vectors"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(mag, g["cv_magnitudes"], rtol=1e-12, atol=0)
    assert abs(mean - float(g["cv_mean"])) <= 1e-12 * abs(float(g["cv_mean"]))


@pytest.mark.parametrize("k", range(4))
def test_oracle_interpolate_lat_matches_reference(k):
    name, vox, el, lat_e, lat_v = golden_cases.interp_cases()[k]
    out = analysis.interpolate_lat(vox, el, lat_e)
    np.testing.assert_array_equal(np.isnan(out), np.isnan(lat_v))
    np.testing.assert_array_equal(out, lat_v)          # same scipy routines: bit-exact
