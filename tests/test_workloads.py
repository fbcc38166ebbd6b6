"""Host-side workload generators and the accuracy bookkeeping (no GPU)."""
import numpy as np

from pyheartsim_b200 import accuracy, synthetic, workloads
from pyheartsim_b200.geometry import lattice_neighbors


def test_scar_ring_from_grid_equals_neighbour_table():
    ijk = workloads._shell_scaled(60_000, 5)
    nb = lattice_neighbors(ijk)
    a = synthetic.scar(ijk, nb, 0.2, np.random.default_rng(3))
    b = synthetic.scar(ijk, None, 0.2, np.random.default_rng(3))
    np.testing.assert_array_equal(a, b)
    assert (a == 0.1).any() and (a == 0.0).any()


def test_payload_matches_reference_style_inputs():
    """A serving request's payload describes the same geometry, scar and pacing
    as the reference-style inputs of the same shell (both models)."""
    for i in (4, 5):
        pl = workloads.shell_payload(i, 40_000, 0, t_phys=30.0)
        (n, P, geom, sp, ap), meta = workloads.shell_inputs(i, 40_000, 0, t_phys=30.0)
        assert pl["meta"] == meta
        np.testing.assert_array_equal(pl["voxel"], geom["voxel"])
        np.testing.assert_array_equal(pl["parameter"]["c_voxel"], P[:, 20])
        np.testing.assert_array_equal(pl["ap"]["s1_pacing_voxel_id"], ap["s1_pacing_voxel_id"])
        assert pl["sp"] == sp


def test_focal_stimulus_per_model():
    """Mitchell-Schaeffer sites are 3-voxel balls paced 2 ms, Aliev-Panfilov
    sites 8-voxel balls paced 5 ms (smaller ones never reach threshold)."""
    (_, _, _, _, ap0), m0 = workloads.shell_inputs(0, 60_000, 0, t_phys=10.0)
    (_, _, _, _, ap1), m1 = workloads.shell_inputs(1, 60_000, 0, t_phys=10.0)
    assert (m0["model"], m0["pacing_ms"]) == (0, 2.0)
    assert (m1["model"], m1["pacing_ms"]) == (1, 5.0)
    assert len(ap1["s1_pacing_voxel_id"]) > 4 * len(ap0["s1_pacing_voxel_id"])


def test_named_configurations():
    (n, P, geom, sp, ap), pdur, el = workloads.sheet_c1()
    assert n == 40_000 and pdur == 1.0 and el.shape == (16, 3) and np.all(el[:, 2] == 1.0)
    assert round(sp['t_final'] / sp['dt']) == 10_000
    (n3, P3, g3, sp3, ap3), pd3, el3 = workloads.atrium_c2(wall=3)
    assert n3 == 91_292 and pd3 is None and el3.shape == (64, 3)
    assert round(sp3['t_final'] / sp3['dt']) == 50_000 and sp3['time_scale'] == 6
    assert ap3['s1_s2_delta_t'] * 6 == workloads.C2_PACING[3][1]
    (n8, _, _, _, ap8), _, _ = workloads.atrium_c2(wall=8)
    assert n8 == 218_403
    assert len(ap8['s1_pacing_voxel_id']) > len(ap3['s1_pacing_voxel_id'])   # deeper S1 cap


def test_compare_activations_counts_and_errors():
    K = accuracy.MAX_ACTIVATIONS
    t_ref = np.full((4, K), -1, np.int32)
    t_tst = np.full((4, K), -1, np.int32)
    t_ref[0, :3] = [10, 200, 400]
    t_tst[0, :3] = [11, 199, 402]
    t_ref[1, :1] = [50]
    t_tst[1, :2] = [50, 300]          # an extra re-activation in the test run
    ref = {"times": t_ref, "counts": np.array([3, 1, 0, 0])}
    tst = {"times": t_tst, "counts": np.array([3, 2, 0, 0])}
    r = accuracy.compare_activations(ref, tst)
    assert r["first"]["max_dlat_steps"] == 1 and r["first"]["voxels_both"] == 2
    assert r["reactivations"][0]["voxels_one_run_only"] == 1
    assert r["reactivations"][0]["max_dlat_steps"] == 1
    assert r["reactivations"][1]["max_dlat_steps"] == 2
    assert r["activation_count_equal_frac"] == 0.75
