"""Device geometry (neighbour table, P_2d, operator tables) against the
reference's own outputs (golden fixtures) and the host compilation."""
import numpy as np
import pytest

from pyheartsim_b200 import _lib, geometry, geometry_gpu, instance, synthetic
from pyheartsim_b200.engine import BatchedEngine
from tests import golden_cases, gpu_cases

pytestmark = pytest.mark.gpu

MS_KEYS = ("tau_open_voxel", "tau_close_voxel", "tau_in_voxel", "tau_out_voxel", "v_gate_voxel")
AP_KEYS = ("k_voxel", "a_voxel", "epsilon_0_voxel", "mu1_voxel", "mu2_voxel")


def parameter_of(P, model):
    """The reference's per-voxel parameter dict behind P_2d columns 15..20."""
    keys = MS_KEYS if model == 0 else AP_KEYS
    par = {k: P[:, 15 + i].copy() for i, k in enumerate(keys)}
    par["c_voxel"] = P[:, 20].copy()
    return par


def d0_of(g):
    return g["D0"] if "D0" in g.files else None


@pytest.mark.parametrize("name", golden_cases.names())
def test_neighbour_table_equals_reference(name, cuda_device):
    g = golden_cases.load(name)["g"]
    nb = geometry_gpu.find_neighbor_voxel_ids(g["ijk"])
    np.testing.assert_array_equal(nb, g["neighbor_id_2d"])     # utility/voxelization.py:102-152


@pytest.mark.parametrize("name", golden_cases.names())
def test_equation_parts_bit_identical_to_reference(name, cuda_device):
    c = golden_cases.load(name)
    g = c["g"]
    P = geometry_gpu.heart_model_equation_parts(c["sp"], c["n"], d0_of(g), g["neighbor_id_2d"],
                                                parameter_of(g["P_2d"], c["sp"]["heart_model_flag"]))
    assert P.dtype == np.float64
    np.testing.assert_array_equal(P, g["P_2d"])                # simulation/equation_parts.py:36-114


def _cases():
    out = []
    for name in golden_cases.names():
        c = golden_cases.load(name)
        out.append((name, c["g"]["voxel"], c["geom"]["Delta"], c["P_2d"], d0_of(c["g"]), c["sp"], c["ap"], None))
    for case in ("small_shell_ms", "small_shell_ms_fibres", "slab_ap"):
        (n, P, geom, sp, ap), pdur = getattr(gpu_cases, case)()
        D0 = synthetic.fibre_tensors(np.rint(geom["voxel"] / geom["Delta"])) if case.endswith("fibres") else None
        out.append((case, geom["voxel"], geom["Delta"], P, D0, sp, ap, pdur))
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_device_tables_equal_host_compilation(case, cuda_device):
    name, voxel, Delta, P, D0, sp, ap, pdur = case
    n = voxel.shape[0]
    model = sp["heart_model_flag"]
    kw = dict(full_cycles=False, tol=1e-7, restart=20, pacing_duration=pdur)
    nb = geometry.lattice_neighbors(np.rint(voxel / Delta))
    host = instance.compile_instance(n, P, {"neighbor_id_2d": nb, "Delta": Delta, "voxel": voxel}, dict(sp),
                                     dict(ap), **kw)
    dev = geometry_gpu.compile_instance(voxel, Delta, parameter_of(P, model), D0, dict(sp), dict(ap), **kw)
    t = dev.host_tables()
    if host.order is None:
        assert dev.order is None
    else:
        np.testing.assert_array_equal(dev.order, host.order)
        np.testing.assert_array_equal(dev.inv, host.inv)
    np.testing.assert_array_equal(t["nb6"], host.nb6)
    np.testing.assert_array_equal(t["coef6"], host.coef6)
    np.testing.assert_array_equal(t["vflags"], host.vflags)
    assert (dev.cw is None) == (host.cw is None)
    if host.cw is not None:
        np.testing.assert_array_equal(t["cw"], host.cw)
        np.testing.assert_array_equal(t["mask6"], host.mask6)
    assert (dev.vparams is None) == (host.vparams is None)
    if host.vparams is not None:
        np.testing.assert_array_equal(t["vparams"], host.vparams)
    assert (dev.coef_edge is None) == (host.coef_edge is None)
    if host.coef_edge is not None:
        np.testing.assert_array_equal(t["nb_edge"], host.nb_edge)
        np.testing.assert_array_equal(t["coef_edge"], host.coef_edge)
    np.testing.assert_array_equal(dev.params, host.params)
    for k in ("n_steps", "n_samples", "sample_stride", "tblock_steps", "dt", "j_stim", "guess", "restart"):
        assert getattr(dev, k) == getattr(host, k), k
    np.testing.assert_array_equal(dev.stim, host.stim)


@pytest.mark.parametrize("case", ["small_shell_ms", "small_shell_ms_fibres"])
def test_device_built_instance_runs_like_the_host_built_one(case, cuda_device):
    (n, P, geom, sp, ap), pdur = getattr(gpu_cases, case)(t_phys=15.0) if case == "small_shell_ms" else \
        gpu_cases.small_shell_ms(t_phys=15.0, fibres=True)
    D0 = synthetic.fibre_tensors(np.rint(geom["voxel"] / geom["Delta"])) if case.endswith("fibres") else None
    kw = dict(full_cycles=False, tol=1e-7, restart=20, pacing_duration=pdur)
    host = instance.compile_instance(n, P, geom, dict(sp), dict(ap), **kw)
    dev = geometry_gpu.compile_instance(geom["voxel"], geom["Delta"], parameter_of(P, sp["heart_model_flag"]), D0,
                                        dict(sp), dict(ap), **kw)
    hist = []
    for inst in (host, dev):
        eng = BatchedEngine()
        s = eng.add(inst)
        while not eng.finished(s):
            eng.advance(50)
        hist.append(eng.history(s))
        eng.close()
    assert np.abs(hist[0]).max() > 0.5
    np.testing.assert_array_equal(hist[1], hist[0])


def test_duplicate_coordinates_rejected(cuda_device):
    ijk = np.array([[0, 0, 0], [1, 0, 0], [0, 0, 0]], dtype=np.int32)
    with pytest.raises(_lib.PhsError):
        geometry_gpu.lattice_neighbors(ijk)


def test_row_order_matches_host_locality_order(cuda_device):
    ijk = synthetic.shell((7.0, 6.0, 5.0), 0.4, 2, 1, 1.5, 3)
    rng = np.random.default_rng(0)
    perm = rng.permutation(ijk.shape[0])
    ijk = ijk[perm]                                  # scrambled caller order
    nb18, order = geometry_gpu.lattice_neighbors(ijk)
    host = instance.locality_order({"voxel": ijk * 0.4, "Delta": 0.4}, ijk.shape[0], "rows")
    np.testing.assert_array_equal(order.cpu().numpy(), host)
    np.testing.assert_array_equal(nb18.cpu().numpy(), geometry.lattice_neighbors(ijk))


def test_device_built_workload_instance_equals_host_built(cuda_device):
    """The serving / benchmark shell builder on the device gives the host
    builder's instance (same geometry, scar, pacing and tables)."""
    from pyheartsim_b200 import workloads
    host, _, _ = workloads.shell_case(3, 30_000, 2, t_phys=50.0, tol=1e-7)
    dev, meta = workloads.shell_case_device(3, 30_000, 2, t_phys=50.0, tol=1e-7)
    t = dev.host_tables()
    np.testing.assert_array_equal(dev.order, host.order)
    np.testing.assert_array_equal(t["nb6"], host.nb6)
    np.testing.assert_array_equal(t["coef6"], host.coef6)
    np.testing.assert_array_equal(t["vflags"], host.vflags)
    assert (dev.cw is None) == (host.cw is None)
    if host.cw is not None:
        np.testing.assert_array_equal(t["cw"], host.cw)
    np.testing.assert_array_equal(dev.stim, host.stim)
    assert dev.n_steps == host.n_steps and dev.model == host.model
