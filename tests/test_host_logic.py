"""Host-side compilation of the reference's inputs, checked against the oracle
(no GPU)."""
import numpy as np
import pytest

from oracle import egm_fp64, simulation_fp64
from pyheartsim_b200 import instance
from pyheartsim_b200.simulation import pacing, unipolar_electrogram_gpu
from tests import golden_cases


def _ref_windows(ap, sp, flag, n_steps, dt, s1_t, pdur, s2_t):
    out = np.zeros(n_steps, dtype=np.uint8)
    for k in range(n_steps):
        a, b = simulation_fp64.pacing_windows(ap, sp, flag, k * dt, s1_t, pdur, s2_t)
        out[k] = (1 if a else 0) | (2 if b else 0)
    return out


@pytest.mark.parametrize("flag", [0, 1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("model", [0, 1])
def test_pacing_schedule_matches_reference_windows(flag, model):
    ts = 1 if model == 0 else 6
    sp = {"heart_model_flag": model, "time_scale": ts, "dt": 0.05 / ts, "t_final": 400 / ts}
    ap = {"pacing_start_time": 10 / ts, "pacing_cycle_length": 37.3 / ts, "s1_t": 3.0 / ts,
          "s1_s2_delta_t": 41.7 / ts, "s1_pacing_voxel_id": [0], "s2_pacing_voxel_id": [1]}
    s1, s2, s1_t, jm, pdur, s2_t = pacing.assign_pacing_parameters(ap, flag, sp)
    n = 8000
    got = pacing.schedule(n, sp["dt"], ap, sp, flag, s1_t, pdur, s2_t)
    want = _ref_windows(ap, sp, flag, n, sp["dt"], s1_t, pdur, s2_t)
    np.testing.assert_array_equal(got, want)


def test_zero_cycle_length_raises_instead_of_hanging():
    sp = {"heart_model_flag": 0, "time_scale": 1}
    ap = {"pacing_start_time": 0.0, "pacing_cycle_length": 0.0}
    with pytest.raises(ValueError):
        pacing.schedule(100, 0.5, ap, sp, 0, 0.0, 5, 0.0)


@pytest.mark.parametrize("t_final,dt,model", [(500, 0.05, 0), (1000 / 6, 0.02 / 6, 1), (12, 0.7, 0), (3, 2.0, 0)])
def test_step_counts_match_reference(t_final, dt, model):
    sp = {"t_final": t_final, "dt": dt, "heart_model_flag": model, "time_scale": 1 if model == 0 else 6}
    assert instance.step_counts(sp) == simulation_fp64.step_schedule(sp)


@pytest.mark.parametrize("name", golden_cases.names())
def test_matrix_free_operator_equals_reference_csr(name):
    c = golden_cases.load(name)
    inst = instance.compile_instance(c["n"], c["P_2d"], c["geom"], c["sp"], c["ap"], reorder=False)
    P = np.array(c["P_2d"], dtype=np.float64)
    nf = np.asarray(c["ap"]["node_flag"])
    P[nf == 4, 20] = 0.0
    L = simulation_fp64.laplacian(P, c["geom"]["neighbor_id_2d"], c["geom"]["Delta"])
    rng = np.random.default_rng(0)
    for _ in range(3):
        u = rng.standard_normal(c["n"])
        np.testing.assert_allclose(_table_laplacian(inst, u), L @ u, rtol=1e-12, atol=1e-12)
    # temporary block rows
    tb = (inst.vflags & 4) != 0
    np.testing.assert_array_equal(tb, nf == 3)


def test_incoming_gradient_terms_reproduce_leadfield():
    c = golden_cases.load("slab_ap_flag1")
    g = c["g"]
    nb = g["neighbor_id_2d"]
    el = g["egm_electrode_xyz"]
    M_ref = egm_fp64.leadfield(el, g["voxel"], None, g["P_2d"][:, 20], float(g["Delta"]), nb)
    ptr, src, dirs = unipolar_electrogram_gpu.incoming_gradient_terms(nb)
    # numpy emulation of the gather the device kernel performs
    n_v, n_e = g["voxel"].shape[0], el.shape[0]
    M = np.zeros((n_v, n_e))
    for w in range(n_v):
        for q in range(ptr[w], ptr[w + 1]):
            v, dd = src[q], dirs[q]
            d = abs(dd) - 1
            l = g["voxel"][v] - el
            ln = np.maximum(np.linalg.norm(l, axis=1), 1.0)
            gval = g["P_2d"][v, 20] / ln ** 3 * l[:, d] / (2 * float(g["Delta"]))
            M[w] += gval if dd > 0 else -gval
    np.testing.assert_allclose(M, M_ref, rtol=1e-12, atol=1e-14)


def test_compile_rejects_bad_tables():
    c = golden_cases.load("sheet_ms_flag4")
    geom = dict(c["geom"])
    nb = geom["neighbor_id_2d"].copy()
    nb[3, 0] = c["n"] + 5
    geom["neighbor_id_2d"] = nb
    with pytest.raises(ValueError):
        instance.compile_instance(c["n"], c["P_2d"], geom, c["sp"], c["ap"])
    P = c["P_2d"].copy()
    P[0, 9] = 0.5
    geom = dict(c["geom"])
    nb = geom["neighbor_id_2d"].copy()
    nb[2, 7] = c["n"]
    geom["neighbor_id_2d"] = nb
    with pytest.raises(ValueError):                      # edge neighbours are checked when used
        instance.compile_instance(c["n"], P, geom, c["sp"], c["ap"])


def _table_laplacian(inst, u_caller):
    """The operator the device applies, from the compiled tables (caller order)."""
    u = u_caller if inst.order is None else u_caller[inst.order]
    lap = (inst.coef6 * (u[inst.nb6] - u[:, None])).sum(axis=1)
    if inst.coef_edge is not None:
        e = inst.nb_edge
        lap = lap + (inst.coef_edge * (u[e[:, 0::2]] - u[e[:, 1::2]])).sum(axis=1)
    return inst.to_caller(lap)


@pytest.mark.parametrize("reorder", [False, "rows", "morton"])
def test_anisotropic_tables_reproduce_reference_laplacian(reorder):
    """Fibre case (D0 != I, every cross term present): face cross terms folded
    into coef6 plus six edge pairs give the reference's CSR L
    (simulation_gpu.py:138-225, restated by the oracle) row for row."""
    c = golden_cases.load("slab_ms_fibres")
    P = c["P_2d"]
    assert np.abs(P[:, 6:9]).max() > 0.1 and np.abs(P[:, 9:15]).max() > 0.1
    inst = instance.compile_instance(c["n"], P, c["geom"], c["sp"], c["ap"], reorder=reorder)
    assert inst.coef_edge is not None and inst.cw is None
    Pc = P.copy()
    Pc[c["ap"]["node_flag"] == 4, 20] = 0.0                 # permanent block, simulation_gpu.py:312-313
    L = simulation_fp64.laplacian(Pc, c["geom"]["neighbor_id_2d"], c["geom"]["Delta"])
    rng = np.random.default_rng(3)
    for _ in range(3):
        u = rng.standard_normal(c["n"])
        np.testing.assert_allclose(_table_laplacian(inst, u), L @ u, rtol=0, atol=1e-12)
    # isotropic case: no edge tables, same operator
    c0 = golden_cases.load("slab_ap_flag1")
    i0 = instance.compile_instance(c0["n"], c0["P_2d"], c0["geom"], c0["sp"], c0["ap"], reorder=reorder)
    assert i0.coef_edge is None and i0.nb_edge is None


@pytest.mark.parametrize("name", golden_cases.names())
def test_lattice_neighbors_and_P2d_match_reference(name):
    from pyheartsim_b200 import geometry
    c = golden_cases.load(name)
    g = c["g"]
    nb = geometry.lattice_neighbors(g["ijk"])
    np.testing.assert_array_equal(nb, g["neighbor_id_2d"])     # utility/voxelization.py convention
    n = c["n"]
    par = {"c_voxel": g["P_2d"][:, 20]}
    keys = (("tau_open_voxel", "tau_close_voxel", "tau_in_voxel", "tau_out_voxel", "v_gate_voxel")
            if c["sp"]["heart_model_flag"] == 0 else
            ("k_voxel", "a_voxel", "epsilon_0_voxel", "mu1_voxel", "mu2_voxel"))
    for col, k in zip(range(15, 20), keys):
        par[k] = g["P_2d"][:, col]
    D0 = list(g["D0"]) if "D0" in g.files else geometry.load_fiber(n)
    P = geometry.heart_model_equation_parts(c["sp"], n, D0, nb, par)
    np.testing.assert_array_equal(P, g["P_2d"])


def test_shell_generator_is_seeded_and_sized():
    from pyheartsim_b200 import synthetic
    a = synthetic.shell(seed=0)
    b = synthetic.shell(seed=0)
    np.testing.assert_array_equal(a, b)
    assert 60_000 < a.shape[0] < 130_000
    nb = synthetic.lattice_neighbors(a) if hasattr(synthetic, "lattice_neighbors") else None
    assert nb is not None and nb.shape == (a.shape[0], 18)


def test_reorder_preserves_the_operator():
    from pyheartsim_b200 import synthetic
    ijk = synthetic.shell((6.0, 5.0, 4.0), 0.4, 2, 1, 1.5, 0)
    s1 = np.arange(5)
    n, P, geom, sp, ap = synthetic.make_case(ijk, 0.4, 0, 0.05, 5.0, s1, flag=4)
    a = instance.compile_instance(n, P, geom, sp, ap, reorder=False)
    b = instance.compile_instance(n, P, geom, sp, ap, reorder="morton")
    assert b.order is not None and not np.array_equal(b.order, np.arange(n))
    rng = np.random.default_rng(1)
    u = rng.standard_normal(n)
    lap_a = (a.coef6 * (u[a.nb6] - u[:, None])).sum(axis=1)
    ub = u[b.order]                                       # device order
    lap_b = (b.coef6 * (ub[b.nb6] - ub[:, None])).sum(axis=1)
    np.testing.assert_allclose(b.to_caller(lap_b), lap_a, rtol=1e-13, atol=1e-13)
    np.testing.assert_array_equal(b.to_caller(b.vflags), a.vflags)
    # tiles of 1024 device-ordered voxels keep most neighbours inside
    tile = np.arange(n) // 1024
    out = (b.coef6 != 0) & (b.nb6 // 1024 != tile[:, None])
    assert out.sum() / n < 1.0


def test_byte_model_closed_forms():
    """The roofline byte model per voxel-step in FP32 with isotropic rows:
    71 + 49 k + 4 k^2 with the int32 neighbour table, 55 + 33 k + 4 k^2 (plus
    the per-block bases, 1/32 byte per row and operator application) with the
    compact one."""
    from pyheartsim_b200 import roofline
    for k in (0, 1, 2, 3, 7):
        assert roofline.per_voxel_step(4, k) == 71 + 49 * k + 4 * k * k
        compact = roofline.per_voxel_step(4, k, nb=roofline.COMPACT_NB)
        assert abs(compact - (55 + 33 * k + 4 * k * k + (1 + k) / 32)) < 1e-9
