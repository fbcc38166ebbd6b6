"""Generate the golden fixtures in ``tests/golden/*.npz`` by running the
reference's OWN, unmodified code in this container.

Test infrastructure only.  Needs a checkout of the reference, named by the
environment variable ``PHS_REFERENCE_DIR``; it exists only where the fixtures
are generated, the fixtures themselves are committed and nothing at test time
reads the reference.

How the reference runs without CuPy or a GPU:

* ``NUMBA_ENABLE_CUDASIM=1`` makes Numba execute the ``@cuda.jit`` kernels
  (simulation/simulation_gpu.py:71-130, simulation/unipolar_electrogram_gpu.py:21-69)
  on the CPU;
* ``cupy_standin.py`` is installed as ``cupy``, ``cupyx.scipy.sparse`` and
  ``cupyx.scipy.sparse.linalg``; its GMRES restates CuPy's documented
  full-cycle GMRES(restart) (called at simulation/simulation_gpu.py:253);
* ``numba.cuda.as_cuda_array`` becomes the identity (simulation_gpu.py:347-352);
* for the FP64 runs the module-global ``np`` of the two reference modules is
  replaced by a proxy whose ``float32`` is ``float64`` (and likewise the
  stand-in's ``float32``), so the reference's own code computes in FP64.

The neighbour tables come from the reference's own
``utility/voxelization.py::find_neighbor_voxel_ids`` (KDTree on integer
coordinates), loaded with stub modules for its plotting imports.

Run:  PHS_REFERENCE_DIR=<reference checkout> python tests/golden/make_golden.py   (a few minutes)
"""
import importlib.util
import os
import sys
import time
import types

os.environ["NUMBA_ENABLE_CUDASIM"] = "1"

import numpy as np  # noqa: E402

REF = os.environ.get("PHS_REFERENCE_DIR", "")
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import cupy_standin  # noqa: E402


def _install_cupy_standin():
    cp = types.ModuleType("cupy")
    for k in ("float32", "float64", "int32", "zeros", "asarray", "array", "asnumpy"):
        setattr(cp, k, getattr(cupy_standin, k))
    cpx = types.ModuleType("cupyx")
    cpx_scipy = types.ModuleType("cupyx.scipy")
    cpx_sparse = types.ModuleType("cupyx.scipy.sparse")
    cpx_sparse.coo_matrix = cupy_standin.sparse.coo_matrix
    cpx_sparse.identity = cupy_standin.sparse.identity
    cpx_linalg = types.ModuleType("cupyx.scipy.sparse.linalg")
    cpx_linalg.gmres = cupy_standin.gmres
    cpx_linalg.cg = cupy_standin.cg
    cpx.scipy = cpx_scipy
    cpx_scipy.sparse = cpx_sparse
    cpx_sparse.linalg = cpx_linalg
    sys.modules.update({"cupy": cp, "cupyx": cpx, "cupyx.scipy": cpx_scipy,
                        "cupyx.scipy.sparse": cpx_sparse,
                        "cupyx.scipy.sparse.linalg": cpx_linalg})
    return cp


class _NP64:
    """numpy with float32 mapped to float64 (FP64 run of the reference)."""

    def __getattr__(self, k):
        if k == "float32":
            return np.float64
        return getattr(np, k)


def _load_reference():
    cp = _install_cupy_standin()
    from numba import cuda
    cuda.as_cuda_array = lambda x: x
    sys.path.insert(0, REF)
    import simulation  # noqa: F401  (the reference package)
    # utility/voxelization.py: stub its plotting and package imports
    for name in ("plotly", "plotly.graph_objects", "plotly.io"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["plotly.io"].renderers = types.SimpleNamespace(default=None)
    sys.modules.setdefault("utility", types.ModuleType("utility"))
    spec = importlib.util.spec_from_file_location(
        "ref_voxelization", os.path.join(REF, "utility", "voxelization.py"))
    vox = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(vox)
    return cp, simulation, vox


def _set_precision(cp, simulation, fp64):
    sg = simulation.simulation_gpu
    eg = simulation.unipolar_electrogram_gpu
    if not hasattr(sg, "_orig_np"):
        sg._orig_np, eg._orig_np = sg.np, eg.np
    if fp64:
        sg.np = _NP64()
        eg.np = _NP64()
        cp.float32 = np.float64
    else:
        sg.np, eg.np = sg._orig_np, eg._orig_np
        cp.float32 = np.float32


def lattice(shape):
    """Integer lattice coordinates in the reference's create_geometry order
    (x outermost, z innermost; tool/create_geometry.py:76-82)."""
    idx = np.indices(shape).reshape(len(shape), -1).T.astype(np.float64)
    if idx.shape[1] == 2:
        idx = np.concatenate([idx, np.zeros((idx.shape[0], 1))], axis=1)
    return idx


MS = dict(tau_in=0.3, tau_out=6.0, tau_open=120.0, tau_close=150.0, v_gate=0.13)
AP = dict(k=8.0, a=0.15, epsilon_0=0.002, mu1=0.2, mu2=0.3)


def fibre_D0(ijk, r=0.3):
    """Anisotropic tensors D0 = r I + (1-r) e e^T with a smoothly rotating fibre
    direction e (the fiber_flag == 1 form of simulation/equation_parts.py:28-29)."""
    th = 0.35 * ijk[:, 0] + 0.2 * ijk[:, 2]
    ph = 0.25 * ijk[:, 1]
    e = np.stack([np.cos(th) * np.cos(ph), np.sin(th) * np.cos(ph), np.sin(ph)], axis=1)
    return [r * np.eye(3) + (1 - r) * np.outer(v, v) for v in e]


def build_case(simulation, vox, name, shape, model, dt_phys, t_phys, flag, s1_pred,
               s2_pred=None, s1_t=0.0, s1_s2=0.0, start=10.0, cycle=300.0,
               node_flag_fn=None, c_base=None, Delta=0.4, fibres=False):
    ijk = lattice(shape)
    n = ijk.shape[0]
    nb = vox.find_neighbor_voxel_ids(ijk)
    voxel = ijk * Delta
    ts = 1 if model == 0 else 6
    sp = {"t_final": t_phys / ts, "dt": dt_phys / ts, "heart_model_flag": model,
          "arrhythmia_flag": flag, "time_scale": ts}
    s1 = np.where(s1_pred(ijk))[0]
    s2 = np.where(s2_pred(ijk))[0] if s2_pred is not None else []
    node_flag = np.zeros(n, dtype=np.int64) if node_flag_fn is None else node_flag_fn(ijk)
    ap = {"pacing_start_time": start / ts, "pacing_cycle_length": cycle / ts,
          "s1_pacing_voxel_id": s1, "s2_pacing_voxel_id": s2, "s1_t": s1_t / ts,
          "s1_s2_delta_t": s1_s2 / ts, "node_flag": node_flag}
    if model == 0:
        par = {"tau_in_voxel": np.full(n, MS["tau_in"]), "tau_out_voxel": np.full(n, MS["tau_out"]),
               "tau_open_voxel": np.full(n, MS["tau_open"]), "tau_close_voxel": np.full(n, MS["tau_close"]),
               "v_gate_voxel": np.full(n, MS["v_gate"]),
               "c_voxel": np.full(n, 1.0 if c_base is None else c_base)}
    else:
        par = {"k_voxel": np.full(n, AP["k"]), "a_voxel": np.full(n, AP["a"]),
               "epsilon_0_voxel": np.full(n, AP["epsilon_0"]), "mu1_voxel": np.full(n, AP["mu1"]),
               "mu2_voxel": np.full(n, AP["mu2"]),
               "c_voxel": np.full(n, (1.6 if c_base is None else c_base) * ts)}
    D0 = fibre_D0(ijk) if fibres else simulation.equation_parts.load_fiber(n)
    P = simulation.equation_parts.heart_model_equation_parts(sp, n, D0, nb, par)
    return dict(name=name, ijk=ijk, voxel=voxel, nb=nb, Delta=Delta, sp=sp, ap=ap, par=par, P=P, D0=D0)


def run_sim(cp, simulation, case, fp64):
    _set_precision(cp, simulation, fp64)
    geom = {"neighbor_id_2d": case["nb"], "Delta": case["Delta"]}
    t0 = time.time()
    u, h, t = simulation.simulation_gpu.compute(case["voxel"].shape[0], case["P"], geom,
                                                dict(case["sp"]), dict(case["ap"]))
    print(f"  {case['name']} fp64={fp64}: {u.shape} in {time.time() - t0:.1f}s", flush=True)
    return u, h, t


def run_egm(cp, simulation, case, u_hist, electrode_xyz, fp64):
    _set_precision(cp, simulation, fp64)
    egm = simulation.unipolar_electrogram_gpu.compute(
        electrode_xyz, case["voxel"], case["D0"], case["par"]["c_voxel"], u_hist,
        case["Delta"], case["nb"])
    return egm


def _pack(prefix, d):
    return {f"{prefix}{k}": np.asarray(v) for k, v in d.items()}


def main():
    if not REF or not os.path.isdir(os.path.join(REF, "simulation")):
        raise SystemExit("set PHS_REFERENCE_DIR to a checkout of the reference")
    cp, simulation, vox = _load_reference()
    import io
    import contextlib
    cases = [
        dict(name="sheet_ms_flag4", shape=(14, 14), model=0, dt_phys=0.05, t_phys=12.0, flag=4,
             s1_pred=lambda x: (x[:, 0] < 3) & (x[:, 1] < 3)),
        dict(name="sheet_ms_blocks", shape=(12, 12), model=0, dt_phys=0.1, t_phys=40.0, flag=4,
             s1_pred=lambda x: (x[:, 0] < 2) & (x[:, 1] < 12),
             node_flag_fn=lambda x: np.where((x[:, 0] == 6) & (x[:, 1] < 8), 4,
                                             np.where((x[:, 0] == 3) & (x[:, 1] >= 6), 3, 0))),
        dict(name="sheet_ms_flag0", shape=(10, 10), model=0, dt_phys=0.1, t_phys=12.0, flag=0,
             s1_pred=lambda x: (x[:, 0] == 0) & (x[:, 1] == 0), start=1.0, cycle=4.0),
        dict(name="slab_ap_flag1", shape=(7, 7, 4), model=1, dt_phys=0.1, t_phys=30.0, flag=1,
             s1_pred=lambda x: x[:, 0] == 0, s2_pred=lambda x: (x[:, 0] < 3) & (x[:, 1] > 3),
             s1_s2=15.0),
        dict(name="slab_ap_flag3", shape=(6, 5, 3), model=1, dt_phys=0.2, t_phys=8.0, flag=3,
             s1_pred=lambda x: x[:, 1] == 0, s2_pred=lambda x: x[:, 2] == 2, s1_s2=2.0),
        dict(name="sheet_ap_flag6", shape=(9, 9), model=1, dt_phys=0.2, t_phys=60.0, flag=6,
             s1_pred=lambda x: (x[:, 0] < 3) & (x[:, 1] < 3),
             s2_pred=lambda x: (x[:, 0] > 5) & (x[:, 1] > 5)),
        dict(name="sheet_ms_flag5", shape=(8, 8), model=0, dt_phys=0.5, t_phys=305.0, flag=5,
             s1_pred=lambda x: x[:, 0] == 0, s2_pred=lambda x: x[:, 0] == 7),
        dict(name="slab_ms_fibres", shape=(7, 6, 4), model=0, dt_phys=0.1, t_phys=12.0, flag=4,
             s1_pred=lambda x: (x[:, 0] < 2) & (x[:, 1] < 2), fibres=True,
             node_flag_fn=lambda x: np.where((x[:, 0] == 4) & (x[:, 1] == 3), 4, 0)),
    ]
    only = set(sys.argv[1:])
    if only:
        cases = [c for c in cases if c["name"] in only]
    out = {}
    for spec in cases:
        case = build_case(simulation, vox, **spec)
        name = case["name"]
        rec = {"ijk": case["ijk"], "voxel": case["voxel"], "neighbor_id_2d": case["nb"],
               "D0": np.asarray(case["D0"], dtype=np.float64),
               "Delta": case["Delta"], "P_2d": case["P"],
               "s1": case["ap"]["s1_pacing_voxel_id"],
               "s2": np.asarray(case["ap"]["s2_pacing_voxel_id"], dtype=np.int64),
               "node_flag": case["ap"]["node_flag"]}
        for k, v in case["sp"].items():
            rec[f"sp_{k}"] = v
        for k in ("pacing_start_time", "pacing_cycle_length", "s1_t", "s1_s2_delta_t"):
            rec[f"ap_{k}"] = case["ap"][k]
        with contextlib.redirect_stdout(io.StringIO()):
            u32, h32, t32 = run_sim(cp, simulation, case, fp64=False)
            u64, h64, t64 = run_sim(cp, simulation, case, fp64=True)
        print(f"  {name}: S={u64.shape[0]} max u={u64.max():.3f}", flush=True)
        rec.update(u_f32=u32, h_f32=h32, t_f32=t32, u_f64=u64, h_f64=h64, t_f64=t64)
        out[name] = rec
    # electrograms of two histories, through the reference's own EGM code
    for name, el in (("sheet_ms_flag4", np.array([[1.0, 1.0, 1.0], [4.0, 2.0, 1.0], [2.6, 4.4, 1.0],
                                                   [5.2, 5.2, 1.0], [0.4, 4.8, 2.0], [3.0, 0.2, 0.5]])),
                     ("slab_ap_flag1", np.array([[-1.0, 1.2, 0.6], [1.2, 3.6, 2.0], [2.4, -0.8, 0.4],
                                                  [3.4, 1.2, 1.6], [1.0, 1.0, 0.6]])),
                     ("slab_ms_fibres", np.array([[-0.8, 0.9, 0.6], [1.4, 2.4, 2.1], [2.6, -0.9, 0.5],
                                                   [1.2, 1.0, -1.1]]))):
        if name not in out:
            continue
        rec = out[name]
        case = dict(voxel=rec["voxel"], nb=rec["neighbor_id_2d"], Delta=rec["Delta"],
                    D0=[d for d in rec["D0"]],
                    par={"c_voxel": rec["P_2d"][:, 20]})
        with contextlib.redirect_stdout(io.StringIO()):
            e32 = run_egm(cp, simulation, case, rec["u_f32"], el, fp64=False)
            e64 = run_egm(cp, simulation, case, rec["u_f64"], el, fp64=True)
        rec.update(egm_electrode_xyz=el, egm_f32=e32, egm_f64=e64)
        print(f"  egm {name}: {e64.shape}", flush=True)
    for name, rec in out.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **rec)
    print("wrote", sorted(out))


if __name__ == "__main__":
    main()
