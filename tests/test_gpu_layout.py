"""Data-layout options of the engine give the same results bit for bit: the
compact neighbour table against the int32 one (FP32 early exit and plain FP64,
isotropic and anisotropic rows, lattice row order and a scattered order that
cannot be compacted), and the staged and compact-table step-kernel variants
against the int32-table kernel."""
import numpy as np
import pytest

from pyheartsim_b200 import _lib, instance
from pyheartsim_b200.engine import BatchedEngine
from tests import gpu_cases

pytestmark = pytest.mark.gpu

STAGED = [5, 6]             # FP32 variants with the producer warp and shared-memory ring
COMPACT = [7, 8]            # FP32 variants that read the compact neighbour table (int32 twins 4, 2)


def _run(inst, precision, **cfg):
    eng = BatchedEngine(precision)
    eng.configure(**cfg)
    s = eng.add(inst)
    tb = eng.table_bytes(s)
    while not eng.finished(s):
        eng.advance(40)
    hist = eng.history(s)
    info = eng.info(s)
    eng.close()
    return hist, tb, info


def _compile(case, pdur, fast, reorder="rows"):
    n, P, geom, sp, ap = case
    kw = dict(full_cycles=False, tol=1e-7, restart=20) if fast else {}
    return instance.compile_instance(n, P, geom, dict(sp), dict(ap), pacing_duration=pdur, reorder=reorder, **kw)


@pytest.mark.parametrize("fast", [True, False])
@pytest.mark.parametrize("name", ["small_shell_ms", "small_shell_ms_fibres", "sheet_ms", "slab_ap"])
def test_compact_table_same_history(name, fast, cuda_device):
    case, pdur = getattr(gpu_cases, name)()
    if not fast:
        n, P, geom, sp, ap = case
        sp = dict(sp)
        sp["t_final"] = min(sp["t_final"], 10.0)      # plain GMRES(50): a shorter run
        case = (n, P, geom, sp, ap)
    inst = _compile(case, pdur, fast)
    prec = _lib.PREC_F32 if fast else _lib.PREC_F64
    variant = 7 if fast else None                       # an FP32 variant that reads the compact table
    h_c, tb_c, i_c = _run(inst, prec, compact_nb=True, variant=variant)
    h_w, tb_w, i_w = _run(inst, prec, compact_nb=False, variant=variant)
    assert (tb_c, tb_w) == (8, 24)
    assert i_c["status"] == i_w["status"] == 0
    assert i_c["arnoldi_steps"] == i_w["arnoldi_steps"]
    np.testing.assert_array_equal(h_c, h_w)


def test_scattered_order_keeps_int32_table(cuda_device):
    """In Z-curve order every slot needs stored offsets: the instance keeps the
    int32 table whatever the setting, with the same results."""
    case, pdur = gpu_cases.small_shell_ms(t_phys=15.0)
    a = _compile(case, pdur, True, reorder="morton")
    h_a, tb_a, _ = _run(a, _lib.PREC_F32, compact_nb=True, variant=7)
    h_b, tb_b, _ = _run(a, _lib.PREC_F32, compact_nb=False, variant=7)
    assert tb_a == tb_b == 24
    np.testing.assert_array_equal(h_a, h_b)


def _batch(fast=True):
    """Three small scarred shells (one with fibres) and a 700 x 700 sheet, so
    that CTAs walk several tiles per phase and the ring wraps."""
    from pyheartsim_b200 import synthetic
    out = []
    for seed, fib in ((1, False), (2, False), (3, True)):
        (n, P, geom, sp, ap), pdur = synthetic.small_shell_case(seed, 6.0, 0.05, 0.15, fib)
        out.append(_compile((n, P, geom, sp, ap), pdur, fast))
    case, pdur = gpu_cases.sheet_ms(nx=700, ny=700, t_phys=3.0)
    out.append(_compile(case, pdur, fast))
    return out


def _run_batch(insts, **cfg):
    eng = BatchedEngine(_lib.PREC_F32)
    eng.configure(auto_balance=False, **cfg)
    slots = [eng.add(x) for x in insts]
    while not all(eng.finished(s) for s in slots):
        eng.advance(20)
    out = [(eng.history(s), eng.info(s)) for s in slots]
    eng.close()
    return out


@pytest.mark.parametrize("fast", [True, False])
def test_staged_and_compact_variants_same_history(fast, cuda_device):
    """The staged kernels (bulk copies into a shared-memory ring) and the
    compact-table kernels compute what the int32-table kernel of the same tile
    length does, bit for bit: early exit and full GMRES cycles, isotropic and anisotropic rows,
    compact and int32 neighbour tables (a compact variant with the tables off
    runs its int32 twin), one and several CTAs per SM."""
    from pyheartsim_b200.engine import step_variant_layout, step_variants
    assert [v for v, *_ in step_variants(_lib.PREC_F32)][-4:] == STAGED + COMPACT
    lay = step_variant_layout(_lib.PREC_F32)
    assert all(lay[v][0] > 0 for v in STAGED) and all(lay[v] == (0, True) for v in COMPACT)
    insts = _batch(fast)
    # partial sums are grouped by tile, so each variant is compared with the
    # int32-table variant of its tile length (512 voxels: 4, 1024: 2)
    vpt = {v: t for v, _, _, t in step_variants(_lib.PREC_F32, with_vpt=True)}
    refs = {vpt[4]: _run_batch(insts, variant=4), vpt[2]: _run_batch(insts, variant=2)}
    for var in STAGED + COMPACT:
        ref = refs[vpt[var]]
        for cps, compact in ((1, True), (0, True), (1, False)):
            got = _run_batch(insts, variant=var, ctas_per_sm=cps, compact_nb=compact)
            for (h0, i0), (h1, i1) in zip(ref, got):
                assert i1["status"] == i0["status"] == 0
                assert i1["arnoldi_steps"] == i0["arnoldi_steps"], (var, cps, compact)
                np.testing.assert_array_equal(h1, h0, err_msg=f"variant {var} cps {cps} compact {compact}")
