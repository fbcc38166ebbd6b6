"""Failure detection without faulting the GPU: a non-finite instance retires
alone, maxiter exhaustion surfaces as the reference's warning, a bad table is
rejected before upload, and a barrier whose partner never arrives ends through
its bounded wait with PHS_ERR_TIMEOUT while the CUDA context stays usable."""
import ctypes
import time

import numpy as np
import pytest

from pyheartsim_b200 import _lib
from pyheartsim_b200.engine import BatchedEngine
from pyheartsim_b200.instance import compile_instance
from pyheartsim_b200.simulation import simulation_gpu
from tests import gpu_cases

pytestmark = pytest.mark.gpu

STEPS = 160


def _instances():
    out = []
    for case in ("sheet_ms", "slab_ap", "small_shell_ms"):
        (n, P, geom, sp, ap), pdur = getattr(gpu_cases, case)()
        out.append(compile_instance(n, P, geom, sp, ap, full_cycles=False, tol=1e-7, restart=20,
                                    pacing_duration=pdur, max_steps=STEPS))
    return out


def _run(insts):
    eng = BatchedEngine(_lib.PREC_F32)
    slots = [eng.add(x) for x in insts]
    eng.advance(STEPS, sync=True)
    res = [(eng.info(s), eng.history(s), eng.state(s)[0]) for s in slots]
    eng.close()
    return res


def test_nonfinite_instance_retires_alone(cuda_device):
    alone = [_run([x])[0] for x in _instances()]
    bad = _instances()[0]
    bad.u0 = float("nan")
    mixed = _run(_instances() + [bad])
    assert mixed[3][0]["status"] == _lib.PHS_ERR_NONFINITE
    assert mixed[3][0]["step"] < STEPS
    for (ia, ha, ua), (im, hm, um) in zip(alone, mixed[:3]):
        assert im["status"] == _lib.PHS_OK and im["step"] == STEPS
        np.testing.assert_array_equal(hm, ha)                  # batch-mates bit-identical
        np.testing.assert_array_equal(um, ua)


def test_maxiter_exhaustion_warns_like_the_reference(cuda_device):
    (n, P, geom, sp, ap), pdur = gpu_cases.sheet_ms(t_phys=3.0)
    with pytest.warns(UserWarning, match="did not converge"):
        simulation_gpu.compute(n, P, geom, dict(sp), dict(ap), pacing_duration=pdur, restart=2, maxiter=1)


def test_bad_neighbour_table_rejected_before_upload(cuda_device):
    inst = _instances()[0]
    inst.nb6 = inst.nb6.copy()
    inst.nb6[5, 2] = inst.n_voxel + 7
    eng = BatchedEngine(_lib.PREC_F32)
    slot = ctypes.c_int(-1)
    desc = inst.desc()
    rc = _lib.lib().phs_instance_add(eng._h, ctypes.byref(desc), ctypes.byref(slot))
    eng.close()
    assert rc == _lib.PHS_ERR_BAD_TABLE


def test_barrier_wait_gives_up_with_timeout_status(cuda_device):
    eng = BatchedEngine(_lib.PREC_F32)
    eng.add(_instances()[0])
    eng.config(_lib.CFG_TEST_TEAM_OVERCOUNT, 1)
    t0 = time.time()
    with pytest.raises(_lib.PhsError) as err:
        eng.advance(4, sync=True)
    assert err.value.status == _lib.PHS_ERR_TIMEOUT
    assert time.time() - t0 < 60
    with pytest.raises(_lib.PhsError):                          # the engine refuses further work
        eng.advance(1, sync=True)
    eng.close()
    # the CUDA context is still usable: a fresh engine runs normally
    res = _run(_instances()[:1])
    assert res[0][0]["status"] == _lib.PHS_OK and res[0][0]["step"] == STEPS
