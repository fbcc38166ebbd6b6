"""GPU parity of the time-stepping path (calls go through the C ABI)."""
import numpy as np
import pytest

from oracle import simulation_fp64
from pyheartsim_b200.simulation import simulation_gpu
from tests import golden_cases, gpu_cases

pytestmark = pytest.mark.gpu

# plain FP64 form vs the reference's own FP64 run / the FP64 oracle
PLAIN_ATOL = 1e-9
# FP32 early-exit form vs the FP64 oracle, max |dVm| over the run's samples
FAST_DVM = 1e-3


@pytest.mark.parametrize("name", golden_cases.names())
def test_plain_fp64_matches_reference_golden(name, cuda_device):
    c = golden_cases.load(name)
    g = c["g"]
    u, h, t = simulation_gpu.compute(c["n"], c["P_2d"], c["geom"], dict(c["sp"]), dict(c["ap"]))
    assert u.dtype == np.float64 and u.shape == g["u_f64"].shape
    np.testing.assert_allclose(u, g["u_f64"], rtol=0, atol=PLAIN_ATOL)
    np.testing.assert_allclose(h, g["h_f64"], rtol=0, atol=PLAIN_ATOL)
    np.testing.assert_array_equal(t, g["t_f64"])


@pytest.mark.parametrize("case", ["sheet_ms", "slab_ap", "small_shell_ms", "small_shell_ms_fibres"])
def test_plain_fp64_matches_oracle(case, cuda_device):
    (n, P, geom, sp, ap), pdur = getattr(gpu_cases, case)()
    u, h, t, lat = simulation_gpu.compute(n, P, geom, dict(sp), dict(ap), pacing_duration=pdur, return_lat=True)
    uo, ho, to, lato = simulation_fp64.compute(n, P, geom, dict(sp), dict(ap), pacing_duration=pdur,
                                               record_lat=True)
    assert u.shape == uo.shape
    assert np.abs(uo).max() > 0.5, "case must actually propagate"
    np.testing.assert_allclose(u, uo, rtol=0, atol=PLAIN_ATOL)
    np.testing.assert_allclose(h, ho, rtol=0, atol=PLAIN_ATOL)
    np.testing.assert_array_equal(lat, lato)


@pytest.mark.parametrize("case", ["sheet_ms", "slab_ap", "small_shell_ms", "small_shell_ms_fibres"])
def test_fast_fp32_lat_within_one_step(case, cuda_device):
    """FP32 state, FP64 dots, Givens early exit: LAT error <= 1 dt against FP64."""
    (n, P, geom, sp, ap), pdur = getattr(gpu_cases, case)()
    u, h, t, lat = simulation_gpu.compute(n, P, geom, dict(sp), dict(ap), pacing_duration=pdur,
                                          dtype=np.float32, fast=True, tol=1e-7, return_lat=True)
    uo, ho, to, lato = simulation_fp64.compute(n, P, geom, dict(sp), dict(ap), pacing_duration=pdur,
                                               record_lat=True)
    assert u.dtype == np.float32
    both = (lat >= 0) & (lato >= 0)
    assert np.array_equal(lat >= 0, lato >= 0)
    assert np.abs(lat[both].astype(np.int64) - lato[both]).max() <= 1
    # measured max |dVm| of these four cases: 2.2e-4 (sheet), 6.7e-6 (AP slab),
    # 4.1e-5 and 3.5e-5 (shells); the bound is about five times the largest
    assert np.abs(u - uo).max() < FAST_DVM


def test_repeat_is_bit_identical(cuda_device):
    (n, P, geom, sp, ap), pdur = gpu_cases.small_shell_ms()
    a = simulation_gpu.compute(n, P, geom, dict(sp), dict(ap), pacing_duration=pdur, dtype=np.float32, fast=True)
    b = simulation_gpu.compute(n, P, geom, dict(sp), dict(ap), pacing_duration=pdur, dtype=np.float32, fast=True)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_isotropic_instance_unchanged_beside_anisotropic(cuda_device):
    """A batch holding an anisotropic instance launches the edge-term kernel; the
    isotropic instance next to it gives the same history as when it runs alone
    (the kernel without edge terms)."""
    from pyheartsim_b200 import instance
    from pyheartsim_b200.engine import BatchedEngine
    (n, P, geom, sp, ap), pdur = gpu_cases.small_shell_ms(t_phys=15.0)
    (nf, Pf, geomf, spf, apf), _ = gpu_cases.small_shell_ms(t_phys=15.0, fibres=True)
    kw = dict(full_cycles=False, tol=1e-7, restart=20, pacing_duration=pdur)
    iso = instance.compile_instance(n, P, geom, dict(sp), dict(ap), **kw)
    ani = instance.compile_instance(nf, Pf, geomf, dict(spf), dict(apf), **kw)
    assert iso.coef_edge is None and ani.coef_edge is not None
    alone = BatchedEngine()
    s0 = alone.add(iso)
    while not alone.finished(s0):
        alone.advance(50)
    ref = alone.history(s0)
    alone.close()
    mix = BatchedEngine()
    a, b = mix.add(iso), mix.add(ani)
    while not (mix.finished(a) and mix.finished(b)):
        mix.advance(50)
    np.testing.assert_array_equal(mix.history(a), ref)
    assert mix.info(b)["status"] == 0
    mix.close()
