"""GPU parity of the unipolar electrogram (calls go through the C ABI)."""
import ctypes

import numpy as np
import pytest

from oracle import egm_fp64
from pyheartsim_b200 import _lib, synthetic
from pyheartsim_b200.geometry import lattice_neighbors
from pyheartsim_b200.simulation import unipolar_electrogram_gpu
from tests import golden_cases

pytestmark = pytest.mark.gpu

EGM_NAMES = [n for n in golden_cases.names()
             if "egm_f64" in np.load(golden_cases.GOLDEN + f"/{n}.npz").files]
# FP64 lead field + FP64 contraction vs FP64 references
F64_RTOL = 1e-10
# BF16 hi/lo split, three products, FP32 accumulation: relative L2 bound
BF16X3_REL_L2 = 1e-3


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name", EGM_NAMES)
def test_egm_fp64_matches_reference_golden(name, cuda_device):
    g = golden_cases.load(name)["g"]
    e = unipolar_electrogram_gpu.compute(g["egm_electrode_xyz"], g["voxel"], golden_cases_D0(g), g["P_2d"][:, 20],
                                         g["u_f64"], float(g["Delta"]), g["neighbor_id_2d"])
    assert rel_l2(e, g["egm_f64"]) < F64_RTOL


def golden_cases_D0(g):
    """The fixture's diffusion tensors (fibre cases), else the reference's D0 = I."""
    if "D0" in g.files:
        return list(g["D0"])
    return [np.eye(3)] * g["voxel"].shape[0]


def wave_history(ijk, Delta, T, seed):
    """Travelling-front Vm history (T, n) with plateau and repolarisation."""
    rng = np.random.default_rng(seed)
    x = ijk @ rng.standard_normal(3) * Delta
    x -= x.min()
    t = np.linspace(0.0, 1.2 * x.max() + 5.0, T)[:, None]
    up = 1.0 / (1.0 + np.exp(-(t - x[None, :]) / 0.6))
    down = 1.0 / (1.0 + np.exp(-(t - x[None, :] - 0.6 * x.max()) / 1.5))
    return up * (1.0 - 0.9 * down)


def shell_case(seed=2, T=200, n_e=96):
    ijk = synthetic.shell((9.0, 8.0, 7.0), 0.4, 3, 2, 2.0, seed)
    nb = lattice_neighbors(ijk)
    rng = np.random.default_rng(seed)
    c = synthetic.scar(ijk, nb, 0.1, rng) * 1.6
    el = synthetic.electrodes_off_surface(ijk, 0.4, n_e, rng)
    V = wave_history(ijk, 0.4, T, seed)
    return ijk * 0.4, nb, c, el, V


def test_egm_fp64_matches_oracle_shell(cuda_device):
    xyz, nb, c, el, V = shell_case()
    e = unipolar_electrogram_gpu.compute(el, xyz, None, c, V, 0.4, nb)
    eo = egm_fp64.compute(el, xyz, None, c, V, 0.4, nb)
    assert rel_l2(e, eo) < F64_RTOL


def test_egm_fp64_general_d0(cuda_device):
    xyz, nb, c, el, V = shell_case(seed=3, T=40, n_e=20)
    rng = np.random.default_rng(3)
    n = xyz.shape[0]
    f = rng.standard_normal((n, 3))
    f /= np.linalg.norm(f, axis=1, keepdims=True)
    D0 = [0.3 * np.eye(3) + 0.7 * np.outer(v, v) for v in f]
    e = unipolar_electrogram_gpu.compute(el, xyz, D0, c, V, 0.4, nb)
    eo = egm_fp64.direct(el, xyz, D0, c, V, 0.4, nb)
    assert rel_l2(e, eo) < F64_RTOL


def test_egm_bf16x3_rel_l2(cuda_device):
    xyz, nb, c, el, V = shell_case(seed=4, T=200, n_e=96)
    e = unipolar_electrogram_gpu.compute(el, xyz, None, c, V, 0.4, nb, mode="bf16x3")
    eo = egm_fp64.compute(el, xyz, None, c, V, 0.4, nb)
    r = rel_l2(e, eo)
    assert r < BF16X3_REL_L2, r


@pytest.mark.parametrize("config", [-1, 0, 1, 2, 3])
@pytest.mark.parametrize("T,K,E", [(77, 5000, 40), (256, 8192, 256), (300, 20000, 130)])
def test_bf16x3_contraction_device_pointers(T, K, E, config, cuda_device):
    """The tcgen05 kernel alone, on torch-owned device buffers, in every tile
    configuration (-1: the default entry point); E = 40 and 130 pad to 128 and
    256 rows, so the 256-wide tiles also read rows past the operand's end."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(T + K + E)
    A = torch.randn(T, K, dtype=torch.float64, generator=g)
    B = torch.randn(E, K, dtype=torch.float64, generator=g)
    ref = (A @ B.T).numpy()
    Tp, Ep, Kp = (T + 127) // 128 * 128, (E + 127) // 128 * 128, (K + 63) // 64 * 64
    dA, dB = A.to(cuda_device), B.to(cuda_device)
    hA = torch.empty(Tp, Kp, dtype=torch.uint16, device=cuda_device)
    lA = torch.empty_like(hA)
    hB = torch.empty(Ep, Kp, dtype=torch.uint16, device=cuda_device)
    lB = torch.empty_like(hB)
    L = _lib.lib()
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.phs_split_bf16(T, K, p(dA), K, 1, p(hA), p(lA), Tp, Kp, s), "split A")
    _lib.check(L.phs_split_bf16(E, K, p(dB), K, 1, p(hB), p(lB), Ep, Kp, s), "split B")
    ws = L.phs_egm_bf16x3_workspace(Tp, Ep, Kp)
    work = torch.empty(ws, dtype=torch.uint8, device=cuda_device)
    out = torch.empty(T, E, dtype=torch.float32, device=cuda_device)
    assert L.phs_egm_bf16x3_config_count() == 4
    if config < 0:
        _lib.check(L.phs_egm_contract_bf16x3(T, E, Tp, Ep, Kp, p(hA), p(lA), p(hB), p(lB), p(out), p(work), s),
                   "contract")
    else:
        _lib.check(L.phs_egm_contract_bf16x3_cfg(T, E, Tp, Ep, Kp, p(hA), p(lA), p(hB), p(lB), p(out), p(work),
                                                 config, s), "contract")
    _lib.check(L.phs_egm_bf16x3_status(p(work), s), "contract status")
    torch.cuda.synchronize()
    got = out.cpu().numpy().astype(np.float64)
    assert rel_l2(got, ref) < 1e-4
