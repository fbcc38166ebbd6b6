"""Seeded cases shared by the GPU tests (sizes the oracle finishes in seconds)."""
import numpy as np

from pyheartsim_b200 import synthetic


def sheet_ms(nx=40, ny=40, t_phys=30.0, dt=0.05, stim_ms=1.0):
    ijk = synthetic.sheet(nx, ny)
    s1 = np.where((ijk[:, 0] < 5) & (ijk[:, 1] < 5))[0]
    return synthetic.make_case(ijk, 0.4, 0, dt, t_phys, s1, flag=4), stim_ms


def slab_ap(nx=16, ny=16, nz=4, t_phys=40.0, dt=0.1):
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ijk = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1)
    s1 = np.where(ijk[:, 0] == 0)[0]
    s2 = np.where((ijk[:, 0] < nx // 2) & (ijk[:, 1] > ny // 2))[0]
    return synthetic.make_case(ijk, 0.4, 1, dt, t_phys, s1, s2_ids=s2, flag=1, s1_s2=20.0), None


def small_shell_ms(seed=1, t_phys=40.0, dt=0.05, scar_cov=0.15, fibres=False):
    return synthetic.small_shell_case(seed, t_phys, dt, scar_cov, fibres)


def small_shell_ms_fibres():
    """small_shell_ms with a rotating fibre field (anisotropic D0, all cross terms)."""
    return small_shell_ms(fibres=True)
