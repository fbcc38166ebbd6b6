"""The streamed result writer produces what the reference's np.savez call
(simulation_individual.py:77-92, 365-366) produces, from chunked history reads
(a host stand-in for the engine; no GPU)."""
import numpy as np
import pytest

from pyheartsim_b200 import results


class FakeEngine:
    def __init__(self, u, h):
        self.u, self.h = u, h
        self.reads = []

    def info(self, slot):
        return {"samples": self.u.shape[0], "n_voxel": self.u.shape[1]}

    def history(self, slot, s0=0, count=None, with_h=False):
        count = self.u.shape[0] - s0 if count is None else count
        self.reads.append(count)
        u = self.u[s0:s0 + count].copy()
        return (u, self.h[s0:s0 + count].copy()) if with_h else u


@pytest.mark.parametrize("egm,save_all,dtype", [(False, True, None), (True, True, np.float32), (True, False, None),
                                                (False, False, np.float32)])
def test_streamed_file_equals_np_savez(tmp_path, egm, save_all, dtype):
    rng = np.random.default_rng(1)
    S, n = 37, 500
    u = rng.standard_normal((S, n))
    h = rng.standard_normal((S, n))
    ids = np.array([3, 77, 120, 499])
    e = rng.standard_normal((S, 4))
    t = np.arange(S, dtype=np.float32)
    lat = np.array([2, 0, 5, 1])
    eng = FakeEngine(u, h)
    path = results.save_simulation_results(tmp_path / "run_simulation_results", eng, 0, geometry_flag=1,
                                           electrode_ids=ids, electrogram=e if egm else None, save_all=save_all,
                                           physical_time=t, lat_electrode=lat, dtype=dtype, chunk=8)
    assert max(eng.reads, default=0) <= 8                        # never the whole history at once
    cast = (lambda a: a.astype(dtype)) if dtype is not None else (lambda a: a)
    ref = {"geometry_flag": 1}
    if egm:
        ref["electrogram_unipolar"] = e
    else:
        ref["action_potential_electrode"] = cast(u[:, ids])
    if save_all:
        ref["action_potential"] = cast(u)
        ref["h"] = cast(h)
        ref["physical_time"] = t
    ref["lat_electrode"] = lat
    np.savez(tmp_path / "ref", **ref)
    a, b = np.load(path), np.load(tmp_path / "ref.npz")
    assert a.files == b.files
    for k in a.files:
        assert a[k].dtype == b[k].dtype and a[k].shape == b[k].shape, k
        np.testing.assert_array_equal(a[k], b[k])
