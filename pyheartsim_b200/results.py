"""Simulation result files in the reference's format, streamed from the device.

simulation_individual.py:77-92 saves ``np.savez(f'{name_prefix}_simulation_results',
**simulation_results)`` with, in this order, ``geometry_flag``, then either
``action_potential_electrode`` (Vm at the electrode voxels, (T, n_e)) or
``electrogram_unipolar`` ((T, n_e)), then, when all voxels are kept,
``action_potential`` and ``h`` ((T, n_voxel)) and ``physical_time``;
simulation_individual.py:365-366 later adds ``lat_electrode``.

:func:`save_simulation_results` writes the same .npz (uncompressed zip of .npy
members, what ``np.savez`` writes, so ``np.load`` returns the same arrays) but
never holds a whole (T, n_voxel) history on the host: the history is read from
the engine's device buffer ``chunk`` samples at a time (in caller order) and
each chunk is appended to its zip member.
"""
import zipfile

import numpy as np


def _member(zf, name, shape, dtype, chunks):
    """One .npy member written from C-ordered chunks along the first axis."""
    dtype = np.dtype(dtype)
    header = {"descr": np.lib.format.dtype_to_descr(dtype), "fortran_order": False, "shape": tuple(int(s) for s in shape)}
    rows = 0
    with zf.open(name + ".npy", "w", force_zip64=True) as f:
        np.lib.format.write_array_header_1_0(f, header)
        for c in chunks:
            c = np.ascontiguousarray(c, dtype=dtype)
            rows += c.shape[0] if c.ndim else 1
            f.write(memoryview(c).cast("B"))
    if len(shape) and rows != shape[0]:
        raise RuntimeError(f"{name}: wrote {rows} rows, header says {shape[0]}")


def _whole(a):
    yield a


def save_simulation_results(path, engine, slot, *, geometry_flag, electrode_ids=None, electrogram=None,
                            save_all=False, physical_time=None, lat_electrode=None, dtype=None, chunk=64):
    """Write the reference's result file for instance ``slot`` of ``engine``.

    ``electrogram`` given -> ``electrogram_unipolar``; else the Vm history at
    ``electrode_ids`` -> ``action_potential_electrode``.  ``save_all`` adds
    ``action_potential``, ``h`` and ``physical_time`` (the reference's
    save_action_potential_of_all_voxel_flag).  ``lat_electrode`` is appended
    last when given.  ``dtype``: stored type of the histories (default the
    engine's; np.float32 matches the reference's shipped arrays).  ``path``
    gets the .npz suffix if it has none (as np.savez does)."""
    path = str(path)
    if not path.endswith(".npz"):
        path += ".npz"
    info = engine.info(slot)
    S = int(info["samples"])
    n = int(info["n_voxel"])
    dt = np.dtype(dtype) if dtype is not None else None

    def hist(with_h):
        for s0 in range(0, S, chunk):
            yield engine.history(slot, s0, min(chunk, S - s0), with_h=with_h)

    with zipfile.ZipFile(path, mode="w", compression=zipfile.ZIP_STORED, allowZip64=True) as zf:
        _member(zf, "geometry_flag", (), np.asarray(geometry_flag).dtype, _whole(np.asarray(geometry_flag)))
        if electrogram is not None:
            e = np.asarray(electrogram)
            _member(zf, "electrogram_unipolar", e.shape, e.dtype, _whole(e))
        else:
            ids = np.asarray(electrode_ids)
            first = engine.history(slot, 0, 1) if S else np.zeros((0, n))
            ed = dt or first.dtype
            _member(zf, "action_potential_electrode", (S, ids.size), ed, (u[:, ids] for u in hist(False)))
        if save_all:
            first = engine.history(slot, 0, 1) if S else np.zeros((0, n))
            hd = dt or first.dtype
            _member(zf, "action_potential", (S, n), hd, (u for u in hist(False)))
            _member(zf, "h", (S, n), hd, (h for _, h in hist(True)))
            pt = np.asarray(physical_time)
            _member(zf, "physical_time", pt.shape, pt.dtype, _whole(pt))
        if lat_electrode is not None:
            la = np.asarray(lat_electrode)
            _member(zf, "lat_electrode", la.shape, la.dtype, _whole(la))
    return path
