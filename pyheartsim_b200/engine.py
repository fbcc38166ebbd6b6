"""Batched engine: many uneven simulation instances advanced together.

Thin Python handle over the ``phs_engine_*`` C ABI (include/phs.h).  Each call
to :meth:`advance` is one persistent sm_100a launch in which every unfinished
instance is advanced by a team of CTAs sized to its voxel count; instances of
different sizes, models and time steps progress independently.  State, solver
workspace, stimulus schedule and history stay on the device between calls.
"""
import ctypes

import numpy as np

from . import _lib


def tensor_to_host(t, stage=None, stage_bytes=128 << 20, stream=None):
    """Copy a 2-D CUDA tensor to a new numpy array through two pinned staging
    buffers (reused when ``stage`` holds large enough ones of the same dtype),
    on ``stream`` (default: a new stream of the tensor's device); each chunk's
    device-to-host copy overlaps the host copy of the one before.  Returns
    (array, staging buffers).  Safe to call from a worker thread."""
    import torch
    rows, n = t.shape
    out = np.empty((rows, n), dtype=np.float32 if t.dtype == torch.float32 else np.float64)
    if rows == 0:
        return out, stage
    dev = t.device
    per = max(1, int(stage_bytes // max(1, n * t.element_size())))
    if stage is None or stage[0].numel() < per * n or stage[0].dtype != t.dtype:
        stage = [torch.empty(per * n, dtype=t.dtype, pin_memory=True) for _ in range(2)]
    stream = stream or torch.cuda.Stream(dev)
    events = [None, None]
    prev = None
    with torch.cuda.stream(stream):
        for k, a in enumerate(range(0, rows, per)):
            b = min(rows, a + per)
            buf = stage[k % 2]
            if events[k % 2] is not None:
                events[k % 2].synchronize()          # its previous chunk has been copied out below
            buf[:(b - a) * n].view(b - a, n).copy_(t[a:b], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
            if prev is not None:
                pa, pb, pbuf, pev = prev
                pev.synchronize()
                np.copyto(out[pa:pb], pbuf[:(pb - pa) * n].numpy().reshape(pb - pa, n))
            prev = (a, b, buf, ev)
            events[k % 2] = ev
        pa, pb, pbuf, pev = prev
        pev.synchronize()
        np.copyto(out[pa:pb], pbuf[:(pb - pa) * n].numpy().reshape(pb - pa, n))
    return out, stage


class BatchedEngine:
    def __init__(self, precision=_lib.PREC_F32):
        self.precision = precision
        self._h = ctypes.c_void_p()
        _lib.check(_lib.lib().phs_engine_create(precision, ctypes.byref(self._h)), "phs_engine_create")
        self._inst = {}

    # -- instances ------------------------------------------------------------
    def add(self, inst):
        """Upload a :class:`pyheartsim_b200.instance.CompiledInstance`; returns its slot."""
        slot = ctypes.c_int(-1)
        desc = inst.desc()
        _lib.check(_lib.lib().phs_instance_add(self._h, ctypes.byref(desc), ctypes.byref(slot)), "phs_instance_add")
        self._inst[slot.value] = inst
        return slot.value

    def remove(self, slot):
        _lib.check(_lib.lib().phs_instance_remove(self._h, slot), "phs_instance_remove")
        self._inst.pop(slot, None)

    def instance(self, slot):
        return self._inst[slot]

    def slots(self):
        return list(self._inst)

    # -- stepping ---------------------------------------------------------------
    def advance(self, n_steps, stream=None, sync=True, ctas_per_sm=0):
        """Advance every unfinished instance by up to ``n_steps`` steps.

        ``stream`` is a cudaStream_t handle (int) or a torch.cuda.Stream.
        Returns the worst instance status: OK, the no-convergence warning, or
        PHS_ERR_NONFINITE when an instance was retired (the others continue;
        see :meth:`info`).  Other failures raise."""
        if stream is not None and hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        st = _lib.lib().phs_engine_advance(self._h, int(n_steps), int(ctas_per_sm),
                                           ctypes.c_void_p(stream) if stream else None, 1 if sync else 0)
        return _lib.check(st, "phs_engine_advance", allow_warn=True, allow_nonfinite=True)

    def info(self, slot):
        i = _lib.InstanceInfo()
        _lib.check(_lib.lib().phs_instance_info_get(self._h, slot, ctypes.byref(i)), "phs_instance_info_get")
        return {k: getattr(i, k) for k, _ in _lib.InstanceInfo._fields_}

    def finished(self, slot):
        i = self.info(slot)
        return i["step"] >= i["n_steps"] or i["status"] == _lib.PHS_ERR_NONFINITE

    # -- results ----------------------------------------------------------------
    def history(self, slot, s0=0, count=None, with_h=False):
        inst = self._inst[slot]
        info = self.info(slot)
        if count is None:
            count = info["samples"] - s0
        dt = _lib.np_dtype(self.precision)
        u = np.empty((count, inst.n_voxel), dtype=dt)
        h = np.empty((count, inst.n_voxel), dtype=dt) if with_h else None
        _lib.check(_lib.lib().phs_instance_read_history(self._h, slot, s0, count, _lib.vptr(u), _lib.vptr(h)),
                   "phs_instance_read_history")
        u = inst.to_caller(u)
        if with_h:
            return u, inst.to_caller(h)
        return u

    def history_device(self, slot, s0=0, count=None, stream=None):
        """A copy of the instance's Vm history rows s0 .. s0+count as a new CUDA
        tensor (count, n) in the caller's voxel order, gathered on the device
        (the engine keeps its rows in device order).  The copy is made on
        ``stream`` (default: the current torch stream) after the engine's
        queued work; the instance may be removed once the stream has it."""
        import torch
        inst = self._inst[slot]
        info = self.info(slot)
        if count is None:
            count = info["samples"] - s0
        u = ctypes.c_void_p()
        hist = ctypes.c_void_p()
        lat = _lib.c_int32_p()
        _lib.check(_lib.lib().phs_instance_device_ptrs(self._h, slot, ctypes.byref(u), ctypes.byref(hist),
                                                       ctypes.byref(lat)), "phs_instance_device_ptrs")
        n = int(inst.n_voxel)
        tdt = torch.float32 if self.precision == _lib.PREC_F32 else torch.float64
        dev = torch.device("cuda", torch.cuda.current_device())
        esz = 4 if tdt == torch.float32 else 8

        class _View:   # the engine's device rows, seen by torch without a copy
            __cuda_array_interface__ = {"data": (hist.value + s0 * n * esz, False), "shape": (count, n),
                                        "typestr": "<f4" if esz == 4 else "<f8", "version": 3, "strides": None}

        torch.cuda.synchronize(dev)            # the engine's launches may be on any stream
        src = torch.as_tensor(_View(), device=dev)
        st = stream or torch.cuda.current_stream(dev)
        with torch.cuda.stream(st):
            if inst.inv is None:
                out = src.clone()
            else:
                inv = getattr(inst, "_inv_dev", None)
                if inv is None or inv.device != dev:
                    inv = torch.as_tensor(inst.inv, device=dev)
                    inst._inv_dev = inv
                out = src.index_select(1, inv)
        return out

    def history_host(self, slot, s0=0, count=None, stage_bytes=128 << 20):
        """The instance's Vm history (count, n) in the caller's voxel order as a
        numpy array, fast: gathered into caller order on the device, copied to
        the host through two reused pinned staging buffers of ``stage_bytes``
        (each chunk's device-to-host copy overlaps the host copy of the one
        before).  Same values as :meth:`history`."""
        t = self.history_device(slot, s0, count)
        st = getattr(self, "_stage", None)
        out, self._stage = tensor_to_host(t, st, stage_bytes)
        return out

    def activation_times(self, slot, max_per_voxel=16, threshold=0.5, stream=None):
        """Every upward crossing of ``threshold`` by Vm in the instance's device
        history (``phs_activation_times``): ``(times, counts)`` in the caller's
        voxel order, ``times[v, i]`` the sample index of crossing i of voxel v
        (-1 past ``counts[v]``).  With a history sampled every step
        (``sample_stride`` 1) the first crossing is the activation step and the
        later ones are the re-activations, in units of dt."""
        import torch
        inst = self._inst[slot]
        info = self.info(slot)
        u = ctypes.c_void_p()
        hist = ctypes.c_void_p()
        lat = _lib.c_int32_p()
        _lib.check(_lib.lib().phs_instance_device_ptrs(self._h, slot, ctypes.byref(u), ctypes.byref(hist),
                                                       ctypes.byref(lat)), "phs_instance_device_ptrs")
        n = int(inst.n_voxel)
        S = int(info["samples"])
        dev = torch.device("cuda", torch.cuda.current_device())
        times = torch.full((n, max(int(max_per_voxel), 1)), -1, dtype=torch.int32, device=dev)
        counts = torch.zeros(n, dtype=torch.int32, device=dev)
        if stream is None:
            stream = torch.cuda.current_stream(dev).cuda_stream
        elif hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        torch.cuda.synchronize(dev)
        _lib.check(_lib.lib().phs_activation_times(S, n, hist, n, int(self.precision == _lib.PREC_F64),
                                                   float(threshold), int(max_per_voxel),
                                                   ctypes.c_void_p(times.data_ptr()),
                                                   ctypes.c_void_p(counts.data_ptr()), ctypes.c_void_p(stream)),
                   "phs_activation_times")
        torch.cuda.synchronize(dev)
        t = times.cpu().numpy()[:, :int(max_per_voxel)]
        c = counts.cpu().numpy()
        if inst.inv is not None:
            t, c = t[inst.inv], c[inst.inv]
        return t, c

    def state(self, slot):
        inst = self._inst[slot]
        dt = _lib.np_dtype(self.precision)
        u = np.empty(inst.n_voxel, dtype=dt)
        h = np.empty(inst.n_voxel, dtype=dt)
        lat = np.empty(inst.n_voxel, dtype=np.int32)
        _lib.check(_lib.lib().phs_instance_read_state(self._h, slot, _lib.vptr(u), _lib.vptr(h),
                                                      _lib.ptr(lat, ctypes.c_int32)), "phs_instance_read_state")
        return inst.to_caller(u), inst.to_caller(h), inst.to_caller(lat)

    def config(self, key, value):
        _lib.check(_lib.lib().phs_engine_config(self._h, int(key), int(value)), "phs_engine_config")

    def configure(self, variant=None, ctas_per_sm=None, auto_balance=None, wave_instances=None,
                  compact_nb=None):
        """Select the step-kernel variant and the CTAs per SM used by advance(),
        whether the 2nd and 3rd advance after an add/remove rebalance first,
        the most instances per launch wave (0: all in one wave) and whether
        instances read their compact neighbour table (same results)."""
        L = _lib.lib()
        if compact_nb is not None:
            _lib.check(L.phs_engine_config(self._h, _lib.CFG_COMPACT_NB, int(bool(compact_nb))),
                       "phs_engine_config")
        if wave_instances is not None:
            _lib.check(L.phs_engine_config(self._h, _lib.CFG_WAVE_INSTANCES, int(wave_instances)),
                       "phs_engine_config")
        if auto_balance is not None:
            _lib.check(L.phs_engine_config(self._h, _lib.CFG_AUTO_BALANCE, int(bool(auto_balance))),
                       "phs_engine_config")
        if variant is not None:
            _lib.check(L.phs_engine_config(self._h, _lib.CFG_VARIANT, int(variant)), "phs_engine_config")
        if ctas_per_sm is not None:
            _lib.check(L.phs_engine_config(self._h, _lib.CFG_CTAS_PER_SM, int(ctas_per_sm)), "phs_engine_config")

    def rebalance(self):
        """Re-split CTAs over instances by recent cost (voxels x Arnoldi iterations)."""
        _lib.check(_lib.lib().phs_engine_rebalance(self._h), "phs_engine_rebalance")

    def set_profile(self, on=True):
        _lib.check(_lib.lib().phs_engine_config(self._h, _lib.CFG_PROFILE, 1 if on else 0), "phs_engine_config")

    def profile(self, slot):
        """Phase timers of an instance in ms (team's first CTA), plus counts."""
        out = (ctypes.c_uint64 * 16)()
        _lib.check(_lib.lib().phs_instance_profile(self._h, slot, out), "phs_instance_profile")
        d = {}
        for i, name in enumerate(_lib.PROFILE_SLOTS):
            d[name] = int(out[i]) if name in ("steps", "arnoldi_iters", "team_ctas", "barriers") else out[i] / 1e6
        return d

    def table_bytes(self, slot):
        """Bytes per voxel of the neighbour table the instance's compact-table
        variants read (8 compact, 24 int32)."""
        b = ctypes.c_int32()
        _lib.check(_lib.lib().phs_instance_table_bytes(self._h, slot, ctypes.byref(b)), "phs_instance_table_bytes")
        return int(b.value)

    def launches(self):
        return int(_lib.lib().phs_engine_launch_count(self._h))

    def close(self):
        if self._h:
            _lib.lib().phs_engine_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._inst.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def step_variant_layout(precision=_lib.PREC_F32):
    """[(ring bytes, reads the compact table)] per step-kernel variant: ring
    bytes > 0 for the staged variants (producer warp, bulk copies into a
    shared-memory ring)."""
    n = len(step_variants(precision))
    ring = np.zeros(n, dtype=np.int32)
    comp = np.zeros(n, dtype=np.int32)
    _lib.check(_lib.lib().phs_step_variant_layout(precision, n, _lib.ptr(ring, ctypes.c_int32),
                                                  _lib.ptr(comp, ctypes.c_int32)), "phs_step_variant_layout")
    return [(int(r), bool(c)) for r, c in zip(ring, comp)]


def step_variants(precision=_lib.PREC_F32, with_vpt=False):
    """[(variant, min CTAs/SM it was compiled for, registers per thread)], with
    the voxels per thread (tile = 256 x VPT voxels) as a fourth entry when
    ``with_vpt``."""
    n = ctypes.c_int32(0)
    _lib.check(_lib.lib().phs_step_variants(precision, ctypes.byref(n), None, None), "phs_step_variants")
    minb = np.zeros(n.value, dtype=np.int32)
    regs = np.zeros(n.value, dtype=np.int32)
    _lib.check(_lib.lib().phs_step_variants(precision, ctypes.byref(n), _lib.ptr(minb, ctypes.c_int32),
                                            _lib.ptr(regs, ctypes.c_int32)), "phs_step_variants")
    if with_vpt:
        vpt = np.zeros(n.value, dtype=np.int32)
        _lib.check(_lib.lib().phs_step_variant_vpt(precision, n.value, _lib.ptr(vpt, ctypes.c_int32)),
                   "phs_step_variant_vpt")
        return [(i, int(minb[i]), int(regs[i]), int(vpt[i])) for i in range(n.value)]
    return [(i, int(minb[i]), int(regs[i])) for i in range(n.value)]
