"""Continuous-batching server for simulation requests.

Requests (a geometry size, a model, a simulated duration, a pacing site) arrive
over time.  The server keeps one FP32 :class:`BatchedEngine` on the GPU and,
between launches,

* admits waiting requests in arrival order while their device footprint fits
  the HBM budget and fewer than ``max_active`` run (FIFO: the head of the
  queue is never overtaken; a few hundred instances at once would leave each
  one or two CTAs and spend the launch on team barriers);
* advances every admitted instance by ``steps_per_launch`` steps in one
  persistent launch (instances of different sizes and models share it, each
  with its own team of CTAs, so new requests overlap with running ones);
* retires instances that reached their last step: gathers the whole 1 kHz Vm
  history into the caller's voxel order on the device, copies it to the host
  through pinned staging buffers and frees the instance (a request's latency
  ends when its history is there).  With ``async_download`` the instance is
  freed right after the gather and the copy runs on a worker thread on its own
  stream while the engine keeps running;
* re-splits CTAs over the running instances by measured cost every
  ``rebalance_every`` launches (the device phase timers run only in the launch
  before each re-split).

Request inputs are compiled on host threads while the GPU runs.  Because the
engine's reductions do not depend on team size or batch-mates, every result is
bit-identical to running the same request alone.
"""
import math
import threading
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import _lib, workloads
from .engine import BatchedEngine


class Request:
    def __init__(self, rid, arrival_s, n_target, duration_ms, model, seed):
        self.rid = rid
        self.arrival_s = arrival_s
        self.n_target = int(n_target)
        self.duration_ms = float(duration_ms)
        self.model = int(model)
        self.seed = int(seed)
        self.inst = None
        self.future = None
        self.admit_s = None
        self.done_s = None
        self.slot = None
        self.history = None
        self.history_bytes = 0
        self.status = None
        self.payload = None        # the request's geometry and parameters (prepare_payloads)


def poisson_requests(count, rate_per_s=20.0, n_min=20_000, n_max=1_000_000, dur_ms=(200.0, 2000.0), seed=0):
    """Seeded request list: Poisson arrivals, log-uniform sizes, uniform
    durations, random model (0 MS / 1 AP) and pacing site (per-request seed)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_per_s, size=count))
    n = np.exp(rng.uniform(np.log(n_min), np.log(n_max), size=count))
    d = rng.uniform(dur_ms[0], dur_ms[1], size=count)
    m = rng.integers(0, 2, size=count)
    return [Request(i, float(t[i]), n[i], d[i], m[i], seed * 100_003 + i) for i in range(count)]


def _payload_one(args):
    i, n_target, seed, t_phys = args
    return workloads.shell_payload(i, n_target, seed, t_phys=t_phys)


def prepare_payloads(reqs, workers=None):
    """Attach to each request what a client sends: its voxel coordinates, scar
    conductivities, pacing site and parameter dicts (seeded synthetic shells,
    made in a process pool; no tables).  The server's builder then only runs
    the device compilation."""
    import multiprocessing as mp
    import os
    from concurrent.futures import ProcessPoolExecutor
    jobs = [(2 * (r.seed % 1000) + r.model, r.n_target, r.seed // 1000, r.duration_ms) for r in reqs]
    workers = workers or min(len(jobs), max(1, (os.cpu_count() or 2) - 1), 32)
    if workers <= 1:
        out = [_payload_one(j) for j in jobs]
    else:
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            out = list(ex.map(_payload_one, jobs, chunksize=4))
    for r, p in zip(reqs, out):
        r.payload = p


_tls = threading.local()


def build(req, tol=1e-7, restart=20, device=False):
    """Compile a request into an FP32 early-exit instance (shell geometry with
    scar).  ``device``: neighbour table, P_2d and operator tables on the GPU,
    on a stream of the calling builder thread (same instance as the host path);
    from the request's payload when it carries one."""
    i = 2 * (req.seed % 1000) + req.model        # parity of i selects the model in shell_case
    if device and req.payload is not None:
        import torch
        if getattr(_tls, "stream", None) is None:
            _tls.stream = torch.cuda.Stream()
        with torch.cuda.stream(_tls.stream):
            return workloads.compile_payload(req.payload, tol=tol, restart=restart, stream=_tls.stream)
    if device:
        import torch
        if getattr(_tls, "stream", None) is None:
            _tls.stream = torch.cuda.Stream()
        with torch.cuda.stream(_tls.stream):
            inst, _ = workloads.shell_case_device(i, req.n_target, req.seed // 1000, t_phys=req.duration_ms, tol=tol,
                                                  restart=restart, stream=_tls.stream)
        return inst
    inst, _, meta = workloads.shell_case(i, req.n_target, req.seed // 1000, t_phys=req.duration_ms, tol=tol,
                                         restart=restart)
    return inst


def footprint_bytes(inst):
    """Device bytes of an FP32 instance (tables incl. the compact neighbour
    table, state, Krylov basis, partials: per voxel of the length padded to
    1024 voxels; history: per voxel)."""
    n = inst.n_voxel
    n_pad = math.ceil(n / 1024) * 1024
    m = min(inst.restart, n)
    tiles = math.ceil(n / 512)
    cb = 5 if getattr(inst, "cw", None) is not None else 24
    eb = 72 if getattr(inst, "coef_edge", None) is not None else 0
    per_voxel = 24 + 8 + cb + eb + 1 + 5 * 4 + (m + 1) * 4 + 4 + (4 if inst.guess else 0)
    hist = n * inst.n_samples * 4 * (2 if inst.save_h else 1)
    return n_pad * per_voxel + hist + tiles * 8 * (m + 2) * 8 + inst.n_steps + 64 * 1024


class _Inline:
    """Executor that builds requests synchronously (build_threads=0)."""

    def submit(self, fn, *a):
        from concurrent.futures import Future
        f = Future()
        f.set_result(fn(*a))
        return f

    def shutdown(self, wait=True):
        pass


class Server:
    def __init__(self, hbm_budget_bytes, steps_per_launch=50, rebalance_every=8, build_threads=8, tol=1e-7,
                 stream=None, engine=None, builder=None, footprint=None, device_build=False, max_active=64,
                 async_download=False):
        self.budget = int(hbm_budget_bytes)
        self.max_active = int(max_active)
        self.S = int(steps_per_launch)
        self.rebalance_every = int(rebalance_every)
        self.tol = tol
        self.builder = builder or (lambda r: build(r, self.tol, device=device_build))
        self.footprint = footprint or footprint_bytes
        if engine is None:
            engine = BatchedEngine(_lib.PREC_F32)
            engine.configure(auto_balance=False)      # the server re-splits the CTAs itself
        self.engine = engine
        self.pool = ThreadPoolExecutor(max_workers=build_threads) if build_threads > 0 else _Inline()
        # retired histories: gathered on the device, the instance freed, and the
        # copy to the host made on this worker while the engine keeps running
        self.async_download = bool(async_download) and hasattr(self.engine, "history_device")
        self.dl = ThreadPoolExecutor(max_workers=1) if self.async_download else None
        self._dl_tls = threading.local()
        self._used_lock = threading.Lock()
        self.stream = stream
        self.used = 0
        self.launches = 0

    def run(self, requests, keep_history=False, time_scale=1.0, log=None):
        """Serve ``requests`` (arrival times in seconds, scaled by ``time_scale``)
        against the wall clock.  Returns per-request records and totals."""
        reqs = sorted(requests, key=lambda r: r.arrival_s)
        for r in reqs:
            r.future = self.pool.submit(self.builder, r)
        queue = deque()
        active = {}
        done = []
        t0 = time.perf_counter()
        nxt = 0
        work = 0.0
        dev_dl = hasattr(self.engine, "history_host")
        downloading = []
        while nxt < len(reqs) or queue or active:
            now = time.perf_counter() - t0
            while nxt < len(reqs) and reqs[nxt].arrival_s * time_scale <= now:
                queue.append(reqs[nxt])
                nxt += 1
            # FIFO admission under the HBM budget
            while queue:
                r = queue[0]
                if not r.future.done() and active:
                    break                                  # head still compiling; keep the GPU busy
                inst = r.future.result()
                fp = self.footprint(inst)
                with self._used_lock:
                    used = self.used
                if active and (used + fp > self.budget or len(active) >= self.max_active):
                    break
                queue.popleft()
                r.inst = inst
                r.slot = self.engine.add(inst)
                if hasattr(inst, "release_tables"):
                    inst.release_tables()          # the engine holds its own copy
                r.admit_s = time.perf_counter() - t0
                r.fp = fp
                with self._used_lock:
                    self.used += fp
                active[r.slot] = r
                if log:
                    log(f"admit {r.rid} n={inst.n_voxel} steps={inst.n_steps} t={r.admit_s:.2f}")
            if not active:
                if nxt < len(reqs):
                    time.sleep(max(0.0, min(0.05, reqs[nxt].arrival_s * time_scale - now)))
                continue
            # phase timers only for the launch whose costs the next re-split uses
            due = (self.launches + 1) % self.rebalance_every == 0
            if due:
                self.engine.set_profile(True)
            self.engine.advance(self.S, stream=self.stream, sync=True)
            self.launches += 1
            if due:
                self.engine.rebalance()
                self.engine.set_profile(False)
            for slot in list(active):
                info = self.engine.info(slot)
                if info["step"] >= info["n_steps"] or info["status"] == _lib.PHS_ERR_NONFINITE:
                    r = active.pop(slot)
                    r.status = info["status"]
                    work += float(r.inst.n_voxel) * info["step"]
                    # the whole 1 kHz Vm history, to the host (caller order made on the device)
                    if self.async_download:
                        import torch
                        hdev = self.engine.history_device(slot)
                        torch.cuda.current_stream().synchronize()   # gathered before the instance goes
                        self.engine.remove(slot)
                        # its footprint stays booked until the gathered copy is on the host
                        r.dl_future = self.dl.submit(self._download, r, hdev, keep_history, t0, time_scale, log)
                        downloading.append(r)
                        continue
                    hist = self.engine.history_host(slot) if dev_dl else self.engine.history(slot)
                    r.history_bytes = hist.nbytes
                    r.history = hist if keep_history else None
                    r.done_s = time.perf_counter() - t0
                    self.engine.remove(slot)
                    with self._used_lock:
                        self.used -= r.fp
                    done.append(r)
                    if log:
                        log(f"done {r.rid} latency={r.done_s - r.arrival_s * time_scale:.2f}s")
        for r in downloading:
            r.dl_future.result()
            done.append(r)
        makespan = time.perf_counter() - t0
        return done, {"makespan_s": makespan, "voxel_steps": work, "launches": self.launches}

    def _download(self, r, hdev, keep_history, t0, time_scale, log):
        """Worker: copy a retired request's gathered history to the host (its
        own pinned staging and stream); the request's latency ends here."""
        from .engine import tensor_to_host
        import torch
        tl = self._dl_tls
        if getattr(tl, "stream", None) is None:
            tl.stream = torch.cuda.Stream(hdev.device)
            tl.stage = None
        hist, tl.stage = tensor_to_host(hdev, tl.stage, stream=tl.stream)
        del hdev
        with self._used_lock:
            self.used -= r.fp
        r.history_bytes = hist.nbytes
        r.history = hist if keep_history else None
        r.done_s = time.perf_counter() - t0
        if log:
            log(f"done {r.rid} latency={r.done_s - r.arrival_s * time_scale:.2f}s")

    def close(self):
        self.pool.shutdown(wait=True)
        if self.dl is not None:
            self.dl.shutdown(wait=True)
        self.engine.close()


def summarize(done, totals, requests, time_scale=1.0):
    lat = np.array([r.done_s - r.arrival_s * time_scale for r in done])
    wait = np.array([r.admit_s - r.arrival_s * time_scale for r in done])
    span = max(r.arrival_s for r in requests) * time_scale if requests else 0.0
    offered = sum(r.inst.n_voxel * r.inst.n_steps for r in done) / max(span, 1e-9)
    return {"requests": len(done), "latency_to": "the whole 1 kHz Vm history on the host",
            "history_bytes": int(sum(r.history_bytes for r in done)),
            "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "p50_queue_s": float(np.percentile(wait, 50)),
            "throughput_voxel_steps_s": totals["voxel_steps"] / totals["makespan_s"],
            "offered_voxel_steps_s": offered, "makespan_s": totals["makespan_s"],
            "launches": totals["launches"], "arrival_span_s": span,
            "failed": int(sum(1 for r in done if r.status == _lib.PHS_ERR_NONFINITE))}
