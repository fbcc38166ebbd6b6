#!/usr/bin/env python3
"""Benchmark of the PyHeartSim B200 hot path.

Metric: voxel-steps/s of the batched FP32 engine (one voxel advanced by one dt,
reaction + Crank-Nicolson diffusion) on the batched configuration: 64 seeded
shells with 50k-400k voxels each (log-uniform, ~10.9M voxels), scar, focal
pacing, half Mitchell-Schaeffer / half Aliev-Panfilov.  One bench "step" is
one dt for every instance.  Inputs (10.9M voxels x ~160 B of state and
solver workspace, ~1.7 GB) are larger than the 126 MB L2, so no flush is
needed between steps.

    python bench.py [--gpus N --steps K --warmup W]      # this build (B200)
    python bench.py --impl reference                     # CPU port of the reference's stepper

Under torchrun each rank runs its own batch (seeds offset by rank: weak
scaling, no data-path collective); the timed region is bracketed by a barrier
and the MAX over ranks is reported.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "voxel-steps/s batched FP32 vs plain FP64 on 1 B200 at LAT err<=dt; p99 latency"
DEFAULT_F32_VARIANT = 2        # the engine's FP32 default when the autotuner is off
# DRAM bytes per voxel-step of step_kernel measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum of the two timed full-size launches of this batch, 2.71
# Arnoldi steps per step, profiles/step_kernel_64shells_dram_fullsize.md), for
# the variants that read the int32 neighbour table and those that read the
# compact one; multiplied by the voxels and steps of one launch below.
STEP_TRAFFIC_BYTES_PER_VOXEL_STEP = {"int32": 267.0, "compact": 201.0}
STEP_TRAFFIC_ARNOLDI_PER_STEP = 2.71
BALANCE_LAUNCHES = 10   # launches per team-balancing round in the pre-steps
WORKLOAD = "64 shells, 50k-400k voxels log-uniform, scar 0-30%, focal pacing, MS+AP, FP32 state / FP64 dots"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=40)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--steps-per-launch", type=int, default=10)
    p.add_argument("--pre-steps", type=int, default=1000,
                   help="steps run before warm-up so the timed window covers propagating fronts")
    p.add_argument("--instances", type=int, default=64)
    p.add_argument("--n-min", type=int, default=50_000)
    p.add_argument("--n-max", type=int, default=400_000)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--tol", type=float, default=1e-7)
    p.add_argument("--t-phys", type=float, default=500.0, help="simulated ms per instance")
    p.add_argument("--no-extras", action="store_true", help="skip e2e, plain-FP64, accuracy and CPU legs")
    p.add_argument("--no-accuracy", action="store_true", help="skip the accuracy leg (c1, c2, c3 sample)")
    p.add_argument("--c2-walls", type=int, nargs="*", default=[3, 8], help="wall thicknesses of the c2 runs")
    p.add_argument("--accuracy-only", action="store_true", help="run only the accuracy leg")
    p.add_argument("--no-tune", action="store_true", help="use the default step-kernel variant")
    p.add_argument("--variant", type=int, default=None,
                   help="run this step-kernel variant (with --ctas-per-sm) instead of tuning (profiling cases)")
    p.add_argument("--ctas-per-sm", type=int, default=0)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--serving-requests", type=int, default=300)
    p.add_argument("--egm-nv", type=int, default=500_000)
    p.add_argument("--egm-ne", type=int, default=2048)
    p.add_argument("--egm-T", type=int, default=1000)
    p.add_argument("--egm-only", action="store_true", help="run only the electrogram leg (profiling case)")
    p.add_argument("--aniso-only", action="store_true", help="run only the anisotropic (fibre) leg")
    p.add_argument("--aniso-instances", type=int, default=16)
    p.add_argument("--geometry-only", action="store_true", help="run only the geometry-preparation leg")
    p.add_argument("--plain-only", action="store_true", help="run only the plain-FP64 leg (profiling case)")
    p.add_argument("--serving-only", action="store_true", help="run only the two serving legs")
    p.add_argument("--serving-async", action="store_true",
                   help="retire served requests with the history copied on a worker thread (comparison runs)")
    return p.parse_args()


# ----------------------------------------------------------------- helpers
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        out.update(sm_mhz=float(np.median(sm)) if sm else None, sm_max_mhz=max(mx) if mx else None,
                   reasons=reasons, samples=len(rows))
        return out


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "of measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "of fallback"


# ----------------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's CPU stepper (port of legacy/compute_simulation_cpu.py)
    on one instance of the batch, on all host cores."""
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return 0
    from oracle import legacy_cpu
    from pyheartsim_b200 import workloads
    sizes = workloads.batch_sizes(args.instances, args.n_min, args.n_max, args.seed)
    i = int(np.argsort(sizes[0::2])[len(sizes[0::2]) // 2]) * 2       # median Mitchell-Schaeffer instance
    _, ref_args, meta = workloads.shell_case(i, int(sizes[i]), args.seed, tol=args.tol)
    run = legacy_cpu.LegacyRun(*ref_args, pacing_duration=meta["pacing_ms"])
    for _ in range(max(args.warmup, 3)):
        run.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        run.step()
    dt = time.perf_counter() - t0
    v = meta["n"] * args.steps / dt
    cores = legacy_cpu.threads()
    line = {"metric": METRIC, "impl": "reference", "value": v, "unit": "voxel-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": f"instance {i} ({meta['n']} voxels, Mitchell-Schaeffer)",
                       "solver": "legacy RK4 (numba parallel) + SciPy BiCGSTAB atol 1e-6"},
            "cpu_baseline": {"value": v, "unit": "voxel-steps/s", "cores": cores, "kind": "port",
                             "sample": f"{args.steps} steps of instance {i} ({meta['n']} voxels)"},
            "e2e": {"value": v, "unit": "voxel-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------- this build
def run_b200(args):
    import torch
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    from pyheartsim_b200 import _lib, geometry_gpu, roofline, workloads
    from pyheartsim_b200.engine import BatchedEngine

    seed = args.seed + 7919 * rank
    # reference-style inputs (P_2d, neighbour table, parameter dicts) built on
    # host processes, compiled into engine instances on the device
    cases = workloads.batched_inputs(args.instances, args.n_min, args.n_max, seed, t_phys=args.t_phys)
    insts = [compile_case(c, m, args.tol) for c, m in cases]
    ns = np.array([m["n"] for _, m in cases], dtype=np.int64)
    S = max(1, args.steps_per_launch)
    K = max(1, args.steps)
    W = max(3, args.warmup)

    def launches_of(count):
        """Launch sizes covering exactly ``count`` steps: full launches of S
        steps, then the remainder."""
        return [S] * (count // S) + ([count % S] if count % S else [])
    stream = torch.cuda.current_stream(dev)

    pre = (args.pre_steps // S) * S
    tune = None
    if args.variant is not None:
        tune = {"best": (args.variant, args.ctas_per_sm), "fixed": True}
    elif not args.no_tune:
        # tuned on a copy of the batch advanced to the timed window's start, so
        # the options are compared mid-propagation and the timed run below
        # covers the same simulated steps whatever the number of options
        from pyheartsim_b200 import autotune
        eng_t = BatchedEngine(_lib.PREC_F32)
        for x in insts:
            eng_t.add(x)
        for _ in range(pre // S):
            eng_t.advance(S, stream=stream, sync=False)
        tune = autotune.tune(eng_t, steps=S, stream=stream)
        eng_t.close()
    eng = BatchedEngine(_lib.PREC_F32)
    slots = [eng.add(x) for x in insts]
    for x in insts:
        x.release_tables()
    if tune is not None:
        eng.configure(variant=tune["best"][0], ctas_per_sm=tune["best"][1])
    # team sizes from each instance's measured cost: the last BALANCE_LAUNCHES x
    # 3 launches of the (untimed) pre-steps run with the phase timers on, in
    # three rounds that each re-split the CTAs by the cost measured in the
    # round before (windows of 100 steps: the Arnoldi counts of single steps
    # vary a lot); then W warm-up steps on the final plan (graph capture)
    rounds = 3
    bal = min(BALANCE_LAUNCHES, max(1, (pre // S) // (rounds + 1)))
    for _ in range(pre // S - rounds * bal):
        eng.advance(S, stream=stream, sync=False)
    eng.set_profile(True)
    for _ in range(rounds):
        eng.rebalance()
        for _ in range(bal):
            eng.advance(S, stream=stream, sync=False)
    eng.rebalance()
    eng.set_profile(False)
    for k in launches_of(W):
        eng.advance(k, stream=stream, sync=False)
    torch.cuda.synchronize(dev)
    info0 = [eng.info(s) for s in slots]
    launches0 = eng.launches()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for k in launches_of(K):
        eng.advance(k, stream=stream, sync=False)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    barrier()
    ms = ev0.elapsed_time(ev1)
    ms_max = ms
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    launches = eng.launches() - launches0
    info1 = [eng.info(s) for s in slots]
    for a, b in zip(info0, info1):
        assert b["step"] - a["step"] == K, "an instance finished inside the timed window"
        assert b["status"] in (0, _lib.PHS_WARN_NO_CONVERGE), f"instance status {b['status']}"
    k_sum = np.array([b["arnoldi_steps"] - a["arnoldi_steps"] for a, b in zip(info0, info1)], dtype=np.float64)
    k_sq = np.array([b["arnoldi_sq"] - a["arnoldi_sq"] for a, b in zip(info0, info1)], dtype=np.float64)
    solves = np.array([b["solves"] - a["solves"] for a, b in zip(info0, info1)], dtype=np.float64)
    iso = [x.cw is not None for x in insts]
    gs = [bool(x.guess) for x in insts]
    # neighbour-table bytes per row: the compact table where the variant reads it
    from pyheartsim_b200.engine import step_variant_layout
    reads_compact = step_variant_layout(_lib.PREC_F32)[step_variant_of(tune)][1]
    nbb = [roofline.COMPACT_NB if (reads_compact and eng.table_bytes(s) == 8) else 24 for s in slots]
    alg_bytes = float(sum(roofline.algorithmic_bytes(4, int(n), K, ks, kq, sv, io, g, nb=nb)
                          for n, ks, kq, sv, io, g, nb in zip(ns, k_sum, k_sq, solves, iso, gs, nbb)))
    local_vs = float(ns.sum()) * K
    total_vs = local_vs * world
    value = total_vs / (ms_max / 1e3)
    pk, pk_src = peaks()
    achieved = alg_bytes / launches / (ms / launches / 1e3) / 1e9 if launches else 0.0
    # achieved is GB/s of algorithmic bytes per launch over the average launch time
    phases = phase_profile(eng, slots, S, stream)
    eng.close()

    line = {"metric": METRIC, "value": value, "unit": "voxel-steps/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded shells; no patient meshes)",
            "config": {"workload": WORKLOAD, "instances": int(len(ns)), "voxels": int(ns.sum()),
                       "steps_per_launch": S, "pre_steps": pre, "gmres": f"early exit, tol {args.tol}, restart 20",
                       "l2": "inputs larger than L2 (no flush)", "parallelism": f"instance-parallel x{world}"},
            "gpu_launches": int(launches),
            "autotune": None if tune is None else {"variant": tune["best"][0], "ctas_per_sm": tune["best"][1],
                                                   "table": tune.get("table")},
            "solver": {"arnoldi_per_solve": float(k_sum.sum() / max(solves.sum(), 1)),
                       "solves_per_step": float(solves.sum() / (K * len(ns))),
                       "arnoldi_per_step": float(k_sum.sum() / (K * len(ns)))},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / pk["hbm_gbs"], "peak_source": pk_src,
                         "traffic": STEP_TRAFFIC_BYTES_PER_VOXEL_STEP["compact" if reads_compact else "int32"]
                         * float(ns.sum()) * S,
                         "traffic_source": ("ncu dram__bytes_read+write per voxel-step of full-size launches of this "
                                            f"batch ({STEP_TRAFFIC_ARNOLDI_PER_STEP} Arnoldi steps per step) x voxels "
                                            "x steps per launch"),
                         "kernel": step_kernel_name(tune),
                         "bytes_per_voxel_step": alg_bytes / local_vs},
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]},
            "phases_ms_per_step": phases}

    if not args.no_extras:
        del insts
        line["e2e"] = e2e_leg(args, cases, dev)
        if rank == 0 and world == 1:
            line["e2e_dropin_c1"] = dropin_c1_leg(dev)
            line["plain_fp64"] = plain_leg(args, cases, value, dev)
            if not args.no_accuracy:
                line["accuracy"] = accuracy_leg(dev, args.tol, walls=tuple(args.c2_walls))
            line["anisotropic"] = aniso_leg(args, dev, tune, count=args.aniso_instances)
            line["geometry"] = geometry_leg(args, dev)
            del cases
            line["serving"] = serving_leg(args, dev, count=args.serving_requests)
            # latency below saturation: Poisson arrivals offering half the batched
            # throughput, same time compression
            line["serving_half_load"] = serving_leg(args, dev, count=max(50, args.serving_requests // 3),
                                                    load=(0.5, value), plain_subset=0)
            line["electrogram"] = egm_leg(args, dev)
            line["cpu_baseline"] = cpu_leg(args)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def step_variant_of(tune):
    return tune["best"][0] if tune is not None else DEFAULT_F32_VARIANT


def step_kernel_name(tune):
    """Template arguments (value type, voxels per thread, minimum CTAs per SM,
    edge terms, staging ring bytes, compact table) of the step-kernel variant
    the timed launches used."""
    from pyheartsim_b200.engine import step_variants, step_variant_layout
    from pyheartsim_b200 import _lib
    var = {v: (minb, vpt) for v, minb, _, vpt in step_variants(_lib.PREC_F32, with_vpt=True)}
    lay = step_variant_layout(_lib.PREC_F32)
    v = step_variant_of(tune)
    minb, vpt = var[v]
    ring, comp = lay[v]
    return f"step_kernel<float,{vpt},{minb},false,{ring},{str(comp and ring == 0).lower()}>"


def phase_profile(eng, slots, S, stream):
    """Device phase timers (first CTA of each team) over 2*S extra steps after the
    timed region, averaged over instances: ms per step spent in each phase."""
    import torch
    eng.set_profile(True)
    eng.advance(2 * S, stream=stream, sync=True)
    torch.cuda.synchronize()
    acc = {}
    totals = []
    per = []
    for s in slots:
        p = eng.profile(s)
        st = max(p.pop("steps"), 1)
        it = p.pop("arnoldi_iters")
        team = p.pop("team_ctas")
        lead = p.pop("leader", 0.0)          # leader bodies, on the team's critical path
        nbar = p.pop("barriers", 0)
        acc["leader"] = acc.get("leader", 0.0) + lead / st
        acc["barriers_per_step"] = acc.get("barriers_per_step", 0.0) + nbar / st
        inst = eng.instance(s)
        per.append([int(inst.n_voxel), int(inst.model), int(team), round(it / st, 2),
                    round(sum(p.values()) / st, 4), round(p["rhs_reaction"] / st, 4), round(p["rhs"] / st, 4)])
        for k, v in p.items():
            acc[k] = acc.get(k, 0.0) + v / st
        acc["arnoldi_iters_per_step"] = acc.get("arnoldi_iters_per_step", 0.0) + it / st
        totals.append(sum(p.values()) / st)
    eng.set_profile(False)
    out = {k: round(v / len(slots), 5) for k, v in acc.items()}
    out["team_ms_per_step_min"] = round(min(totals), 5)
    out["team_ms_per_step_max"] = round(max(totals), 5)
    # CTA-weighted busy fraction of the launch: teams that finish their steps
    # early leave their CTAs idle until the slowest team is done
    teams = np.array([r[2] for r in per], dtype=np.float64)
    busy = np.array(totals)
    out["cta_utilization"] = round(float((teams * busy).sum() / (teams.sum() * busy.max())), 4)
    out["per_instance"] = sorted(per, key=lambda r: -r[4])[:12]
    return out


def compile_case(case, meta, tol, stream=None):
    """Engine instance of one reference-style input set, compiled on the device
    (FP32 early exit at ``tol``, restart 20, 1 kHz Vm history)."""
    from pyheartsim_b200 import geometry_gpu
    return geometry_gpu.compile_reference_inputs(*case, full_cycles=False, tol=tol, atol=1e-5, restart=20,
                                                 save_h=False, pacing_duration=meta["pacing_ms"] / case[3]["time_scale"],
                                                 stream=stream)


def e2e_leg(args, cases, dev):
    """The whole batched job through the public API, from the reference-style
    inputs on the host (P_2d, neighbour table, voxel coordinates and parameter
    dicts of every instance) to every instance's full 1 kHz Vm history and
    final state on the host: upload and device compilation of the tables,
    every instance run to its last step (500 ms: 10,000 steps for
    Mitchell-Schaeffer, 25,000 for Aliev-Panfilov) with graph-replayed launches
    on a CUDA stream, download.  Wall time of each part."""
    import torch
    from pyheartsim_b200 import _lib
    from pyheartsim_b200.engine import BatchedEngine
    stream = torch.cuda.Stream(dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        insts = [compile_case(c, m, args.tol, stream=stream) for c, m in cases]
    eng = BatchedEngine(_lib.PREC_F32)
    slots = [eng.add(x) for x in insts]
    for x in insts:
        x.release_tables()
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    h2d = sum(c[1].nbytes + np.asarray(c[2]['neighbor_id_2d']).size * 4 + np.asarray(c[2]['voxel']).nbytes
              for c, _ in cases)
    S = 10 * max(1, args.steps_per_launch)
    steps_total = max(x.n_steps for x in insts)
    # histories of instances that have finished are gathered into caller order
    # on the device and copied to the host on a worker thread (pinned staging,
    # its own stream) while the engine runs the others
    from concurrent.futures import ThreadPoolExecutor
    from pyheartsim_b200.engine import tensor_to_host
    pool = ThreadPoolExecutor(max_workers=1)
    ctx = {}

    def copy_out(t):
        if "stream" not in ctx:
            ctx["stream"] = torch.cuda.Stream(dev)
            ctx["stage"] = None
        out, ctx["stage"] = tensor_to_host(t, ctx["stage"], stream=ctx["stream"])
        return out

    pending = {}
    d2h = 0
    during = 0

    def collect(running):
        nonlocal d2h, during
        for s in slots:
            if s in pending or not eng.finished(s):
                continue
            u, h, lat = eng.state(s)
            hdev = eng.history_device(s, stream=stream)
            stream.synchronize()
            pending[s] = pool.submit(copy_out, hdev)
            nbytes = hdev.numel() * hdev.element_size() + u.nbytes + h.nbytes + lat.nbytes
            d2h += nbytes
            if running:
                during += nbytes
    k = 0
    while not all(eng.finished(s) for s in slots):
        for _ in range(10):
            eng.advance(S, stream=stream, sync=False)
        eng.advance(S, stream=stream, sync=True)     # refresh the finished flags: finished instances leave the plan
        k += 11
        collect(running=not all(eng.finished(s) for s in slots))
    t2 = time.perf_counter()
    collect(running=False)
    for s in slots:
        pending[s].result()
    pool.shutdown(wait=True)
    t3 = time.perf_counter()
    vs = float(sum(x.n_voxel * x.n_steps for x in insts))
    eng.close()
    return {"value": vs / (t3 - t0), "unit": "voxel-steps/s", "h2d_bytes_per_step": h2d / steps_total,
            "d2h_bytes_per_step": d2h / steps_total, "voxel_steps": vs, "steps_longest_instance": int(steps_total),
            "seconds": t3 - t0, "compile_upload_s": t1 - t0, "run_s": t2 - t1, "download_after_run_s": t3 - t2,
            "d2h_bytes_while_running": int(during), "launches": int(k), "run_only_value": vs / (t2 - t1),
            "path": "reference-style inputs on the host -> device compile (geometry_gpu.compile_reference_inputs) "
                    "-> engine, graph replay on a stream -> full 1 kHz history and final state on the host "
                    "(histories gathered into caller order on the device as instances finish, copied through "
                    "pinned staging on a worker thread while the others run)"}


def dropin_c1_leg(dev):
    """The drop-in call itself (simulation_gpu.compute, then
    unipolar_electrogram_gpu.compute) on the plain sheet: 200 x 200 voxels,
    500 ms = 10,000 steps, 16 electrodes; host inputs in, host arrays out, wall
    time per call.  Plain FP64 (the reference's GMRES(50) full cycles) and the
    FP32 early-exit form."""
    from pyheartsim_b200 import workloads
    from pyheartsim_b200.simulation import simulation_gpu, unipolar_electrogram_gpu
    (n, P, geom, sp, ap), pdur, el = workloads.sheet_c1()
    out = {"voxels": int(n), "steps": 10000, "electrodes": int(el.shape[0])}
    for name, kw in (("plain_fp64", {}), ("fast_fp32", dict(dtype=np.float32, fast=True, tol=1e-7))):
        t0 = time.perf_counter()
        u, h, t = simulation_gpu.compute(n, P, geom, dict(sp), dict(ap), pacing_duration=pdur, **kw)
        t1 = time.perf_counter()
        mode = "fp64" if name == "plain_fp64" else "bf16x3"
        egm = unipolar_electrogram_gpu.compute(el, geom['voxel'], None, P[:, 20], u, geom['Delta'],
                                               geom['neighbor_id_2d'], mode=mode)
        t2 = time.perf_counter()
        out[name] = {"simulate_s": t1 - t0, "voxel_steps_per_s": n * 10000 / (t1 - t0), "electrogram_s": t2 - t1,
                     "electrogram_mode": mode, "history_shape": list(u.shape)}
    return out


def plain_leg(args, cases, fast_value, dev):
    """Plain FP64 drop-in semantics (full GMRES(50) cycles, FP64) on the median
    instance of the batch, one instance on the whole GPU: throughput, the byte
    model's roofline (k = m = 50 Arnoldi steps per cycle, one true-residual test
    per cycle) and the device phase times."""
    import torch
    from pyheartsim_b200 import _lib, roofline, workloads
    from pyheartsim_b200.engine import BatchedEngine
    ns = np.array([m["n"] for _, m in cases])
    i = int(np.argsort(ns)[len(ns) // 2])
    meta = cases[i][1]
    sizes = workloads.batch_sizes(args.instances, args.n_min, args.n_max, args.seed)
    inst, _, _ = workloads.shell_case(i, int(sizes[i]), args.seed, fast=False)
    eng = BatchedEngine(_lib.PREC_F64)
    slot = eng.add(inst)
    stream = torch.cuda.current_stream(dev)
    pre = min(args.pre_steps, 400)
    eng.advance(pre, stream=stream, sync=True)
    steps = 20
    info0 = eng.info(slot)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    eng.advance(steps, stream=stream, sync=False)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms = ev0.elapsed_time(ev1)
    info = eng.info(slot)
    k_sum = info["arnoldi_steps"] - info0["arnoldi_steps"]
    k_sq = info["arnoldi_sq"] - info0["arnoldi_sq"]
    cycles = k_sum / 50.0
    alg = roofline.algorithmic_bytes(8, meta["n"], steps, k_sum, k_sq, iso=inst.cw is not None, checks=cycles)
    # device phase times over 4 more steps
    eng.set_profile(True)
    eng.advance(4, stream=stream, sync=True)
    prof = eng.profile(slot)
    eng.close()
    st = max(prof.pop("steps"), 1)
    prof.pop("team_ctas", None)
    it = prof.pop("arnoldi_iters")
    nbar = prof.pop("barriers", 0)
    pk, pk_src = peaks()
    achieved = alg / (ms / 1e3) / 1e9
    v = meta["n"] * steps / (ms / 1e3)
    return {"value": v, "unit": "voxel-steps/s", "instance": i, "voxels": int(meta["n"]), "steps": steps,
            "ms_per_step": ms / steps, "arnoldi_per_step": k_sum / steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / pk["hbm_gbs"], "peak_source": pk_src,
                         "bytes_per_voxel_step": alg / (meta["n"] * steps),
                         "note": "the 51-column FP64 Krylov basis of this instance fits in L2"},
            "phases_ms_per_step": {**{k: round(v_ / st, 4) for k, v_ in prof.items()},
                                   "barriers_per_step": round(nbar / st, 2)},
            "speedup_batched_fp32": (fast_value / v) if fast_value else None}


def geometry_leg(args, dev, n_target=1_000_000, reps=3):
    """Instance preparation for one seeded ~1M-voxel scarred fibre shell: the
    host path (vectorised numpy neighbour table, P_2d and table compilation)
    against the device path (phs_lattice_neighbors, phs_equation_parts,
    phs_operator_tables, instance add from device tables).  Wall time with the
    device synchronised; the device path's best of ``reps``."""
    import torch
    from pyheartsim_b200 import _lib, geometry, geometry_gpu, instance, synthetic
    from pyheartsim_b200.engine import BatchedEngine
    ijk = synthetic.shell_for_size(n_target, seed=args.seed + 5)
    n = ijk.shape[0]
    rng = np.random.default_rng(args.seed)
    c_scale = synthetic.scar(ijk, geometry.lattice_neighbors(ijk), 0.15, rng)
    D0 = synthetic.fibre_tensors(ijk)
    par = synthetic.model_parameters(0, n, np.full(n, 1.0) * c_scale)
    sp = {'t_final': 100.0, 'dt': 0.05, 'heart_model_flag': 0, 'arrhythmia_flag': 4, 'time_scale': 1}
    ap = {'pacing_start_time': 10.0, 'pacing_cycle_length': 300.0, 's1_pacing_voxel_id': np.arange(20),
          's2_pacing_voxel_id': np.zeros(0, np.int64), 's1_t': 0.0, 's1_s2_delta_t': 0.0,
          'node_flag': np.zeros(n, dtype=np.int64)}
    kw = dict(full_cycles=False, tol=1e-7, restart=20, pacing_duration=2.0)
    voxel = ijk * 0.4
    t0 = time.perf_counter()
    nb = geometry.lattice_neighbors(ijk)
    P = geometry.heart_model_equation_parts(sp, n, D0, nb, par)
    host = instance.compile_instance(n, P, {"neighbor_id_2d": nb, "Delta": 0.4, "voxel": voxel}, sp, ap, **kw)
    t_host = time.perf_counter() - t0
    times = []
    for _ in range(reps):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        inst = geometry_gpu.compile_instance(voxel, 0.4, par, D0, sp, ap, **kw)
        torch.cuda.synchronize(dev)
        times.append(time.perf_counter() - t0)
    eng = BatchedEngine(_lib.PREC_F32)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    eng.add(inst)
    torch.cuda.synchronize(dev)
    t_add_dev = time.perf_counter() - t0
    t0 = time.perf_counter()
    eng.add(host)
    t_add_host = time.perf_counter() - t0
    eng.close()
    return {"voxels": int(n), "workload": "scarred fibre shell, MS, anisotropic D0 (edge terms)",
            "host_numpy_s": t_host, "device_s": min(times), "device_s_all": times,
            "speedup": t_host / min(times), "engine_add_device_tables_s": t_add_dev,
            "engine_add_host_tables_s": t_add_host}


def aniso_leg(args, dev, tune=None, count=16):
    """Anisotropic tensors (rule-based fibre field, every cross term present):
    ``count`` seeded shells of n_min..n_max voxels through the edge-term kernel,
    warmed up and timed like the main batch (CUDA events on the launch stream)."""
    import torch
    from pyheartsim_b200 import _lib, roofline, workloads
    from pyheartsim_b200.engine import BatchedEngine
    batch = workloads.batched_shells(count, args.n_min, args.n_max, args.seed + 11, tol=args.tol,
                                     t_phys=args.t_phys, fibres=True)
    insts = [b[0] for b in batch]
    ns = np.array([m["n"] for _, m in batch], dtype=np.int64)
    eng = BatchedEngine(_lib.PREC_F32)
    if tune is not None:
        eng.configure(variant=tune["best"][0], ctas_per_sm=tune["best"][1])
    slots = [eng.add(x) for x in insts]
    stream = torch.cuda.current_stream(dev)
    S = max(1, args.steps_per_launch)
    for _ in range(max(1, 300 // S)):
        eng.advance(S, stream=stream, sync=False)
    eng.set_profile(True)
    for _ in range(2):
        eng.rebalance()
        eng.advance(S, stream=stream, sync=False)
    eng.rebalance()
    eng.set_profile(False)
    eng.advance(S, stream=stream, sync=False)
    torch.cuda.synchronize(dev)
    info0 = [eng.info(s) for s in slots]
    launches0 = eng.launches()
    K = max(1, 100 // S) * S
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(K // S):
        eng.advance(S, stream=stream, sync=False)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ms = ev0.elapsed_time(ev1)
    launches = eng.launches() - launches0
    info1 = [eng.info(s) for s in slots]
    eng.close()
    for a, b in zip(info0, info1):
        assert b["step"] - a["step"] == K, "an instance finished inside the timed window"
    k_sum = np.array([b["arnoldi_steps"] - a["arnoldi_steps"] for a, b in zip(info0, info1)], dtype=np.float64)
    k_sq = np.array([b["arnoldi_sq"] - a["arnoldi_sq"] for a, b in zip(info0, info1)], dtype=np.float64)
    solves = np.array([b["solves"] - a["solves"] for a, b in zip(info0, info1)], dtype=np.float64)
    alg = float(sum(roofline.algorithmic_bytes(4, int(n), K, ks, kq, sv, x.cw is not None, bool(x.guess), edge=True)
                    for n, ks, kq, sv, x in zip(ns, k_sum, k_sq, solves, insts)))
    pk, pk_src = peaks()
    achieved = alg / (ms / 1e3) / 1e9
    return {"value": float(ns.sum()) * K / (ms / 1e3), "unit": "voxel-steps/s", "instances": int(count),
            "voxels": int(ns.sum()), "steps": int(K), "ms_per_step": ms / K, "gpu_launches": int(launches),
            "arnoldi_per_solve": float(k_sum.sum() / max(solves.sum(), 1)),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / pk["hbm_gbs"], "peak_source": pk_src,
                         "bytes_per_voxel_step": alg / (float(ns.sum()) * K)},
            "fibres": "D0 = 0.3 I + 0.7 e e^T, helix +-60 deg through the wall"}


def accuracy_leg(dev, tol, walls=(3, 8), c3_count=4):
    """The FP32 early-exit path (tol, restart 20, extrapolated guess) against the
    plain FP64 path (the reference's GMRES(50) full cycles, within 1e-9 of the
    FP64 oracle) on the named configurations, over their whole runs, from
    per-step device histories: activation times of every voxel (first and
    re-activations) in units of dt, max |dVm| over the 1 kHz samples, and the
    electrograms' relative L2 errors.

    * c2: the rotor shell (Aliev-Panfilov, S1 plane + S2 quadrant, 1000 ms =
      50,000 steps, 64 electrodes) at each wall thickness in ``walls``;
    * c1: the 200 x 200 Mitchell-Schaeffer sheet, 500 ms, 16 electrodes (its
      plain FP64 run against the FP64 oracle is
      tests/test_gpu_configs.py::test_c1_sheet_full_run_matches_oracle);
    * c3_sample: the ``c3_count`` smallest instances of the benchmark batch,
      half Mitchell-Schaeffer and half Aliev-Panfilov, over their 500 ms."""
    import torch
    from pyheartsim_b200 import accuracy, workloads
    torch.cuda.empty_cache()          # per-step histories of the rotor shell need tens of GB
    out = {"reference": "plain FP64 path (GMRES(50) full cycles)", "test": f"FP32 early exit, tol {tol}"}
    t0 = time.perf_counter()
    case, pdur, el = workloads.sheet_c1()
    out["c1"] = accuracy.compare_case(case, pdur, el, tol=tol)
    out["c1"]["voxels"] = int(case[0])
    for w in walls:
        case, pdur, el = workloads.atrium_c2(wall=w)
        r = accuracy.compare_case(case, pdur, el, tol=tol)
        r["wall_voxels"] = int(w)
        r["s1_mm"], r["s1_s2_ms"] = workloads.C2_PACING.get(w, workloads.C2_PACING[3])
        out[f"c2_wall{w}"] = r
    sizes = workloads.batch_sizes(64, 50_000, 400_000, 0)
    picks = []
    for model in (0, 1):
        idx = [i for i in np.argsort(sizes) if i % 2 == model][:max(1, c3_count // 2)]
        picks += [int(i) for i in idx]
    sample = []
    for i in picks:
        _, case, meta = workloads.shell_case(i, int(sizes[i]), 0)
        r = accuracy.compare_case(case, meta["pacing_ms"] / case[3]["time_scale"], tol=tol)
        sample.append({"instance": i, "model": meta["model"], "voxels": int(case[0]),
                       "first_max_dlat_steps": r["first"]["max_dlat_steps"] if r["first"] else None,
                       "first_voxels_one_run_only": r["first"]["voxels_one_run_only"] if r["first"] else None,
                       "reactivation_max_dlat_steps": max([x["max_dlat_steps"] or 0 for x in r["reactivations"]],
                                                          default=None),
                       "activation_count_equal_frac": r["activation_count_equal_frac"],
                       "max_abs_dvm_1khz": r["max_abs_dvm_1khz"], "steps": r["steps"],
                       "plain_fp64_s": r["plain_fp64_s"], "fast_fp32_s": r["fast_fp32_s"]})
    out["c3_sample"] = sample
    out["seconds"] = time.perf_counter() - t0
    return out


def serving_leg(args, dev, count=300, compress=20.0, rate=20.0, dur_ms=(200.0, 2000.0), load=None,
                plain_subset=4):
    """Continuous batching under Poisson arrivals (20k-1M voxels, random model
    and pacing site), time-compressed: simulated durations divided by
    ``compress`` and the arrival rate multiplied by it, so the offered load in
    voxel-steps/s is that of ``rate`` requests/s of ``dur_ms`` (several times
    what one B200 serves) while ``count`` requests finish in seconds.  Latency
    runs from arrival to the request's whole 1 kHz Vm history on the host.
    ``load = (fraction, capacity)``: instead, the arrival rate whose requests
    offer that fraction of ``capacity`` voxel-steps/s.

    The plain-FP64-serial comparison is measured on the first ``plain_subset``
    requests: each run alone through the plain FP64 path (GMRES(50) full
    cycles), one after another in arrival order, compile to history on the
    host; their FIFO latencies are set beside the same requests' latencies in
    the continuous-batching run."""
    import torch
    from pyheartsim_b200 import _lib, serving, workloads
    from pyheartsim_b200.engine import BatchedEngine
    d = (dur_ms[0] / compress, dur_ms[1] / compress)
    r_eff = rate * compress
    if load is not None:
        frac, capacity = load
        probe = serving.poisson_requests(count, rate_per_s=1.0, dur_ms=d, seed=args.seed)
        # voxel-steps of a request: physical dt 0.05 ms (MS) or 0.02 ms (AP)
        work = np.mean([r.n_target * r.duration_ms / (0.05 if r.model == 0 else 0.02) for r in probe])
        r_eff = frac * capacity / work
    reqs = serving.poisson_requests(count, rate_per_s=r_eff, dur_ms=d, seed=args.seed)
    t_prep = time.perf_counter()
    serving.prepare_payloads(reqs)               # the clients' geometry and parameters (before the clock)
    t_prep = time.perf_counter() - t_prep
    free = torch.cuda.mem_get_info(dev)[0]
    srv = serving.Server(hbm_budget_bytes=int(free * 0.8), steps_per_launch=100,
                         stream=torch.cuda.current_stream(dev).cuda_stream, device_build=True,
                         async_download=args.serving_async)
    done, totals = srv.run(reqs)
    srv.close()
    out = serving.summarize(done, totals, reqs)
    out["builder"] = ("requests carry voxel coordinates, scar conductivities, pacing site and parameter dicts "
                      f"(made before the clock, {t_prep:.1f} s); the server builds neighbour table, P_2d and "
                      "operator tables on the GPU, one stream per builder thread")
    out["arrival_rate_per_s"] = r_eff
    out["durations_ms"] = list(d)
    out["time_compression"] = compress
    out["history_download"] = "worker thread, pinned staging, own stream" if args.serving_async else "synchronous"
    if plain_subset:
        by_id = {r.rid: r for r in done}
        sub = sorted(reqs, key=lambda r: r.arrival_s)[:plain_subset]
        t = 0.0
        rows = []
        for r in sub:
            i = 2 * (r.seed % 1000) + r.model
            t0 = time.perf_counter()
            inst, _, _ = workloads.shell_case(i, r.n_target, r.seed // 1000, t_phys=r.duration_ms, fast=False)
            eng = BatchedEngine(_lib.PREC_F64)
            slot = eng.add(inst)
            while not eng.finished(slot):
                eng.advance(1000)
            eng.history(slot)
            eng.close()
            run_s = time.perf_counter() - t0
            t = max(t, r.arrival_s) + run_s
            rows.append({"rid": r.rid, "voxels": int(inst.n_voxel), "steps": int(inst.n_steps), "run_s": run_s,
                         "plain_serial_latency_s": t - r.arrival_s,
                         "batched_latency_s": by_id[r.rid].done_s - by_id[r.rid].arrival_s})
        out["plain_fp64_serial_subset"] = {
            "requests": rows, "measured": True,
            "voxel_steps_per_s": float(sum(x["voxels"] * x["steps"] for x in rows)
                                       / max(sum(x["run_s"] for x in rows), 1e-9))}
    return out


def egm_leg(args, dev, history=None):
    """Electrogram contraction at its configured size: lead field of n_e seeded
    electrodes 2 mm off an n_v-voxel shell (FP64, on device), Vm history of T
    samples from an S1-S2 run of the FP32 engine, BF16 hi/lo x3 on tcgen05 vs the
    FP64 contraction."""
    import ctypes
    import torch
    from pyheartsim_b200 import _lib, synthetic, workloads
    from pyheartsim_b200.engine import BatchedEngine
    from pyheartsim_b200.geometry import lattice_neighbors
    from pyheartsim_b200.instance import compile_instance
    from pyheartsim_b200.simulation.unipolar_electrogram_gpu import incoming_gradient_terms
    L = _lib.lib()
    rng = np.random.default_rng(args.seed + 4)
    ijk = workloads._shell_scaled(args.egm_nv, args.seed + 4)
    nb = lattice_neighbors(ijk)
    n_v, n_e, T = ijk.shape[0], args.egm_ne, args.egm_T
    xyz = ijk * 0.4
    x = ijk[:, 0]
    s1 = np.where(x <= x.min() + 3)[0]
    s2 = np.where((x < np.median(x)) & (ijk[:, 1] > np.median(ijk[:, 1])))[0]
    case = synthetic.make_case(ijk, 0.4, 0, 0.05, float(T), s1, s2_ids=s2, flag=1, s1_s2=250.0)
    inst = compile_instance(*case, full_cycles=False, tol=1e-7, restart=20, save_h=False)
    eng = BatchedEngine(_lib.PREC_F32)
    slot = eng.add(inst)
    t0 = time.perf_counter()
    while not eng.finished(slot):
        eng.advance(2000, sync=True)
    sim_s = time.perf_counter() - t0
    samples = eng.info(slot)["samples"]
    T = min(T, samples)
    # the history stays on the device: read it back into a torch tensor
    Vf32 = torch.from_numpy(eng.history(slot, 0, T)).to(dev)
    eng.close()
    el = synthetic.electrodes_off_surface(ijk, 0.4, n_e, rng)
    c = torch.tensor(case[1][:, 20], dtype=torch.float64, device=dev)
    ptr, srcv, dirs = incoming_gradient_terms(nb)
    dxyz = torch.tensor(xyz, dtype=torch.float64, device=dev)
    dex = torch.tensor(el, dtype=torch.float64, device=dev)
    dptr = torch.tensor(ptr, device=dev)
    dsrc = torch.tensor(srcv, device=dev)
    ddir = torch.tensor(dirs, device=dev)
    Mt = torch.empty((n_e, n_v), dtype=torch.float64, device=dev)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    ev[0].record(stream)
    _lib.check(L.phs_egm_leadfield_f64(n_v, n_e, p(dxyz), p(dex), p(c), None, p(dptr), p(dsrc), p(ddir),
                                       1.0 / 0.8, p(Mt), sp), "leadfield")
    ev[1].record(stream)
    V64 = Vf32.double()
    ref = torch.empty((T, n_e), dtype=torch.float64, device=dev)
    ev[2].record(stream)
    _lib.check(L.phs_egm_contract_f64(T, n_v, n_e, p(V64), n_v, p(Mt), p(ref), sp), "contract_f64")
    ev[3].record(stream)
    Tp, Ep, Kp = (T + 127) // 128 * 128, (n_e + 127) // 128 * 128, (n_v + 63) // 64 * 64
    vh = torch.empty((Tp, Kp), dtype=torch.uint16, device=dev)
    vl = torch.empty_like(vh)
    mh = torch.empty((Ep, Kp), dtype=torch.uint16, device=dev)
    ml = torch.empty_like(mh)
    _lib.check(L.phs_split_bf16(T, n_v, p(Vf32), n_v, 0, p(vh), p(vl), Tp, Kp, sp), "split V")
    _lib.check(L.phs_split_bf16(n_e, n_v, p(Mt), n_v, 1, p(mh), p(ml), Ep, Kp, sp), "split M")
    work = torch.empty(L.phs_egm_bf16x3_workspace(Tp, Ep, Kp), dtype=torch.uint8, device=dev)
    out = torch.empty((T, n_e), dtype=torch.float32, device=dev)
    reps = 3

    def contract(cfg):
        _lib.check(L.phs_egm_contract_bf16x3_cfg(T, n_e, Tp, Ep, Kp, p(vh), p(vl), p(mh), p(ml), p(out), p(work),
                                                 cfg, sp), "contract_bf16x3")

    # tile configuration from the autotuner (median of 3 timed calls each)
    from pyheartsim_b200 import autotune
    best, cfg_ms = autotune.tune_electrogram(T, n_e, Tp, Ep, Kp, vh, vl, mh, ml, out, work, stream=stream)
    contract(best)
    ev[4].record(stream)
    for _ in range(reps):
        contract(best)
    ev[5].record(stream)
    _lib.check(L.phs_egm_bf16x3_status(p(work), sp), "contract_bf16x3 status")
    torch.cuda.synchronize()
    ms_bf = ev[4].elapsed_time(ev[5]) / reps
    ms_f64 = ev[2].elapsed_time(ev[3])
    flops = 2.0 * T * n_e * n_v
    pk, pk_src = peaks()
    r = ref.cpu().numpy()
    o = out.double().cpu().numpy()
    rel = float(np.linalg.norm(o - r) / np.linalg.norm(r))
    # the same BF16 parts multiplied exactly in FP64: separates the split's
    # representation error from the kernel's accumulation
    b = lambda t: t.view(torch.bfloat16)[:, :n_v].double()
    ideal = (b(vh)[:T] @ b(mh)[:n_e].T + b(vh)[:T] @ b(ml)[:n_e].T + b(vl)[:T] @ b(mh)[:n_e].T).cpu().numpy()
    rel_ideal = float(np.linalg.norm(ideal - r) / np.linalg.norm(r))
    rel_kernel = float(np.linalg.norm(o - ideal) / np.linalg.norm(r))
    tf_exec = 3 * flops / (ms_bf / 1e3) / 1e12
    return {"config": {"voxels": int(n_v), "electrodes": int(n_e), "samples": int(T),
                       "history": "S1-S2 run of the FP32 engine (Mitchell-Schaeffer, S2 at 250 ms)",
                       "simulation_s": sim_s},
            "bf16x3_ms": ms_bf, "tile_config": int(best),
            "tile_config_ms": {autotune.EGM_TILE_NAMES[k]: v for k, v in cfg_ms.items()},
            "useful_tflops": flops / (ms_bf / 1e3) / 1e12, "executed_tflops": tf_exec,
            "tensor_frac": tf_exec / pk["bf16_tflops"], "peak_tflops": pk["bf16_tflops"], "peak_source": pk_src,
            "fp64_contract_ms": ms_f64, "fp64_tflops": flops / (ms_f64 / 1e3) / 1e12,
            "leadfield_ms": ev[0].elapsed_time(ev[1]), "rel_l2_bf16x3_vs_fp64": rel,
            "rel_l2_exact_product_of_parts": rel_ideal, "rel_l2_kernel_vs_exact_parts": rel_kernel}


def cpu_leg(args):
    """Port of the reference's legacy CPU stepper on the median MS instance,
    bounded to ``--cpu-seconds`` of stepping after JIT warm-up."""
    from oracle import legacy_cpu
    from pyheartsim_b200 import workloads
    sizes = workloads.batch_sizes(args.instances, args.n_min, args.n_max, args.seed)
    i = int(np.argsort(sizes[0::2])[len(sizes[0::2]) // 2]) * 2
    _, ref_args, meta = workloads.shell_case(i, int(sizes[i]), args.seed)
    run = legacy_cpu.LegacyRun(*ref_args, pacing_duration=meta["pacing_ms"])
    for _ in range(3):
        run.step()
    t0 = time.perf_counter()
    steps = 0
    while time.perf_counter() - t0 < args.cpu_seconds:
        run.step()
        steps += 1
    dt = time.perf_counter() - t0
    return {"value": meta["n"] * steps / dt, "unit": "voxel-steps/s", "cores": legacy_cpu.threads(), "kind": "port",
            "sample": f"{steps} steps of instance {i} ({meta['n']} voxels, MS) from t=0 in {dt:.1f} s"}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.egm_only:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"electrogram": egm_leg(args, dev)}), flush=True)
        return 0
    if args.geometry_only:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"geometry": geometry_leg(args, dev)}), flush=True)
        return 0
    if args.accuracy_only:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"accuracy": accuracy_leg(dev, args.tol, walls=tuple(args.c2_walls))}), flush=True)
        return 0
    if args.serving_only:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        out = {"serving": serving_leg(args, dev, count=args.serving_requests, plain_subset=0)}
        print(json.dumps(out), flush=True)
        return 0
    if args.plain_only:
        import torch
        from pyheartsim_b200 import workloads
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        cases = workloads.batched_inputs(args.instances, args.n_min, args.n_max, args.seed, t_phys=args.t_phys)
        print(json.dumps({"plain_fp64": plain_leg(args, cases, None, dev)}), flush=True)
        return 0
    if args.aniso_only:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"anisotropic": aniso_leg(args, dev, count=args.aniso_instances)}), flush=True)
        return 0
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
