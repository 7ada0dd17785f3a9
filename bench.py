#!/usr/bin/env python
"""Throughput of the sphere DEM time step on B200.

Metric: particle-steps/s of the FP64 DEM step (contact search, contact and
wall forces, integration, wall update) on the 1,000,000-sphere polydisperse
workload: log-normal radii (median 1 mm, sigma 0.2, clipped 0.5-2 mm), random
sequential placement in a periodic-x/y 0.2 x 0.2 x 0.4 m domain, top wall at
20 kPa, dt = 2e-7 s, grid 50 x 50 x 100 (seeded synthetic input; no dataset).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sphk|reference]

A step is one time step of the whole scene.  ``value`` is device-timed
throughput with the state resident in HBM (CUDA events on the launching
stream around exactly K steps; the ~2.5 GB state exceeds the 126 MB L2, so no
flush is needed).  ``e2e`` is the same metric through the C ABI with host
buffers: upload of the pinned host state, K steps, download of the state.
With N > 1 every rank runs an independent replica (own seed): the DEM step of
one scene has no cross-rank exchange here, so scaling is weak and no
collective sits on the data path; timing is the max over ranks.
``--impl reference`` times the reference's own kernel bodies (oracle/_ref,
compiled as host C++) on the host cores over a bounded sample of the same
workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-steps/s at 1M FP64 spheres"
UNIT = "particle-steps/s"
WORKLOAD = ("polydisperse settling: 1,000,000 log-normal spheres (median 1 mm, sigma 0.2, "
            "0.5-2 mm), RSA in periodic-x/y 0.2x0.2x0.4 m, 20 kPa top wall, FP64, dt 2e-7 s, "
            "grid 50x50x100, contact model 2")


def parse():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", choices=("sphk", "reference"), default="sphk")
    ap.add_argument("--n", type=int, default=1_000_000, help="particles (default: the 1M workload)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="bound on the timed CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-instances", type=int, default=512,
                    help="members of the batched settling ensemble (0: skip that leg)")
    ap.add_argument("--batch-steps", type=int, default=2000)
    ap.add_argument("--batch-sample", type=int, default=16,
                    help="members run one by one for the per-instance baseline")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-jammed", action="store_true",
                    help="skip the contact-laden (jammed) batched ensemble")
    ap.add_argument("--adjoint-n", type=int, default=100_000,
                    help="spheres of the calibration column (0: skip the adjoint leg)")
    ap.add_argument("--adjoint-steps", type=int, default=4000)
    ap.add_argument("--adjoint-checkpoint", type=int, default=100)
    ap.add_argument("--adjoint-fd-steps", type=int, default=40,
                    help="steps of the central-difference check on the jammed column")
    ap.add_argument("--no-darcy", action="store_true",
                    help="skip the Darcy-flow leg (the 1M workload with the fluid grid on)")
    ap.add_argument("--darcy-steps", type=int, default=400)
    ap.add_argument("--no-render", action="store_true",
                    help="skip the ray-tracer leg (one 800 x 800 image of the 1M workload)")
    ap.add_argument("--render-frames", type=int, default=10)
    ap.add_argument("--no-packed", action="store_true",
                    help="skip the contact-heavy leg (a jammed 1M-sphere column, ~6 contacts each)")
    ap.add_argument("--packed-steps", type=int, default=1000)
    ap.add_argument("--packed-side", type=int, default=100,
                    help="spheres per lattice edge of the packed column (default: 100^3 = 1M)")
    ap.add_argument("--no-bonded", action="store_true",
                    help="skip the bonded-tension leg (253,952 spheres, ~1.3M bonds)")
    ap.add_argument("--bonded-steps", type=int, default=1000)
    ap.add_argument("--profile-workload", choices=("polydisperse", "packed", "tension"),
                    help="only run one workload in profile mode (direct launches, for ncu)")
    ap.add_argument("--no-settling", action="store_true",
                    help="skip the 10k settling leg (the reference's CPU-runnable case)")
    ap.add_argument("--settling-steps", type=int, default=1000)
    return ap.parse_args()


def scene(n: int, seed: int):
    from sphere_b200 import scenes
    if n == 1_000_000:
        return scenes.polydisperse(seed=seed)
    # the same workload at another size: keep the number density and cell size
    s = (n / 1_000_000) ** (1.0 / 3.0)
    L = (0.2 * s, 0.2 * s, 0.4 * s)
    num = tuple(max(3, int(round(v / 0.004))) for v in L)
    return scenes.polydisperse(n=n, seed=seed, L=L, num=num)


def dist_env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", rank))
    return rank, world, local


def reduce_max(x, world, device="cuda"):
    """The largest of every rank's x (the timing rule: max over ranks)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during timing."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a moment to start: wait for its first sample
            # so that the region it brackets is covered
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 5.0:
                time.sleep(0.02)
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, window=None):
        out = self._summary()
        if window:
            out["window"] = window
        return out

    def _summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": 0}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(np_, ncells, contacts, nbonds=0):
    """Compulsory HBM bytes of one step, the hot path's standard model.

    Per particle 368 B of state: a read of 192 B (x,r 32, vel,fixvel 32,
    vel0 24, angvel 24, angvel0 24, angpos 24, xysum 16, es,ev 16) and a
    write of 176 B (the same less r and fixvel).  Then 52 B per active
    directed contact (partner 4 + history read 24 + write 24).  The whole
    step adds 16 B of sort key/permutation per particle, 16 B of start/end
    per cell and 136 B per bond.  Returns (step kernels, whole step, tight):
    `tight` is the step kernels' minimum for this input, see
    `tight_bytes`."""
    step_kernel = 368 * np_ + 52 * contacts
    whole = step_kernel + 16 * np_ + 16 * ncells + 136 * nbonds
    return step_kernel, whole, tight_bytes(np_, contacts)


def tight_bytes(np_, contacts):
    """The step kernels' minimum traffic for a given input, below the
    standard model in two places: fixvel is one flag byte, not a double, and
    the es/ev sums (read 16 + write 16) move only for a particle whose energy
    rates are nonzero, which needs a contact; min(np, contacts) bounds the
    number of such particles from above.  329 B per particle: a read of 169 B
    and a write of 160 B."""
    return 329 * np_ + 32 * min(np_, contacts) + 52 * contacts


def cpu_reference_run(sb, warmup, max_steps, seconds, kind_pref="reference"):
    """Time the reference's kernel bodies (oracle/_ref) -- or, where they are
    not built, the plain-C oracle -- on the host cores over a bounded sample:
    `warmup` untimed steps, then steps until `max_steps` or `seconds`."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle
    from sphere_b200.state import config_from_spherebin, state_from_spherebin
    kind = "reference" if (kind_pref == "reference" and pyoracle.LIB_REF.exists()) else "port"
    lib = pyoracle.load("ref" if kind == "reference" else "orc")
    cfg = config_from_spherebin(sb)
    run = pyoracle.OracleRun(lib, cfg, state_from_spherebin(sb))
    threads = lib.orc_threads(0)
    if warmup:
        rc = run.step(warmup, 0)
        if rc:
            raise RuntimeError(f"CPU oracle returned {rc}")
    done, t0 = 0, time.perf_counter()
    while done < max_steps and (time.perf_counter() - t0) < seconds:
        rc = run.step(1, 0)
        if rc:
            raise RuntimeError(f"CPU oracle returned {rc}")
        done += 1
    el = time.perf_counter() - t0
    return {"value": cfg.np * done / el, "unit": UNIT, "cores": int(threads), "kind": kind,
            "sample": f"{done} timed steps (after {warmup} warm-up) of the {cfg.np}-sphere "
                      f"workload, {el:.1f} s, OpenMP over particles"}


def gpu_arm(args, rank, world, local):
    import numpy as np
    import torch
    from sphere_b200.sphk import Simulation
    from sphere_b200.state import config_from_spherebin, state_from_spherebin

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    sb = scene(args.n, args.seed + 1000 * rank)
    cfg = config_from_spherebin(sb)
    st0 = state_from_spherebin(sb)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return reduce_max(x, world, "cuda")

    stream = torch.cuda.Stream()
    sim = Simulation(cfg, device=local)
    sim.upload(st0)
    # The clock samples (every 100 ms) cover the warm-up, the timed steps and
    # the profiled steps: a timed region of a few milliseconds falls between
    # two samples, the GPU's clocks under this load do not.
    clocks = ClockSampler(local).__enter__()
    sim.step(args.warmup, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    sim.sync()

    # ---- device-resident throughput: exactly K steps between events -------
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rebuilds0 = sim.stats()["cell_rebuilds"]
    barrier()
    start.record(stream)
    sim.step(args.steps, stream=stream.cuda_stream)
    end.record(stream)
    end.synchronize()
    barrier()
    sim.sync()
    ms = max_over_ranks(start.elapsed_time(end))
    stats = sim.stats()

    # ---- per-phase device time (profile mode, events between phases) ------
    nprof = min(max(args.steps, 50), 200)
    sim.set_profile(True)
    sim.profile(reset=True)
    sim.step(nprof)
    sim.sync()
    prof = sim.profile(reset=True)
    sim.set_profile(False)
    sim.close()
    clocks.__exit__(None, None, None)

    # ---- end to end through the C ABI with pinned host buffers ------------
    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.from_numpy(a[:0]).dtype, pin_memory=True)
        out = t.numpy()
        out[...] = a
        return out, t
    # the host side holds what the reference's state file holds: contact
    # slots, half-step velocities and accelerations stay on the device
    file_fields = ("x", "xysum", "vel", "force", "angpos", "angvel", "torque", "es_dot", "es",
                   "ev_dot", "ev", "p", "walls_nx", "walls_mvfd", "bonds", "bonds_delta",
                   "bonds_omega")
    keep = []
    st_h, st_out = st0.copy(), st0.copy()
    for st in (st_h, st_out):
        for f, v in list(st.__dict__.items()):
            if not isinstance(v, np.ndarray):
                continue
            if f not in file_fields:
                setattr(st, f, None)
            elif v.size:
                arr, t = pinned(v)
                keep.append(t)
                setattr(st, f, arr)
    sim2 = Simulation(cfg, device=local)
    h2d = sum(getattr(st_h, f).nbytes for f in file_fields if getattr(st_h, f) is not None)
    d2h = h2d
    barrier()
    t0 = time.perf_counter()
    sim2.upload(st_h)
    sim2.step(args.steps)
    sim2.sync()
    sim2.download(st_out)
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    sim2.close()

    n_total = cfg.np * world
    value = n_total * args.steps / (ms * 1e-3)
    e2e_value = n_total * args.steps / e2e_s
    step_ms = (prof["topo"] + prof["contact"] + prof["force"]) / max(1, prof["steps"])
    C = stats["active_contacts"]
    b_step, b_whole, b_tight = algorithmic_bytes(cfg.np, cfg.ncells, C, cfg.nb0)
    peak, peak_kind = measured_peak_hbm()
    achieved = b_step / (step_ms * 1e-3) / 1e9
    # per step: the rebuild gate, k_bonds (with bonds), k_topo, k_contact
    # (contact models 2 and 3), k_force_tiles, k_tail, and with dynamic walls
    # k_walls on its graph branch; the 7 cell-list kernels only in steps
    # whose cell list changed (a conditional graph node)
    rebuilt = stats["cell_rebuilds"] - rebuilds0
    per_step = (4 + (1 if cfg.nb0 else 0) + (1 if cfg.contactmodel in (2, 3) else 0)
                + (1 if cfg.nw else 0))
    launches = args.steps * per_step + 7 * rebuilt
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "particles_per_gpu": cfg.np, "ncells": cfg.ncells,
                   "dt": cfg.dt, "active_contacts": C, "l2": "state (~1.5 GB) exceeds L2",
                   "parallelism": "independent replicas" if world > 1 else "single GPU",
                   "graph_steps": 8},
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                "seconds": e2e_s},
        "gpu_launches": launches, "cell_rebuilds_timed": rebuilt,
        "roofline": {"bound": "hbm", "kernel": "k_topo+k_contact+k_force", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": (profiled_traffic("polydisperse_1m") or {}).get("bytes_per_step")
                                if cfg.np == 1_000_000 else None,
                     "algorithmic_bytes_per_launch": b_step,
                     "launch_ms": step_ms,
                     "tight_bytes_per_launch": b_tight,
                     "tight_frac": b_tight / (step_ms * 1e-3) / 1e9 / peak,
                     "whole_step_algorithmic_bytes": b_whole,
                     "whole_step_frac": (b_whole / (ms / args.steps * 1e-3) / 1e9) / peak},
        "phase_ms_per_step": {k: prof[k] / max(1, prof["steps"])
                              for k in ("cells", "bonds", "topo", "contact", "force", "walls")},
        "clocks": clocks.summary("warm-up, timed and profiled steps of this workload"),
    }
    if args.batch_instances > 0:
        out["batched"] = batched_leg(args, rank, world, local, barrier, max_over_ranks)
        if not args.no_jammed:
            out["batched_jammed"] = batched_leg(args, rank, world, local, barrier,
                                                max_over_ranks, kind="jammed")
    if args.adjoint_n > 0 and rank == 0:
        out["adjoint"] = adjoint_leg(args, local)
        if not args.no_jammed:
            out["adjoint_contacts"] = adjoint_contacts_leg(args, local)
    if not args.no_settling and rank == 0:
        out["settling"] = settling_leg(args, local)
    if not args.no_packed and rank == 0:
        out["packed"] = packed_leg(args, local)
    if not args.no_bonded and rank == 0:
        out["bonded"] = bonded_leg(args, local)
    if not args.no_darcy and rank == 0:
        out["darcy"] = darcy_leg(args, local, sb)
    if not args.no_render and rank == 0:
        out["render"] = render_leg(args, local, sb)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_reference_run(sb, 1, 1000, args.cpu_seconds)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return out


def binpack(nps, world):
    """Members to ranks: largest first onto the least-loaded rank."""
    order = sorted(range(len(nps)), key=lambda i: (-nps[i], i))
    load = [0] * world
    bins = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        bins[r].append(i)
        load[r] += nps[i]
    return [sorted(b) for b in bins]


def batched_leg(args, rank, world, local, barrier, max_over_ranks, kind="settling"):
    """A batched ensemble: every member this rank holds, stepped together by
    one context, against the same members run one by one.

    kind "settling": the configs' ensemble (``scenes.ensemble_member``),
    members that start apart and settle; the autotuner also picks their
    cell size.  kind "jammed": the same counts, stiffnesses and frictions
    with every member a jammed lattice (``scenes.jammed_member``, about six
    contacts per sphere from the first step), so the force laws run in every
    timed step."""
    import torch
    from sphere_b200 import autotune, scenes
    from sphere_b200.sphk import BatchSimulation, Simulation
    from sphere_b200.state import config_from_spherebin, state_from_spherebin

    n_inst = args.batch_instances
    if kind == "jammed":
        build = lambda i, cf=None: scenes.jammed_member(i)
        cell_factors = (None,)
    else:
        build = lambda i, cf=2.0: scenes.ensemble_member(i, cell_factor=cf)
        cell_factors = autotune.CELL_FACTORS
    nps = [build(i).np for i in range(n_inst)]
    mine = binpack(nps, world)[rank]
    tuned = None
    if args.no_autotune:
        cell_factor, skin, gsteps, shapes = (2.0 if kind != "jammed" else None), 0.1, 8, 0
    else:
        sub = mine[:: max(1, len(mine) // 64)][:64]
        t0 = time.perf_counter()
        ch = autotune.tune(lambda cf: [build(i, cf) for i in sub], warmup=10, steps=40,
                           device=local, cell_factors=cell_factors)
        cell_factor, skin, gsteps, shapes = ch.cell_factor, ch.verlet_skin, ch.graph_steps, ch.shapes
        tuned = {"members": len(sub), "seconds": time.perf_counter() - t0,
                 "trials": ch.trials}
    members = [build(i, cell_factor) for i in mine]
    cfgs = [config_from_spherebin(sb) for sb in members]
    states = [state_from_spherebin(sb) for sb in members]
    stream = torch.cuda.Stream()   # not the default stream (handle 0)
    K = args.batch_steps

    # ---- batched: all members in one context, inputs resident ---------------
    t_e2e = time.perf_counter()
    sim = BatchSimulation(cfgs, device=local, graph_steps=gsteps, verlet_skin=skin,
                          block_shapes=shapes)
    sim.upload(states)
    sim.step(args.warmup, stream=stream.cuda_stream)
    sim.sync()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    start.record(stream)
    sim.step(K, stream=stream.cuda_stream)
    end.record(stream)
    end.synchronize()
    barrier()
    sim.sync()
    ms_batch = max_over_ranks(start.elapsed_time(end))
    _ = sim.download_all()
    e2e_s = max_over_ranks(time.perf_counter() - t_e2e)
    contacts = sim.stats()["active_contacts"]
    sim.close()

    # ---- per-instance baseline: a sample of the same members, one by one -----
    per = {}
    if rank == 0 and args.batch_sample > 0:
        sample = list(range(0, len(members), max(1, len(members) // args.batch_sample)))
        sample = sample[: args.batch_sample]
        tot_ms = 0.0
        for j in sample:
            one = Simulation(cfgs[j], device=local, graph_steps=gsteps, verlet_skin=skin)
            one.upload(states[j])
            one.step(args.warmup, stream=stream.cuda_stream)
            one.sync()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            one.step(K, stream=stream.cuda_stream)
            b.record(stream)
            b.synchronize()
            one.sync()
            tot_ms += a.elapsed_time(b)
            one.close()
        est_ms = tot_ms * len(members) / len(sample)
        per = {"sampled_members": len(sample), "sampled_ms": tot_ms,
               "estimated_ms_all_members": est_ms,
               "instances_per_s": len(members) / (est_ms * 1e-3),
               "speedup_batched_vs_per_instance": est_ms / ms_batch}
    n_part = sum(nps)
    what = ("settling members (N log-uniform 500-20000)" if kind != "jammed" else
            "jammed members (counts, k_n, mu of the settling members; r 1 mm simple-cubic "
            "lattices at a 20 kPa overlap, periodic x/y)")
    return {
        "metric": "batched instances/s", "value": n_inst / (ms_batch * 1e-3), "unit": "instances/s",
        "workload": f"{n_inst} {what}, {n_part} spheres, {K} steps each, one context per GPU",
        "particles": n_part, "steps": K, "ms": ms_batch, "scaling": "strong",
        "particle_steps_per_s": n_part * K / (ms_batch * 1e-3),
        "active_contacts_end": contacts,
        "choice": {"cell_factor": cell_factor, "verlet_skin": skin, "graph_steps": gsteps,
                   "block_shapes": autotune.SHAPE_NAMES[shapes]},
        "autotune": tuned,
        "e2e": {"value": n_inst / e2e_s, "unit": "instances/s", "seconds": e2e_s,
                "note": "create + upload + warm-up + timed steps + download"},
        "per_instance": per,
    }


def height_profile_loss(x, r, lo, hi, target):
    """Mean squared deviation of the 64-bin height profile (highest sphere
    top per x-bin, 0 when empty) from `target`, and dLoss/dx."""
    import numpy as np
    bins = len(target)
    top = x[:, 2] + r
    b = np.clip(((x[:, 0] - lo) / (hi - lo) * bins).astype(np.int64), 0, bins - 1)
    h = np.zeros(bins)
    arg = np.full(bins, -1)
    order = np.lexsort((top, b))           # by bin, then by height
    last = np.r_[b[order][1:] != b[order][:-1], True]
    for i in order[last]:
        h[b[i]] = top[i]
        arg[b[i]] = i
    loss = float(np.mean((h - target) ** 2))
    xbar = np.zeros_like(x)
    for k in range(bins):
        if arg[k] >= 0:
            xbar[arg[k], 2] = 2.0 * (h[k] - target[k]) / bins
    return loss, xbar


def adjoint_leg(args, local):
    """The calibration column: time of the checkpointed adjoint against the
    differentiable forward, gradients of the height-profile loss, and a
    finite-difference check of the k_n gradient on a contact-rich scene."""
    import numpy as np
    import torch
    from sphere_b200 import adjoint, scenes
    from sphere_b200.sphk import Simulation
    from sphere_b200.state import config_from_spherebin, state_from_spherebin

    sb = scenes.column(args.adjoint_n, seed=args.seed)
    steps, K = args.adjoint_steps, args.adjoint_checkpoint
    cfg = config_from_spherebin(sb)
    st0 = state_from_spherebin(sb)
    stream = torch.cuda.Stream()   # not the default stream (handle 0)
    # the plain step (the reference's arithmetic) for scale
    plain = Simulation(cfg, device=local)
    plain.upload(st0)
    plain.step(args.warmup, stream=stream.cuda_stream)
    plain.sync()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    plain.step(steps, stream=stream.cuda_stream)
    b.record(stream)
    b.synchronize()
    plain.sync()
    ms_plain = a.elapsed_time(b)
    plain.close()
    # differentiable forward with checkpoints, then the adjoint: iterations
    # of a calibration loop in one context.  The first allocates the
    # checkpoint buffers and captures the segment graphs; the ratio is the
    # median over the later ones, which reuse them.
    sim = Simulation(cfg, device=local)
    target = np.random.default_rng(args.seed + 7).uniform(0.2, 0.32, 64)
    iters = []
    for _ in range(4):
        sim.upload(st0)
        sim.diff_begin(mu=None, checkpoint_every=K)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.step(steps)
        sim.sync()
        t_fwd = time.perf_counter() - t0
        st = sim.download()
        loss, xbar = height_profile_loss(st.x[:, :3], st.x[:, 3], 0.0, float(sb.L[0]), target)
        t0 = time.perf_counter()
        g = sim.diff_backward(xbar)
        t_bwd = time.perf_counter() - t0
        stats = sim.stats()
        sim.diff_end()
        iters.append((t_fwd, t_bwd))
    sim.close()

    # central differences of every gradient on a dense colliding scene
    fsb = scenes.collision(n=2000, seed=args.seed + 3, periodic=0, vmax=0.2, wmax=50.0)
    fsteps = 60
    fd = fd_checks(fsb, fsteps, 20, local, args.seed + 4)
    fd["scene"] = f"collision, {fsb.np} spheres, {fsteps} steps, checkpoints every 20"
    return {
        "metric": "adjoint/forward time ratio",
        "value": float(np.median([b / f for f, b in iters[1:]])), "unit": "ratio",
        "higher_is_better": False,
        "workload": f"calibration column: {sb.np} spheres (radii as the 1M workload), RSA in "
                    f"0.1x0.1x0.3 m on the floor of a 0.6x0.6x0.35 m box, FP64, dt 5e-7 s, "
                    f"{steps} steps, checkpoints every {K}",
        "forward_s": float(np.median([f for f, _ in iters[1:]])),
        "backward_s": float(np.median([b for _, b in iters[1:]])),
        "iterations": [{"forward_s": f, "backward_s": b, "ratio": b / f} for f, b in iters],
        "plain_step_ms": ms_plain / steps,
        "diff_forward_step_ms": 1e3 * float(np.median([f for f, _ in iters[1:]])) / steps,
        "loss": loss, "grad": {"k_n": g["k_n"], "k_t": g["k_t"], "gamma_n": g["gamma_n"],
                               "mu_global": float(g["mu"].sum()),
                               "mu_particles_nonzero": int(np.count_nonzero(g["mu"]))},
        "device_bytes": stats["device_bytes"],
        "fd_check": fd,
    }


def fd_checks(sb, fsteps, fK, local, seed, h_rel=1e-6, v_weight=1e-3):
    """Central differences (step h_rel of each parameter) of a seeded linear
    loss of the final positions and velocities, L = w.x + u.v, against the
    adjoint's gradients with respect to k_n, k_t, gamma_n, the global mu and
    the mu of the three particles with the largest adjoint: one list entry
    per parameter (u: normal weights scaled by v_weight).  The difference
    L(+h) - L(-h) is summed from the
    elementwise differences of the two final states, w.(x+ - x-) + u.(v+ -
    v-): the loss itself is of the order of the positions (centimetres
    times sqrt(N)), and rounding its two sums would bury the change of
    order h that the difference measures."""
    import numpy as np
    from sphere_b200 import adjoint

    rng = np.random.default_rng(seed)
    wx = rng.normal(size=(sb.np, 3))
    wv = rng.normal(size=(sb.np, 3)) * v_weight
    mu0 = np.full(sb.np, float(sb.mu_s))
    base = dict(k_n=float(sb.k_n), k_t=float(sb.k_t), gamma_n=float(sb.gamma_n))

    def run(k_n, k_t, gamma_n, mu):
        s_, st_ = adjoint.run_forward(sb, fsteps, k_n, k_t, gamma_n, mu, checkpoint_every=fK,
                                      device=local)
        return s_, (np.array(st_.x[:, :3]), np.array(st_.vel[:, :3]))

    s_, _ = run(base["k_n"], base["k_t"], base["gamma_n"], mu0)
    ga = s_.diff_backward(wx, wv)
    s_.close()
    checks = []

    def central(name, adj, plus, minus, h):
        sp, (xp, vp) = plus()
        sp.close()
        sm, (xm, vm) = minus()
        sm.close()
        fd = (float(np.sum(wx * (xp - xm))) + float(np.sum(wv * (vp - vm)))) / (2.0 * h)
        checks.append({"param": name, "adjoint": adj, "central_difference": fd,
                       "rel_error": abs(adj - fd) / abs(fd) if fd else None})

    for name in ("k_n", "k_t", "gamma_n"):
        h = h_rel * base[name]
        pp, pm = dict(base), dict(base)
        pp[name] += h
        pm[name] -= h
        central(name, float(ga[name]), lambda p=pp: run(**p, mu=mu0),
                lambda p=pm: run(**p, mu=mu0), h)
    h = h_rel * float(sb.mu_s)
    central("mu", float(ga["mu"].sum()), lambda: run(**base, mu=mu0 + h),
            lambda: run(**base, mu=mu0 - h), h)
    for i in np.argsort(-np.abs(ga["mu"]))[:3]:
        e = np.zeros(sb.np)
        e[i] = h
        central(f"mu[{int(i)}]", float(ga["mu"][i]), lambda e=e: run(**base, mu=mu0 + e),
                lambda e=e: run(**base, mu=mu0 - e), h)
    return {"h": f"{h_rel:g} relative",
            "loss": f"w.x + u.v, seeded normal weights (u scaled {v_weight:g})",
            "difference": "elementwise, w.(x+ - x-) + u.(v+ - v-)",
            "checks": checks, "max_rel_error": max(c["rel_error"] or 0.0 for c in checks)}


def adjoint_contacts_leg(args, local):
    """The adjoint where the contacts do the work: the calibration column
    replaced by a jammed, stirred block (``scenes.jammed_column``: 100,800
    spheres of r 1 mm held at a 20 kPa overlap by the six implicit walls,
    seeded velocities and spins, so contacts stick and slide from the first
    step).  Reports the adjoint/forward time ratio over the full run with the
    height-profile loss, every gradient, and a central-difference check of
    the gradients with respect to k_n, k_t, gamma_n and the global mu on a
    jammed block of the same kind where the loss is smooth in the
    parameters over the difference's step: 16^3 spheres at k_n = k_t = 1e4,
    gamma_n 0.1 of critical, stirred 100 times more gently, so that every
    contact holds and sticks through the 40 steps (h = 1e-3 relative,
    velocity-weighted linear loss).  On the timed block itself a central
    difference measures no derivative: its stirring opens contacts and
    moves them across the stick/slip limit within the run (kinks a step h
    can cross), and at k_n = 1e6 the locked lattice's response to a small
    h is near the FP64 resolution of its trajectories."""
    import numpy as np
    import torch
    from sphere_b200 import adjoint, scenes
    from sphere_b200.sphk import Simulation
    from sphere_b200.state import config_from_spherebin, state_from_spherebin

    sb = scenes.jammed_column()
    steps, K = args.adjoint_steps, args.adjoint_checkpoint
    cfg = config_from_spherebin(sb)
    st0 = state_from_spherebin(sb)
    target = np.random.default_rng(args.seed + 17).uniform(0.12, 0.13, 64)
    sim = Simulation(cfg, device=local)
    iters = []
    for _ in range(3):
        sim.upload(st0)
        sim.diff_begin(mu=None, checkpoint_every=K)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.step(steps)
        sim.sync()
        t_fwd = time.perf_counter() - t0
        st = sim.download()
        C = sim.stats()["active_contacts"]
        loss, xbar = height_profile_loss(st.x[:, :3], st.x[:, 3], 0.0, float(sb.L[0]), target)
        t0 = time.perf_counter()
        g = sim.diff_backward(xbar)
        t_bwd = time.perf_counter() - t0
        sim.diff_end()
        iters.append((t_fwd, t_bwd))
    sim.close()

    # central differences on a smooth block of the same kind
    fsteps = args.adjoint_fd_steps
    fsb = scenes.jammed_column(nx=16, ny=16, nz=16, k=1e4, gamma_frac=0.1, vmax=5e-5, wmax=0.2)
    fd = fd_checks(fsb, fsteps, 10, local, args.seed + 18, h_rel=1e-3, v_weight=1e3)
    fd["scene"] = (f"jammed block 16x16x16 ({fsb.np} spheres, r 1 mm, six implicit walls), "
                   "k_n = k_t = 1e4, gamma_n 0.1 of critical, velocities U(+-5e-5) m/s, spins "
                   f"U(+-0.2) rad/s, every contact sticking; {fsteps} steps, checkpoints every 10")
    ratios = [b / f for f, b in iters[1:]]
    return {
        "metric": "adjoint/forward time ratio", "value": float(np.median(ratios)), "unit": "ratio",
        "higher_is_better": False,
        "workload": f"jammed, stirred column: {sb.np} spheres of r 1 mm, simple-cubic block "
                    "40x40x63 at a 20 kPa overlap held by the six implicit walls, velocities "
                    "U(+-0.005) m/s, spins U(+-20) rad/s, k_n = k_t = 1e6, mu 0.3, gamma_n 1e-3 of "
                    f"critical, FP64, dt 5e-7 s, {steps} steps, checkpoints every {K}",
        "active_contacts_end": C,
        "forward_s": float(np.median([f for f, _ in iters[1:]])),
        "backward_s": float(np.median([b for _, b in iters[1:]])),
        "iterations": [{"forward_s": f, "backward_s": b, "ratio": b / f} for f, b in iters],
        "loss": loss,
        "grad": {"k_n": g["k_n"], "k_t": g["k_t"], "gamma_n": g["gamma_n"],
                 "mu_global": float(g["mu"].sum()),
                 "mu_particles_nonzero": int(np.count_nonzero(g["mu"]))},
        "fd_check": fd,
    }


def darcy_leg(args, local, sb):
    """The Darcy flow (src/darcy.cuh) on the headline workload: the fluid
    grid is the 50 x 50 x 100 cell grid, initialised as DEM::initDarcy does
    from a uniform pressure.  Reports the per-step time of the Darcy kernels
    (profile mode), the whole step with and without them (graphs), and the
    kernels' algorithmic bytes against the measured HBM bandwidth."""
    import numpy as np
    import torch
    from sphere_b200.darcy import DarcyState
    from sphere_b200.sphk import Simulation, darcy_init
    from sphere_b200.state import config_from_spherebin, state_from_spherebin

    nu = 8.9e-4
    cfg = config_from_spherebin(sb)
    st0 = state_from_spherebin(sb)
    ds = DarcyState.zeros(cfg.num)
    shape = tuple(int(v) for v in cfg.num)
    ds.set_cells(H=np.full(shape, 1.0e4))
    stability = darcy_init(cfg, nu, st0.x, ds)
    stream = torch.cuda.Stream()
    K = args.darcy_steps

    def timed(with_flow):
        sim = Simulation(cfg, device=local)
        sim.upload(st0)
        if with_flow:
            sim.darcy_upload(ds, nu)
        sim.step(args.warmup, stream=stream.cuda_stream)
        sim.sync()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sim.step(K, stream=stream.cuda_stream)
        b.record(stream)
        b.synchronize()
        sim.sync()
        ms = a.elapsed_time(b) / K
        prof = None
        if with_flow:
            sim.set_profile(True)
            sim.profile(reset=True)
            sim.step(min(K, 100))
            sim.sync()
            prof = sim.profile()
        sim.close()
        return ms, prof

    ms_plain, _ = timed(False)
    ms_flow, prof = timed(True)
    darcy_ms = prof["darcy"] / max(1, prof["steps"])
    ncell = int(np.prod(shape))
    # compulsory bytes: the particles' positions once (32 B) and their
    # cell-list entries (4 B); per cell the porosity's start/end words (8),
    # the old porosity (8) and the new porosity, change, conductivity and
    # transmissivity (56); the explicit step's T, Ss, W, dphi, H (56) and new
    # H (8); the gradient's H, K, phi (24) and dH, V (48)
    b_step = 36 * cfg.np + (8 + 8 + 56 + 56 + 8 + 24 + 48) * ncell
    peak, peak_kind = measured_peak_hbm()
    achieved = b_step / (darcy_ms * 1e-3) / 1e9
    return {
        "metric": "Darcy flow time per step", "value": darcy_ms, "unit": "ms",
        "higher_is_better": False,
        "workload": f"{WORKLOAD}; Darcy flow on the {shape[0]}x{shape[1]}x{shape[2]} cell grid, "
                    f"nu {nu} Pa s, uniform starting pressure",
        "cells": ncell, "steps": K, "stability_criterion": stability,
        "cells_per_s": ncell / (darcy_ms * 1e-3),
        "step_ms_without_flow": ms_plain, "step_ms_with_flow": ms_flow,
        "roofline": {"bound": "hbm", "kernel": "k_darcy_*", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "algorithmic_bytes_per_step": b_step},
    }


def profiled_traffic(workload_key):
    """DRAM bytes per step of the step kernels of one workload, from the
    committed ncu summary of the 1M workloads (profiles/
    step_kernels_1m_dram.md: one line `traffic <workload> <kernel> <bytes>`
    per kernel, a capture of the current code), or None when absent."""
    p = ROOT / "profiles" / "step_kernels_1m_dram.md"
    if not p.exists():
        return None
    out = {}
    for ln in p.read_text().splitlines():
        f = ln.strip().strip("`").split()
        if len(f) == 4 and f[0] == "traffic" and f[1] == workload_key:
            out[f[2]] = float(f[3])
    if not out:
        return None
    return {"bytes_per_step": sum(out.values()), "per_kernel": out,
            "source": "profiles/step_kernels_1m_dram.md"}


def timed_steps(sim, K, warmup, local, stream, nprof=200):
    """Warm-up, then exactly K steps between CUDA events on `stream`, then
    per-phase times from up to `nprof` profile-mode steps; the clock samples
    cover all three.  Returns (ms per step, phases per step, clocks)."""
    import torch
    clocks = ClockSampler(local).__enter__()
    sim.step(warmup, stream=stream.cuda_stream)
    sim.sync()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    sim.step(K, stream=stream.cuda_stream)
    b.record(stream)
    b.synchronize()
    sim.sync()
    ms = a.elapsed_time(b) / K
    prof = None
    if nprof:
        sim.set_profile(True)
        sim.profile(reset=True)
        sim.step(min(K, nprof))
        sim.sync()
        prof = sim.profile(reset=True)
        sim.set_profile(False)
        prof = {k: prof[k] / max(1, prof["steps"])
                for k in ("cells", "bonds", "topo", "contact", "force", "walls")}
    clocks.__exit__(None, None, None)
    return ms, prof, clocks.summary("warm-up, timed and profiled steps of this workload")


def settling_leg(args, local):
    """The plain settling scene (``scenes.settling``: 10,000 spheres of r =
    0.01 m on a jittered lattice in a 0.5 x 0.5 x 2 m box, dt = 1e-6 s,
    1000 steps), the reference's own CPU-runnable case: particle-steps/s on
    the GPU through the whole run, and beside it the reference's kernel
    bodies on the host cores over the same 1000 steps."""
    import torch
    from sphere_b200 import scenes
    from sphere_b200.sphk import Simulation
    from sphere_b200.state import config_from_spherebin, state_from_spherebin

    sb = scenes.settling()
    cfg = config_from_spherebin(sb)
    K = args.settling_steps
    stream = torch.cuda.Stream()
    with Simulation(cfg, device=local) as sim:
        sim.upload(state_from_spherebin(sb))
        ms, prof, clocks = timed_steps(sim, K, 0, local, stream, nprof=0)
        C = sim.stats()["active_contacts"]
    out = {
        "metric": "particle-steps/s, 10k settling", "value": cfg.np / (ms * 1e-3),
        "unit": UNIT, "higher_is_better": True, "ms_per_step": ms, "steps": K,
        "workload": "plain settling: 10,000 spheres, r 0.01 m, rho 2600, jittered cubic lattice "
                    "(2.2 r, +-0.1 r) in a 0.5x0.5x2 m box, frictional walls, g -9.81, kn = kt = "
                    "1e6, gamma_n 100, mu 0.5, FP64, dt 1e-6 s, grid 24x24x96, from rest",
        "active_contacts_end": C, "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        base = cpu_reference_run(sb, 0, K, 120.0)
        out["cpu_baseline"] = base
        out["speedup_vs_cpu_baseline"] = out["value"] / base["value"]
    return out


def bonded_leg(args, local):
    """The bonded-tension workload (``scenes.tension``: 253,952 spheres on an
    FCC bar along x, a bond between every pair of lattice neighbours, about
    5 bonds per sphere counted once, stretched at 0.01 m/s end to end): the
    step with bond forces, breaking and bond-order force gathering.  The K
    timed steps start from the unbroken bar and run past half of its bonds
    breaking; reports particle-steps/s, the bond share of the step, the
    whole step against the measured HBM bandwidth with 136 B per bond, and
    the reference's kernel bodies on the host cores over a bounded sample."""
    import numpy as np
    import torch
    from sphere_b200 import scenes
    from sphere_b200.sphk import Simulation
    from sphere_b200.state import config_from_spherebin, state_from_spherebin

    sb = scenes.tension()
    cfg = config_from_spherebin(sb)
    st0 = state_from_spherebin(sb)
    K = args.bonded_steps
    stream = torch.cuda.Stream()
    with Simulation(cfg, device=local) as sim:
        sim.upload(st0)
        sim.step(args.warmup, stream=stream.cuda_stream)   # warm-up, then back to the start
        sim.sync()
        sim.upload(st0)
        ms, _, clocks = timed_steps(sim, K, 0, local, stream, nprof=0)
        st = sim.download()
        C = sim.stats()["active_contacts"]
        broken = int((st.bonds[:, 0] >= cfg.np).sum())
        # the per-phase times over the same steps, from the start again
        sim.upload(st0)
        sim.set_profile(True)
        sim.profile(reset=True)
        sim.step(min(K, 400))
        sim.sync()
        prof = sim.profile(reset=True)
    nb = cfg.nb0
    phases = {k: prof[k] / max(1, prof["steps"])
              for k in ("cells", "bonds", "topo", "contact", "force", "walls")}
    _, b_whole, _ = algorithmic_bytes(cfg.np, cfg.ncells, C, nb)
    peak, peak_kind = measured_peak_hbm()
    achieved = b_whole / (ms * 1e-3) / 1e9
    b_bonds = 136 * nb
    out = {
        "metric": "particle-steps/s, bonded tension", "value": cfg.np / (ms * 1e-3), "unit": UNIT,
        "higher_is_better": True, "ms_per_step": ms, "steps": K,
        "workload": f"bonded tension: {cfg.np:,} spheres, r U(0.9, 1.1) mm, FCC bar along x "
                    f"(62x32x32 cells, spacing 2.25 mm), {nb:,} bonds (every lattice neighbour), "
                    "homogeneous stretch at 0.01 m/s end to end, end layers held, sigma_b = tau_b "
                    "= 0.003, FP64, dt 1e-7 s, from the unbroken bar",
        "bonds": nb, "bonds_per_particle": nb / cfg.np,
        "broken_fraction_end": broken / nb, "active_contacts_end": C,
        "phase_ms_per_step": phases,
        "bond_share_of_step": phases["bonds"] / max(1e-12, sum(phases.values())),
        "roofline": {"bound": "hbm", "kernel": "whole step", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "algorithmic_bytes_per_step": b_whole,
                     "k_bonds_achieved": b_bonds / (phases["bonds"] * 1e-3) / 1e9
                     if phases["bonds"] > 0 else None,
                     "k_bonds_algorithmic_bytes": b_bonds,
                     "traffic": (profiled_traffic("tension_254k") or {}).get("bytes_per_step")
                                if cfg.np == 253_952 else None,
                     "traffic_per_kernel": (profiled_traffic("tension_254k") or {}).get("per_kernel")
                                           if cfg.np == 253_952 else None},
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        base = cpu_reference_run(sb, 0, 1000, args.cpu_seconds)
        out["cpu_baseline"] = base
        out["speedup_vs_cpu_baseline"] = out["value"] / base["value"]
    return out


def packed_leg(args, local):
    """The contact-heavy workload: a jammed simple-cubic column of 1M spheres
    (``scenes.packed``: 100 x 100 x 100, r = 1 mm, periodic x/y, 20 kPa top
    wall), where every sphere holds about six contacts through the run.  It
    measures the force laws and the 52 B per directed contact that the
    headline workload, whose spheres barely touch, leaves out.  Reports
    particle-steps/s over K graph steps, the contact search, contact force
    and integration kernels against the measured HBM bandwidth with the
    measured contact count, and the reference's kernel bodies on the host
    cores over a bounded sample of the same steps."""
    import numpy as np
    import torch
    from sphere_b200 import scenes
    from sphere_b200.sphk import Simulation
    from sphere_b200.state import config_from_spherebin, state_from_spherebin

    side = args.packed_side
    sb = scenes.packed(nx=side, ny=side, nz=side)
    cfg = config_from_spherebin(sb)
    stream = torch.cuda.Stream()
    K = args.packed_steps
    sim = Simulation(cfg, device=local)
    sim.upload(state_from_spherebin(sb))
    sim.step(args.warmup, stream=stream.cuda_stream)
    sim.sync()
    # the column must still be jammed: a lattice that had started to fly
    # apart would pile spheres into the edge cells and time nothing useful
    vmax = float(np.abs(sim.download().vel[:, :3]).max())
    if not vmax < 0.05 or sim.stats()["active_contacts"] < 5 * cfg.np:
        sim.close()
        return {"unavailable": f"packed column not jammed after warm-up (max speed {vmax:.3g} m/s)"}
    rebuilds0 = sim.stats()["cell_rebuilds"]
    ms, prof, clocks = timed_steps(sim, K, 0, local, stream)
    stats = sim.stats()
    sim.close()
    C = stats["active_contacts"]
    kern_ms = prof["topo"] + prof["contact"] + prof["force"]
    b_step, _, b_tight = algorithmic_bytes(cfg.np, cfg.ncells, C)
    peak, peak_kind = measured_peak_hbm()
    achieved = b_step / (kern_ms * 1e-3) / 1e9
    traffic = profiled_traffic("packed_1m") if side == 100 else None
    out = {
        "metric": METRIC, "value": cfg.np / (ms * 1e-3), "unit": UNIT, "higher_is_better": True,
        "ms_per_step": ms, "steps": K,
        "workload": f"packed column: {cfg.np:,} spheres of r 1 mm on a jammed simple-cubic "
                    f"lattice ({side}x{side}x{side}, overlap 8e-8 m), periodic x/y, 20 kPa top "
                    f"wall, FP64, dt 2e-7 s, grid {side // 2}x{side // 2}x100, contact model 2, "
                    "no normal viscosity",
        "active_contacts": C, "contacts_per_particle": C / cfg.np,
        "cell_rebuilds_timed": stats["cell_rebuilds"] - rebuilds0,
        "roofline": {"bound": "hbm", "kernel": "k_topo+k_contact+k_force", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "algorithmic_bytes_per_launch": b_step,
                     "launch_ms": kern_ms, "tight_bytes_per_launch": b_tight,
                     "tight_frac": b_tight / (kern_ms * 1e-3) / 1e9 / peak,
                     "traffic": traffic["bytes_per_step"] if traffic else None,
                     "traffic_per_kernel": traffic["per_kernel"] if traffic else None},
        "phase_ms_per_step": prof,
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        base = cpu_reference_run(sb, 1, 1000, args.cpu_seconds)
        out["cpu_baseline"] = base
        out["speedup_vs_cpu_baseline"] = out["value"] / base["value"]
    return out


def render_leg(args, local, sb):
    """The ray tracer (DEM::render) on the headline workload: 800 x 800
    images of the 1M spheres, plain and through the velocity colour map, each
    call including the image's copy to the host.  The CPU baseline runs the
    reference's own kernels (oracle/_ref; the plain-C restatement where that
    is not built) on a band of rows on all host cores and scales to a frame:
    the reference tests every sphere for every pixel."""
    import numpy as np
    from sphere_b200.sphk import Simulation
    from sphere_b200.state import config_from_spherebin, state_from_spherebin

    cfg = config_from_spherebin(sb)
    st0 = state_from_spherebin(sb)
    W = H = 800
    sim = Simulation(cfg, device=local)
    sim.upload(st0)
    out = {}
    for name, method, maxval in (("normal", 0, 0.0), ("vel", 2, 0.05)):
        img = sim.render(method, maxval, 0.0, W, H)   # warm-up: scratch allocation
        t0 = time.perf_counter()
        for _ in range(args.render_frames):
            img = sim.render(method, maxval, 0.0, W, H)
        out[name] = (time.perf_counter() - t0) / args.render_frames * 1e3
    covered = int(((img[..., :3] != 255).any(axis=2)).sum())
    sim.close()
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import pyoracle
        kind = "reference" if pyoracle.LIB_REF.exists() else "port"
        lib_orc = pyoracle.load("orc")
        lib = pyoracle.load("ref") if kind == "reference" else lib_orc
        rows = 2
        t0 = time.perf_counter()
        pyoracle.render(lib, lib_orc, st0, sb.L, 0, 0.0, 0.0, W, H, rows=(H // 2, rows))
        secs = time.perf_counter() - t0
        frame_s = secs * H / rows
        cpu = {"value": 1.0 / frame_s, "unit": "frames/s", "cores": os.cpu_count(), "kind": kind,
               "sample": f"{rows} of {H} rows of the plain 800 x 800 image ({secs:.1f} s), "
                         f"scaled to a frame"}
    ms = out["normal"]
    return {
        "metric": "ray-traced frames/s at 1M spheres, 800 x 800", "value": 1e3 / ms,
        "unit": "frames/s", "higher_is_better": True,
        "workload": f"{WORKLOAD}; DEM::render's camera and shading",
        "ms_per_frame": out, "pixels_covered": covered,
        "sphere_pixel_tests_per_s_equivalent": cfg.np * W * H / (ms * 1e-3),
        "cpu_baseline": cpu,
    }


def reference_arm(args, rank, world):
    if rank != 0:
        return None
    sb = scene(args.n, args.seed)
    base = cpu_reference_run(sb, min(args.warmup, 1), args.steps, 60.0)
    return {
        "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": WORKLOAD, "particles_per_gpu": sb.np, "parallelism": "host cores"},
        "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def profile_workload(args):
    """One workload in profile mode only (every kernel a direct launch, one
    step after another with events between the phases), for ncu: a profiler
    cannot follow the kernels of the step graphs.  `warmup` steps, then
    `steps` steps; prints the phase times per step.  Per step the launches
    are the cell-list kernels, k_bonds (with bonds), k_topo, k_contact (models
    2 and 3), k_force_tiles and the wall kernel, in that order."""
    import torch
    from sphere_b200 import scenes
    from sphere_b200.sphk import Simulation
    from sphere_b200.state import config_from_spherebin, state_from_spherebin

    w = args.profile_workload
    if w == "packed":
        side = args.packed_side
        sb = scenes.packed(nx=side, ny=side, nz=side)
    elif w == "tension":
        sb = scenes.tension()
    else:
        sb = scene(args.n, args.seed)
    with Simulation(config_from_spherebin(sb), device=0) as sim:
        sim.upload(state_from_spherebin(sb))
        sim.set_profile(True)
        sim.step(args.warmup)
        sim.sync()
        sim.profile(reset=True)
        sim.step(args.steps)
        sim.sync()
        prof = sim.profile(reset=True)
    torch.cuda.synchronize()
    return {"profile_workload": w, "particles": sb.np, "steps": args.steps,
            "phase_ms_per_step": {k: prof[k] / max(1, prof["steps"])
                                  for k in ("cells", "bonds", "topo", "contact", "force", "walls")}}


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.profile_workload:
        from sphere_b200 import build
        build.build()
        print(json.dumps(profile_workload(args)))
        return
    if args.impl == "reference":
        out = reference_arm(args, rank, world)
    else:
        from sphere_b200 import build
        if rank == 0:
            build.build()
        out = gpu_arm(args, rank, world, local)
    if rank == 0 and out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
