#!/usr/bin/env python
"""Headline benchmark: particle-steps/s of the 1,048,576-particle PCISPH dam
break (eta = 1 %, min 3 / max 50 corrections) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0 (see the keys below). A "step" is one full
simulation step over the whole particle set: grid, radix sort, neighbour
lists, density, non-pressure forces, the eta-controlled corrector loop,
walls and velocity interpolation.

  value     particle-steps/s with the state resident in HBM, device-timed with
            CUDA events on the simulation's stream, max over ranks;
  e2e       the same metric through the C ABI with host buffers: each step
            uploads positions and velocities from pinned host memory, steps,
            and downloads positions, velocities and densities (what the
            reference's update() copies back for its front end);
  roofline  the dominant kernel's algorithmic bytes per launch over its mean
            launch time, against the measured HBM copy bandwidth;
  cpu_baseline  the FP64 oracle of the same method (OpenMP, every host core)
            on a bounded sample of the same scene.
Multi-GPU: each rank runs an independent replica of the scene (its own seed);
a single dam break is not partitioned (replicas only), so there is no
collective on the step path -- one barrier and one max-reduction of the
timings.

--impl reference times the reference's own CPU implementation: its kernels
compiled as host code (oracle/_ref) with the reference's physics (fixed three
corrections) on the same scene, on every host core, rank 0 only.
"""
from __future__ import annotations

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

METRIC = "particle-steps/s, 1M-particle PCISPH dam break at eta=1%"
UNIT = "particle-steps/s"

# Algorithmic bytes per particle of each kernel (compulsory FP32 SoA
# traffic; neighbour re-reads and list traffic not counted).
ALG_BYTES = {
    "cell_keys": 24,          # pos 16 -> key + id 8
    "radix_sort": 16,         # one read + write of the (key, value) pairs
    "reorder": 77,            # pos, vel, pressure 36 in + 36 out, cell ranges 5
    "reorder_pos": 53,        # after an upload: slot + key 8, pos + id 20 in and out, cell ranges 5
    "reorder_state": 84,      # ... then slot 4, vel, half-step vel, (rho, p) 40 in and out
    "build_nbr": 24,          # pos 16 + key 4 -> count 4
    "density_x": 20,          # pos 16 -> rho 4 (learned: + vel 16, 8 features 32)
    "pci_init": 132,          # non-pressure forces 52 + first prediction 80
    "pci_density": 28,        # x* 16, p 4 -> p, rho* 8
    "pci_force_predict": 120,  # pressure force 40 + prediction 80
    "pci_commit": 96,         # final integrate, walls, interpolation
    "wcsph_force": 228,       # forces 52 + integrate 80 + walls/interpolation 96
    "mlp_infer": 36,          # features 32 -> initial pressure 4
}
TUNE_KEYS = ("bucket", "nbr_block", "nbr_schedule", "density_block", "init_block", "pci_density_block", "force_block",
             "xsph_block")


# Kernels per timed group (radix_sort is 3 kernels per 8-bit pass).
def _kernels_per_group(name: str, sort_passes: int) -> int:
    return 3 * sort_passes if name == "radix_sort" else 1


CORRECTOR_KERNELS = ("batch_begin", "pci_density", "batch_decide", "pci_force_predict")


def corrector_launches(prof: dict, steps: int, sort_passes: int, persistent: bool) -> int:
    """Kernel launches of `steps` steps from a per-kernel profile taken with
    the launches corrector; the persistent corrector replaces its four kinds
    of kernel with one launch per step."""
    total = sum(l * _kernels_per_group(k, sort_passes) for k, (l, _) in prof.items())
    if persistent:
        total -= sum(prof[k][0] for k in CORRECTOR_KERNELS if k in prof)
        total += steps
    return int(total)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference", "reference-cuda"], default="ours",
                    help="reference: the reference's kernels as host code on every core; reference-cuda: its own "
                         "CUDA path (kernels and PCISPH launcher compiled for this GPU), beside this build on the "
                         "same physics")
    ap.add_argument("--scene", default="C2")
    ap.add_argument("--warm-start", choices=["zero", "previous", "learned"], default="learned",
                    help="zero: plain PCISPH (each step's corrector starts from p = 0)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-steps", type=int, default=20)
    ap.add_argument("--mlp", choices=["silu6", "relu7"], default="silu6",
                    help="the learned warm start's network: silu6, the configured 6-input SiLU network, or relu7")
    ap.add_argument("--no-variant", action="store_true",
                    help="learned: do not train and compare the other network")
    ap.add_argument("--presolve", type=int, default=256, help="initial-pressure corrector passes before the warm-up")
    ap.add_argument("--train-steps", type=int, default=None,
                    help="plain-PCISPH steps recorded for training (learned; default 400, C3: 100)")
    ap.add_argument("--train-iters", type=int, default=10000, help="Adam steps (learned)")
    ap.add_argument("--train-batch", type=int, default=65536)
    ap.add_argument("--train-lr", type=float, default=3e-3, help="peak learning rate of the cosine schedule")
    ap.add_argument("--xsph", type=float, default=None, help="override the scene's XSPH velocity smoothing factor")
    ap.add_argument("--no-graph", action="store_true", help="launch kernel by kernel instead of CUDA graphs")
    ap.add_argument("--corrector", choices=["launches", "persistent", "both"], default="both",
                    help="the corrector loop: three kernels per correction, one cooperative launch per step, or "
                         "both timed and the faster one reported (config-profile PCISPH and C3)")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (default launch configuration)")
    ap.add_argument("--tune-cache", default=None,
                    help="JSON cache of tuned launch configurations: a bucket found there is not tuned again; "
                         "new results are added")
    ap.add_argument("--c1-no-whole-run", action="store_true",
                    help="C1: skip the untimed runs of all configured steps (implicit and staggered coupling)")
    ap.add_argument("--eval-steps", type=int, default=None,
                    help="steps after the recorded ones over which the warm starts are compared (0: skip)")
    args = ap.parse_args()
    short = args.scene in ("C3", "C4")
    if args.train_steps is None:
        args.train_steps = 100 if short else 400
    if args.eval_steps is None:
        args.eval_steps = 300 if short else 1000   # C3, C4: 300 steps
    return args



def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sms, maxs, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sms.append(float(parts[1]))
                    maxs.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sms)) if sms else None, "sm_max_mhz": max(maxs) if maxs else None,
                "reasons": sorted(reasons), "samples": len(sms)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """Per-particle DRAM bytes of each kernel from the committed ncu capture summary."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def cpu_baseline_port(sc, snap, steps: int, weights=None, arch: int = 0, boundary=None) -> dict:
    """The FP64 oracle (a C port of the same method, OpenMP on every host
    core) on a bounded sample: `steps` steps of the same scene from the same
    state the GPU's timed steps start from. With the learned warm start each
    step's initial pressure comes from the same network on the CPU (FP64
    features, BF16 rounding points) and the oracle's corrector starts there.
    boundary: the scene's static boundary particles, if any."""
    import oracle
    import psb_project_b200 as P
    learned = weights is not None and sc.warm_start == P.WARM_LEARNED
    osc = sc.replace(warm_start=P.WARM_PREVIOUS) if learned else sc
    bnd = None if boundary is None else np.asarray(boundary, np.float64)
    sim = oracle.OracleSim(osc, snap["pos"], snap["vel"], snap["vel_half"], snap["pressure"], boundary=bnd)
    t0 = time.perf_counter()
    iters = []
    for _ in range(steps):
        if learned:
            sim.p[:] = oracle.learned_pressure(sc, sim.pos, sim.vel, sim.p, weights, arch, bnd)
        iters.append(sim.step().iters)
    dt = time.perf_counter() - t0
    start = "learned warm start (CPU features and network)" if learned else \
        {P.WARM_ZERO: "zero start", P.WARM_PREVIOUS: "previous-pressure start"}.get(sc.warm_start, "")
    return {"value": sc.n * steps / dt, "unit": UNIT, "cores": host_cores(), "kind": "port",
            "iters_per_step": iters,
            "sample": f"{steps} steps of the {sc.n:,}-particle scene from the GPU's timed start state, {start} "
                      f"({sum(iters)} corrections, {np.mean(iters):.2f} per step), FP64 oracle, "
                      f"{host_cores()} threads on {cpu_model()}"}


def cpu_baseline_c1(fl, sp, fsnap, bsnap, steps: int) -> dict:
    """C1 on the CPU: the FP64 oracle's fluid and DEM steps coupled as the
    GPU couples them (the spheres as the fluid's boundary particles, their
    motion solved inside the fluid's corrector, the reaction of its last
    prediction as the spheres' external force), from the state the GPU's
    timed steps start from, OpenMP on every host core."""
    import oracle
    fluid = oracle.OracleSim(fl, fsnap["pos"], fsnap["vel"], fsnap["vel_half"], fsnap["pressure"],
                             boundary=np.asarray(bsnap["pos"], np.float64))
    balls = oracle.OracleSim(sp, bsnap["pos"], bsnap["vel"], bsnap["vel_half"])
    coupled = oracle.Coupling(fl, fluid, sp, balls, implicit=True)
    t0 = time.perf_counter()
    iters = []
    for _ in range(steps):
        iters.append(coupled.step()[0].iters)
    dt = time.perf_counter() - t0
    return {"value": (fl.n + sp.n) * steps / dt, "unit": UNIT, "cores": host_cores(), "kind": "port",
            "iters_per_step": iters,
            "sample": f"{steps} coupled steps of the {fl.n:,} fluid particles and {sp.n:,} spheres from the GPU's timed "
                      f"start state ({np.mean(iters):.2f} corrections per step), FP64 oracle, {host_cores()} threads "
                      f"on {cpu_model()}"}


def oracle_error(sim, sc, snap) -> dict:
    """The error of one GPU step against the FP64 oracle on the same state:
    the first step from the timed start state, through the C ABI; the oracle
    starts its corrector from the GPU's own initial pressure (the warm
    start's output, psb_warm_start), so both run the same method on the same
    inputs. Errors are relative: density element-wise, pressure and
    velocity to the field's max, position to the step's largest
    displacement."""
    import oracle
    import psb_project_b200 as P
    sim.upload(snap["pos"], snap["vel"], snap["vel_half"], snap["pressure"])
    _, p0 = sim.warm_start()
    sim.step(1)
    out = sim.download()
    sg = sim.stats()
    orc = oracle.OracleSim(sc.replace(warm_start=P.WARM_PREVIOUS), snap["pos"], snap["vel"], snap["vel_half"], p0)
    so = orc.step()
    rel = lambda a, b: float(np.max(np.abs(np.asarray(a, np.float64) - b)) / max(float(np.max(np.abs(b))), 1e-300))
    disp = float(np.max(np.abs(orc.pos - snap["pos"])))
    # The wall projection (collisionBox) acts on a particle whose predicted
    # position reaches the bound (x <= Min + r), and then removes its normal
    # velocity. A prediction within rounding of the bound can land on it in
    # FP32 and just inside it in FP64: the two results then differ by that
    # particle's normal velocity. Such particles are counted and reported
    # apart; the velocity error is over the others.
    r = np.float32(sc.particle_radius)
    lo = (np.asarray(sc.box_min, np.float32) + r).astype(np.float64)
    hi = (np.asarray(sc.box_max, np.float32) - r).astype(np.float64)
    on_b = lambda x: np.any((np.asarray(x, np.float64) <= lo) | (np.asarray(x, np.float64) >= hi), axis=1)
    flip = on_b(out["pos"]) != on_b(orc.pos)
    vmax = max(float(np.max(np.abs(orc.vel))), 1e-300)
    dv = np.max(np.abs(np.asarray(out["vel"], np.float64) - orc.vel), axis=1) / vmax
    return {"density": float(np.max(np.abs(out["density"] - orc.rho) / orc.rho)),
            "pressure": rel(out["pressure"], orc.p), "velocity": float(np.max(dv[~flip], initial=0.0)),
            "position": float(np.max(np.abs(out["pos"] - orc.pos))) / max(disp, 1e-300),
            "wall_projection_flips": int(np.count_nonzero(flip)),
            "velocity_at_flips": float(np.max(dv[flip], initial=0.0)),
            "iters_gpu": int(sg.iters), "iters_oracle": int(so.iters),
            "sample": "first step from the timed start state, FP32 GPU against the FP64 oracle from the same "
                      "initial pressure; density element-wise, pressure and velocity relative to the field max, "
                      "position relative to the step's largest displacement; velocity over the particles on whose "
                      "wall projection both agree (the others counted in wall_projection_flips)"}


def run_reference(args):
    from psb_project_b200.replicas import env_ranks
    rank, world, _ = env_ranks()
    if rank != 0:
        return
    import oracle
    import psb_project_b200 as P
    sc = P.config_scene(args.scene)
    sc_ref = P.dam_break(sc.blocks[0].nxyz, sc.blocks[0].spacing, sc.box_max, sc.h, method=P.PCISPH,
                         profile=P.PROFILE_REF, dt=sc.dt, mass=sc.mass, seed=sc.blocks[0].seed)
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference kernels built for the "
                          "host) is not present: build() compiles it where the reference tree exists"}))
        return
    pos = oracle.scene_positions(sc_ref).astype(np.float64)
    ref = oracle.RefSim(sc_ref, pos)
    for _ in range(args.warmup):
        ref.pcisph_update()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ref.pcisph_update()
    dt = time.perf_counter() - t0
    value = sc_ref.n * args.steps / dt
    cores = host_cores()
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{sc.name}: reference physics (3 fixed corrections)", "particles": sc_ref.n,
                   "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{args.steps} timed steps of the {sc_ref.n:,}-particle scene, the reference's "
                                   f"kernels run as host code on {cores} threads ({cpu_model()})"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def run_ours(args):
    import torch
    import psb_project_b200 as P

    from psb_project_b200 import replicas
    rep_ = replicas.init("nccl")
    rank, world, local = rep_.rank, rep_.world, rep_.local
    torch.cuda.set_device(local)

    modes = {"zero": P.WARM_ZERO, "previous": P.WARM_PREVIOUS, "learned": P.WARM_LEARNED}
    base = P.config_scene(args.scene)
    if args.xsph is not None:
        base = base.replace(xsph=args.xsph)
    if world > 1:       # replicas: same scene, own seed per rank
        base.blocks[0].seed = rep_.seed(base.blocks[0].seed)
    # a warm start is a PCISPH corrector's; WCSPH (C0) has none
    is_pci = base.method == P.PCISPH and base.profile == P.PROFILE_CONFIG
    sc = base.replace(warm_start=modes[args.warm_start] if is_pci else P.WARM_ZERO)
    n = sc.n
    stream = torch.cuda.current_stream()

    def barrier():
        rep_.barrier()
        torch.cuda.synchronize()

    max_over_ranks = rep_.max_over_ranks

    tune = None       # the autotuner's choice, given to every context created after it
    archs = {"silu6": P.runtime.MLP_SILU6, "relu7": P.runtime.MLP_RELU7}
    arch = archs[args.mlp]
    weights = {}      # trained networks by name

    corr_mode = None  # the faster corrector, given to every context created after it is known

    def make(mode, net=None, graph=True):
        s_ = P.Simulation(base.replace(warm_start=mode))
        s_.set_stream(stream.cuda_stream)
        if net is not None:
            s_.mlp_set_arch(archs[net])
            s_.mlp_set_weights(weights[net])
        if tune is not None:
            s_.tune_set(**{k: tune[k] for k in TUNE_KEYS})
        if graph and pcisph_cfg and not args.no_graph:
            s_.set_graph(True)
        if pcisph_cfg and corr_mode is not None:
            s_.set_corrector(corr_mode)
        return s_

    # Set-up (untimed): the dam at rest with its initial pressure, then plain
    # PCISPH for the recorded steps (learned: its converged pressures are the
    # training targets), then the warm-up. The timed passes all restart from
    # the snapshot taken after it.
    pcisph_cfg = sc.method == P.PCISPH and sc.profile == P.PROFILE_CONFIG
    gen = make(P.WARM_ZERO, graph=False)
    gen.upload(P.scene_positions(sc))
    if pcisph_cfg and args.presolve > 0:
        gen.presolve(args.presolve)      # initial pressure of the dam at rest
    train_info = None
    learned = sc.warm_start == P.WARM_LEARNED
    nets = [args.mlp] + ([] if args.no_variant else [k for k in archs if k != args.mlp])
    if learned:
        # plain PCISPH steps record (features, converged pressure); the 7-input
        # network's features include the 6-input one's, so one recording serves both
        t0 = time.perf_counter()
        gen.mlp_set_arch(P.runtime.MLP_RELU7)
        gen.mlp_collect(stride=64, capacity=max(1, (args.train_steps + 1) * ((n + 63) // 64)))
        gen.step(args.train_steps)
        gen.mlp_collect(0)
        rows, _, _ = gen.mlp_dataset(fetch=False)
        train_info = {"recorded_steps": args.train_steps, "rows": int(rows), "record_s": round(time.perf_counter() - t0, 2),
                      "adam_steps": args.train_iters // 10 * 10 + 1, "batch": args.train_batch, "lr": args.train_lr,
                      "schedule": "cosine, 10 chunks", "networks": {}}
        for net in nets:
            t1 = time.perf_counter()
            gen.mlp_set_arch(archs[net])
            gen.mlp_set_weights(P.mlp_init_weights(rank, archs[net]))
            loss0 = gen.mlp_train(1, args.train_batch, 1e-3, seed=11)
            loss = gen.mlp_fit(args.train_iters, args.train_batch, args.train_lr, chunks=10, seed=12)
            weights[net] = gen.mlp_get_weights()
            train_info["networks"][net] = {"params": int(weights[net].size), "loss_first": loss0, "loss_last": loss,
                                           "train_s": round(time.perf_counter() - t1, 2)}
        train_info["train_s"] = train_info["networks"][args.mlp]["train_s"]
    gen.step(args.warmup)
    snap = gen.download()
    gen.close()
    sim = make(sc.warm_start, args.mlp if learned else None)
    barrier()

    def restore(s):
        s.upload(snap["pos"], snap["vel"], snap["vel_half"], snap["pressure"])

    # A working set that L2 (126 MB) could hold between steps is flushed
    # before every timed step, outside the step's events (a 256 MB write).
    ws_mb = int(n * (3 * 16 * 2 + 8 * 2 + 4 * 2 + 16 * 4 + 8 + 4 + 4 * sc.nbr_cap + 4) / 1e6)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda") if ws_mb < 256 else None

    def device_pass(s, profile=False):
        restore(s)
        s.step(3)                 # untimed: captures the graphs on first use (the first step after an
                                  # upload has its own, then one per state parity)
        restore(s)
        if profile:
            s.profile(True)
            s.profile_reset()
        barrier()
        iters = []
        if flush is None:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                s.step(1)
                iters.append(s.stats().iters)
            e1.record(stream)
            barrier()
            ms_ = e0.elapsed_time(e1)
        else:
            ev = []
            for _ in range(args.steps):
                flush.fill_(1)
                a_, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a_.record(stream)
                s.step(1)
                b_.record(stream)
                iters.append(s.stats().iters)
                ev.append((a_, b_))
            barrier()
            ms_ = sum(a_.elapsed_time(b_) for a_, b_ in ev)
        prof = None
        if profile:
            prof = s.profile_read()
            s.profile(False)
        return max_over_ranks(ms_), iters, prof

    # ---- autotuner (untimed): launch configuration for this size bucket ----------
    if not args.no_tune:
        tune = tuned(sim, restore, args)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    # ---- device-resident timing, each corrector mode (same steps, same snapshot) ----
    modes_c = {"launches": P.CORRECTOR_LAUNCHES, "persistent": P.CORRECTOR_PERSISTENT}
    chosen = [args.corrector] if args.corrector != "both" or not pcisph_cfg else ["launches", "persistent"]
    if not pcisph_cfg:
        chosen = ["launches"]
    corr = {}
    for name in chosen:
        if pcisph_cfg:
            sim.set_corrector(modes_c[name])
        ms_c, it_c, _ = device_pass(sim)
        corr[name] = {"ms_per_step": ms_c / args.steps, "value": world * n * args.steps / (ms_c / 1e3),
                      "iters_mean": float(np.mean(it_c)), "ms": ms_c, "iters": it_c}
    best = min(corr, key=lambda k: corr[k]["ms"])
    ms_max, iters = corr[best]["ms"], corr[best]["iters"]
    value = world * n * args.steps / (ms_max / 1e3)
    # ---- per-kernel timing: the same K steps with CUDA events around every launch ----
    # (the launches corrector: its passes are separate kernels)
    if pcisph_cfg:
        sim.set_corrector(P.CORRECTOR_LAUNCHES)
    _, _, prof = device_pass(sim, profile=True)
    if pcisph_cfg:
        corr_mode = modes_c[best]
        sim.set_corrector(corr_mode)
    # ---- end to end through the C ABI with host buffers ------------------------------
    pin = lambda shape: torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()
    h = {"pos": pin((n, 3)), "vel": pin((n, 3)), "vel_half": pin((n, 3)), "density": pin((n,)), "pressure": pin((n,))}
    for k in ("pos", "vel", "vel_half", "pressure"):
        h[k][:] = snap[k]
    warm = sc.warm_start != P.WARM_ZERO
    barrier()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        sim.upload(h["pos"], h["vel"], h["vel_half"], h["pressure"] if warm else None)
        sim.step(1)
        sim.download(h if warm else {k: h[k] for k in ("pos", "vel", "vel_half", "density")})
    e3.record(stream)
    barrier()
    e2e_value = world * n * args.steps / (max_over_ranks(e2.elapsed_time(e3)) / 1e3)
    h2d = n * (36 + (4 if warm else 0))
    d2h = n * (40 + (4 if warm else 0))
    clk = clocks.stop()
    # ---- warm starts compared over the evaluation window ------------------------------
    # Every mode runs the same eval_steps steps from the snapshot (the steps
    # after the recorded ones), device-timed; each step's final density error
    # (the max of (rho* - rho0)/rho0 the loop stopped at) is kept so the modes
    # are compared at the same error statistics.
    def eval_pass(s):
        restore(s)
        s.step(3)                 # untimed graph capture, as in device_pass
        restore(s)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        its, errs = [], []
        e0.record(stream)
        for _ in range(args.eval_steps):
            s.step(1)
            st = s.stats()
            its.append(st.iters)
            errs.append(st.err[st.iters])
        e1.record(stream)
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1))
        its = np.asarray(its)
        errs = np.asarray(errs)
        return {"iters_mean": float(its.mean()), "iters_p50": float(np.median(its)), "iters_max": int(its.max()),
                "not_converged_steps": int(np.sum(its >= sc.max_iters)), "ms_per_step": ms / len(its),
                "value": world * n * len(its) / (ms / 1e3), "final_err_mean": float(errs.mean()),
                "final_err_max": float(errs.max())}

    comparison = {}
    if pcisph_cfg and args.eval_steps > 0:
        comparison["steps"] = "%d..%d of the dam break" % (
            (args.train_steps if train_info else 0) + args.warmup + 1,
            (args.train_steps if train_info else 0) + args.warmup + args.eval_steps)
        comparison[args.warm_start] = eval_pass(sim)
        if learned:
            comparison[args.warm_start]["network"] = args.mlp
        others = [("zero", P.WARM_ZERO, None), ("previous", P.WARM_PREVIOUS, None)]
        if learned:
            others += [("learned_" + net, P.WARM_LEARNED, net) for net in nets[1:]]
        for name, mode, net in others:
            if mode == sc.warm_start and net is None:
                continue
            other = make(mode, net)
            comparison[name] = eval_pass(other)
            other.close()
        this = comparison[args.warm_start]
        for name, _, _ in others:
            if name in comparison and name != args.warm_start:
                o = comparison[name]
                o["iters_ratio_over_" + args.warm_start] = o["iters_mean"] / max(this["iters_mean"], 1e-9)
                o["time_ratio_over_" + args.warm_start] = o["ms_per_step"] / this["ms_per_step"]
    sim.close()

    passes = (max(1, int(np.ceil(np.log2(np.prod(sc.dims))))) + 7) // 8
    launches = corrector_launches(prof, args.steps, passes, best == "persistent")
    tot_ms = sum(v[1] for v in prof.values())
    dom = max((k for k in prof if k in ALG_BYTES), key=lambda k: prof[k][1])
    l_dom, ms_dom = prof[dom]
    per_launch_s = ms_dom / l_dom / 1e3
    achieved = ALG_BYTES[dom] * n / per_launch_s / 1e9
    peak, peak_kind = peaks()
    traffic = ncu_traffic().get(dom)
    kernels = {k: {"launches": l, "ms": round(v, 3), "share": round(v / tot_ms, 4)} for k, (l, v) in prof.items()}

    cpu = None
    err = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_port(sc, snap, args.cpu_sample_steps, weights.get(args.mlp), arch)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": host_cores(), "kind": "port", "sample": f"failed: {ex}"}
        if pcisph_cfg:
            try:
                probe = make(sc.warm_start, args.mlp if learned else None, graph=False)
                err = oracle_error(probe, sc, snap)
                probe.close()
            except Exception as ex:
                err = {"failed": str(ex)}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": sc.name, "particles": n,
                       **({"eta": sc.eta, "min_iters": sc.min_iters, "max_iters": sc.max_iters,
                           "warm_start": args.warm_start, "xsph": sc.xsph} if pcisph_cfg else {"method": "WCSPH"}),
                       "dt": sc.dt, "h": sc.h, "network": args.mlp if learned else None,
                       "graph": pcisph_cfg and not args.no_graph, "corrector": best if pcisph_cfg else None,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": ("working set > L2 (state, lists and scratch ~%d MB per GPU)" % ws_mb) if flush is None
                             else ("L2 flushed before each timed step (256 MB write outside the step's events; "
                                   "working set ~%d MB per GPU)" % ws_mb),
                       "timed_steps": "steps %d..%d of the dam break" % (
                           (args.train_steps if train_info else 0) + args.warmup + 1,
                           (args.train_steps if train_info else 0) + args.warmup + args.steps),
                       "presolve_passes": args.presolve},
            "iters_per_step": {"mean": float(np.mean(iters)), "p50": float(np.median(iters)),
                               "p95": float(np.percentile(iters, 95)), "max": int(np.max(iters)),
                               "min": int(np.min(iters))},
            "corrector_modes": {k: {kk: v[kk] for kk in ("ms_per_step", "value", "iters_mean")} for k, v in corr.items()},
            "comparison": comparison,
            "learned_training": train_info,
            "autotune": tune,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None if traffic is None else traffic * n,
                         "alg_bytes_per_particle": ALG_BYTES[dom], "mean_launch_us": per_launch_s * 1e6},
            "kernels": kernels,
            "gpu_launches": launches,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "clocks": clk,
            "cpu_baseline": cpu,
            "oracle_error": err,
        }
        print(json.dumps(out))
    rep_.close()


def tuned(sim, restore, args) -> dict:
    """The launch configuration for the simulation's size bucket: from the
    cache file when it has the bucket, else measured by the autotuner on the
    restored state (and added to the cache)."""
    bucket = sim.size_bucket(sim.scene.n)
    if args.tune_cache and os.path.exists(args.tune_cache):
        sim.load_tune(args.tune_cache)
        t = sim.tune_get(bucket)
        if any(t[k] for k in sim.TUNE_FIELDS):
            t["source"] = args.tune_cache
            return t
    restore(sim)
    sim.step(2)
    t = sim.autotune(trials=5)
    if args.tune_cache:
        sim.save_tune(args.tune_cache)
    return t


def run_batch(args):
    """Config C3: 64 independent PCISPH dam breaks stepped as one batch
    (psb_create_batch), each step one CUDA-graph launch with the corrector a
    device-side while loop, the learned warm start on. Over N GPUs the scenes
    are split by size (replicas.assign_scenes) with no collective on the step
    path; the total work is fixed, so the scaling is strong."""
    import torch
    import psb_project_b200 as P
    from psb_project_b200 import replicas

    rep_ = replicas.init("nccl")
    rank, world, local = rep_.rank, rep_.world, rep_.local
    torch.cuda.set_device(local)
    modes = {"zero": P.WARM_ZERO, "previous": P.WARM_PREVIOUS, "learned": P.WARM_LEARNED}
    all_scenes = P.batch_scenes()
    mine = replicas.assign_scenes([s.n for s in all_scenes], world)[rank]
    scenes = [all_scenes[i].replace(warm_start=modes[args.warm_start]) for i in mine]
    n = sum(s.n for s in scenes)
    n_all = sum(s.n for s in all_scenes)
    stream = torch.cuda.current_stream()
    max_over_ranks = rep_.max_over_ranks

    def barrier():
        rep_.barrier()
        torch.cuda.synchronize()

    tune = None       # the autotuner's choice, given to every context created after it

    corr_mode = None  # the faster corrector, given to every context created after it is known

    def make(mode, graph=True):
        b = P.BatchSimulation([s.replace(warm_start=mode) for s in scenes])
        b.set_stream(stream.cuda_stream)
        b.set_graph(graph and not args.no_graph)
        if tune is not None:
            b.tune_set(**{k: tune[k] for k in TUNE_KEYS})
        if corr_mode is not None:
            b.set_corrector(corr_mode)
        return b

    # set-up (untimed): initial pressure, plain steps recorded for training, warm-up
    gen = make(P.WARM_ZERO, graph=False)
    gen.upload(P.batch_positions(scenes))
    gen.presolve(args.presolve)
    train_info, weights = None, None
    if args.warm_start == "learned":
        t0 = time.perf_counter()
        gen.mlp_collect(stride=64, capacity=(args.train_steps + 1) * ((n + 63) // 64))
        gen.step(args.train_steps)
        gen.mlp_collect(0)
        rows, _, _ = gen.mlp_dataset(fetch=False)
        t1 = time.perf_counter()
        gen.mlp_set_weights(P.mlp_init_weights(rank))
        loss0 = gen.mlp_train(1, args.train_batch, 1e-3, seed=11)
        loss = gen.mlp_fit(args.train_iters, args.train_batch, args.train_lr, chunks=10, seed=12)
        weights = gen.mlp_get_weights()
        train_info = {"recorded_steps": args.train_steps, "rows": int(rows), "adam_steps": args.train_iters // 10 * 10 + 1,
                      "batch": args.train_batch, "lr": args.train_lr, "schedule": "cosine, 10 chunks",
                      "loss_first": loss0, "loss_last": loss, "record_s": round(t1 - t0, 2),
                      "train_s": round(time.perf_counter() - t1, 2)}
    gen.step(args.warmup)
    snap = gen.download()
    parts = {k: gen.split(snap[k]) for k in ("pos", "vel", "vel_half", "pressure")}
    gen.close()
    start = (args.train_steps if train_info else 0) + args.warmup + 1

    def restore(b):
        b.upload(snap["pos"], snap["vel"], snap["vel_half"], snap["pressure"])

    def timed_pass(b, steps, profile=False):
        restore(b)
        b.step(3)                 # untimed: captures the graphs on first use, as in run_ours
        if profile:
            b.profile(True)
            b.profile_reset()
        before = b.batch_stats()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.step(steps)
        e1.record(stream)
        barrier()
        after = b.batch_stats()
        prof = None
        if profile:
            prof = b.profile_read()
            b.profile(False)
        per_scene = (after["iters_total"] - before["iters_total"]) / steps
        unconv = after["unconverged_steps"] - before["unconverged_steps"]
        return max_over_ranks(e0.elapsed_time(e1)), per_scene, unconv, prof

    sim = make(modes[args.warm_start])
    if weights is not None:
        sim.mlp_set_weights(weights)
    if not args.no_tune:
        tune = tuned(sim, restore, args)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    modes_c = {"launches": P.CORRECTOR_LAUNCHES, "persistent": P.CORRECTOR_PERSISTENT}
    chosen = ["launches", "persistent"] if args.corrector == "both" else [args.corrector]
    corr = {}
    for name in chosen:
        sim.set_corrector(modes_c[name])
        ms_c, ps_c, unc_c, _ = timed_pass(sim, args.steps)
        corr[name] = {"ms_per_step": ms_c / args.steps, "value": n_all * args.steps / (ms_c / 1e3),
                      "iters_mean": float(np.mean(ps_c)), "ms": ms_c, "per_scene": ps_c, "unconv": unc_c}
    best = min(corr, key=lambda k: corr[k]["ms"])
    ms_max, per_scene, unconv = corr[best]["ms"], corr[best]["per_scene"], corr[best]["unconv"]
    value = n_all * args.steps / (ms_max / 1e3)
    sim.set_corrector(P.CORRECTOR_LAUNCHES)      # per-kernel profile: the passes as separate kernels
    _, _, _, prof = timed_pass(sim, min(args.steps, 20), profile=True)
    corr_mode = modes_c[best]
    sim.set_corrector(corr_mode)
    # end to end: host buffers in and out every step
    pin = lambda shape: torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()
    h = {"pos": pin((n, 3)), "vel": pin((n, 3)), "vel_half": pin((n, 3)), "density": pin((n,)), "pressure": pin((n,))}
    for k in ("pos", "vel", "vel_half", "pressure"):
        h[k][:] = snap[k]
    barrier()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        sim.upload(h["pos"], h["vel"], h["vel_half"], h["pressure"])
        sim.step(1)
        sim.download(h)
    e3.record(stream)
    barrier()
    e2e_value = n_all * args.steps / (max_over_ranks(e2.elapsed_time(e3)) / 1e3)
    clk = clocks.stop()
    # learned vs plain over the evaluation window, from the same snapshot
    comparison = {}
    if args.eval_steps > 0:
        comparison["steps"] = "%d..%d of every scene" % (start + 2, start + 1 + args.eval_steps)
        for name, mode in (("learned", P.WARM_LEARNED), ("zero", P.WARM_ZERO)):
            if name == "learned" and weights is None:
                continue
            b = sim if mode == modes[args.warm_start] else make(mode)
            if weights is not None:
                b.mlp_set_weights(weights)
            ms, ps, unc, _ = timed_pass(b, args.eval_steps)
            comparison[name] = {"iters_mean": float(np.mean(ps)), "iters_mean_weighted": float(np.average(ps, weights=[s.n for s in scenes])),
                                "unconverged_steps": int(np.sum(unc)), "ms_per_step": ms / args.eval_steps,
                                "value": n_all * args.eval_steps / (ms / 1e3)}
            if b is not sim:
                b.close()
        if "learned" in comparison:
            z, l_ = comparison["zero"], comparison["learned"]
            z["iters_ratio_over_learned"] = z["iters_mean"] / max(l_["iters_mean"], 1e-9)
            z["time_ratio_over_learned"] = z["ms_per_step"] / l_["ms_per_step"]
    sim.close()

    passes = (max(1, int(np.ceil(np.log2(sum(int(np.prod(s.dims)) for s in scenes))))) + 7) // 8
    prof_steps = min(args.steps, 20)
    launches = corrector_launches(prof, prof_steps, passes, best == "persistent")
    tot_ms = sum(v[1] for v in prof.values())
    # the corrector passes skip the scenes that have converged, so their
    # launches do not cover every particle: the roofline kernel is the
    # costliest of the sweeps that do
    partial = ("pci_density", "pci_force_predict")
    dom = max((k for k in prof if k in ALG_BYTES and k not in partial), key=lambda k: prof[k][1])
    l_dom, ms_dom = prof[dom]
    per_launch_s = ms_dom / l_dom / 1e3
    achieved = ALG_BYTES[dom] * n / per_launch_s / 1e9
    peak, peak_kind = peaks()
    kernels = {k: {"launches": l, "ms": round(v, 3), "share": round(v / tot_ms, 4)} for k, (l, v) in prof.items()}
    # CPU baseline: the oracle on the first scenes of this rank's share, up to
    # ~150k particles, each from its own timed start state
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            done_n, secs, its, picked = 0, 0.0, [], 0
            for s_i, sc_i in enumerate(scenes):
                if done_n >= 150000:
                    break
                one = cpu_baseline_port(sc_i, {k: parts[k][s_i] for k in parts}, args.cpu_sample_steps, weights)
                done_n += sc_i.n
                secs += sc_i.n * args.cpu_sample_steps / one["value"]
                its += one["iters_per_step"]
                picked += 1
            cpu = {"value": done_n * args.cpu_sample_steps / secs, "unit": UNIT, "cores": host_cores(), "kind": "port",
                   "sample": f"{args.cpu_sample_steps} steps of each of the first {picked} scenes ({done_n:,} particles) "
                             f"from their timed start states, {args.warm_start} start ({np.mean(its):.2f} corrections "
                             f"per scene-step), FP64 oracle, {host_cores()} threads on {cpu_model()}"}
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": host_cores(), "kind": "port", "sample": f"failed: {ex}"}
    if rank == 0:
        out = {
            "metric": "particle-steps/s, 64 batched PCISPH dam breaks at eta=1% (C3)", "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "C3: 64 PCISPH dam breaks, N log-uniform in [4096, 131072], seed 3",
                       "particles": n_all, "scenes": len(all_scenes), "scenes_on_rank0": len(scenes),
                       "eta": scenes[0].eta, "warm_start": args.warm_start, "dt": scenes[0].dt, "h": scenes[0].h,
                       "graph": not args.no_graph, "corrector": best,
                       "parallelism": f"scenes split over {world} GPUs by size" if world > 1 else "single GPU",
                       "l2": "working set > L2 (~%d MB)" % int(n * (3 * 16 * 2 + 8 * 2 + 4 * 2 + 16 * 4 + 8 + 4 + 4 * scenes[0].nbr_cap + 4) / 1e6),
                       "timed_steps": "steps %d..%d of every scene" % (start + 2, start + 1 + args.steps)},
            "iters_per_step": {"mean_over_scenes": float(np.mean(per_scene)), "max_scene": float(np.max(per_scene)),
                               "min_scene": float(np.min(per_scene)), "unconverged_steps": int(np.sum(unconv))},
            "corrector_modes": {k: {kk: v[kk] for kk in ("ms_per_step", "value", "iters_mean")} for k, v in corr.items()},
            "comparison": comparison,
            "learned_training": train_info,
            "autotune": tune,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                         "alg_bytes_per_particle": ALG_BYTES[dom], "mean_launch_us": per_launch_s * 1e6},
            "kernels": kernels, "kernels_steps": prof_steps,
            "gpu_launches": int(launches * args.steps / prof_steps),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": n_all * 40, "d2h_bytes_per_step": n_all * 44},
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(out))
    rep_.close()


C4_SPHERE = ((1.5, 0.21, 0.5), 0.2)     # centre (m), radius (m): in the path of the collapsing block


def run_c4(args):
    """Config C4: the 4,194,304-particle PCISPH dam break (eta 0.5 %) around a
    static 0.2 m sphere sampled as boundary particles, learned warm start,
    with the density colour field's iso-0.5 surface extracted on a 256^3
    node grid every 10 steps (marching cubes on the GPU, the mesh copied to
    the host). `value` counts particle-steps over the wall time of steps and
    extractions together. Multi-GPU: replicas with their own seeds."""
    import torch
    import psb_project_b200 as P
    from psb_project_b200 import replicas

    rep_ = replicas.init("nccl")
    rank, world, local = rep_.rank, rep_.world, rep_.local
    torch.cuda.set_device(local)
    modes = {"zero": P.WARM_ZERO, "previous": P.WARM_PREVIOUS, "learned": P.WARM_LEARNED}
    base = P.config_scene("C4")
    if world > 1:
        base.blocks[0].seed = rep_.seed(base.blocks[0].seed)
    sc = base.replace(warm_start=modes[args.warm_start])
    n = sc.n
    centre, radius = C4_SPHERE
    bnd = P.sphere_shell(centre, radius, sc.spacing)
    grid = P.iso_grid((0.0, 0.0, 0.0), tuple(b / 255.0 for b in sc.box_max), (256, 256, 256))
    stream = torch.cuda.current_stream()
    max_over_ranks = rep_.max_over_ranks
    tune = None

    def barrier():
        rep_.barrier()
        torch.cuda.synchronize()

    def make(mode):
        s_ = P.Simulation(base.replace(warm_start=mode))
        s_.set_stream(stream.cuda_stream)
        s_.set_boundary(bnd)
        if tune is not None:
            s_.tune_set(**{k: tune[k] for k in TUNE_KEYS})
        return s_

    gen = make(P.WARM_ZERO)
    gen.upload(P.scene_positions(sc))
    gen.presolve(args.presolve)
    train_info, weights = None, None
    if args.warm_start == "learned":
        t0 = time.perf_counter()
        gen.mlp_collect(stride=64, capacity=(args.train_steps + 1) * ((n + 63) // 64))
        gen.step(args.train_steps)
        gen.mlp_collect(0)
        rows, _, _ = gen.mlp_dataset(fetch=False)
        t1 = time.perf_counter()
        gen.mlp_set_weights(P.mlp_init_weights(rank))
        loss0 = gen.mlp_train(1, args.train_batch, 1e-3, seed=11)
        loss = gen.mlp_fit(args.train_iters, args.train_batch, args.train_lr, chunks=10, seed=12)
        weights = gen.mlp_get_weights()
        train_info = {"recorded_steps": args.train_steps, "rows": int(rows), "adam_steps": args.train_iters // 10 * 10 + 1,
                      "batch": args.train_batch, "lr": args.train_lr, "loss_first": loss0, "loss_last": loss,
                      "record_s": round(t1 - t0, 2), "train_s": round(time.perf_counter() - t1, 2)}
    gen.step(args.warmup)
    snap = gen.download()
    gen.close()
    start = (args.train_steps if train_info else 0) + args.warmup + 1

    def restore(s_):
        s_.upload(snap["pos"], snap["vel"], snap["vel_half"], snap["pressure"])

    sim = make(modes[args.warm_start])
    if weights is not None:
        sim.mlp_set_weights(weights)
    if not args.no_tune:
        tune = tuned(sim, restore, args)
    vert = np.empty((16 << 20, 3), np.float32)
    tri = np.empty((32 << 20, 3), np.int32)

    def timed_run(s_, steps, mc_every):
        restore(s_)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        its, mesh, mc_ev = [], (0, 0), []
        e0.record(stream)
        for k in range(steps):
            s_.step(1)
            its.append(s_.stats().iters)
            if mc_every and (k + 1) % mc_every == 0:
                m0 = torch.cuda.Event(enable_timing=True)
                m1 = torch.cuda.Event(enable_timing=True)
                m0.record(stream)
                mesh = s_.extract_surface_into(grid, 0.5, vert, tri)
                m1.record(stream)
                mc_ev.append((m0, m1))
        e1.record(stream)
        barrier()
        mc_ms = sum(a.elapsed_time(b) for a, b in mc_ev)       # the extractions' own device time
        timed_run.mc_ms = max_over_ranks(mc_ms)
        return max_over_ranks(e0.elapsed_time(e1)), np.asarray(its), mesh

    restore(sim)
    sim.step(3)                                      # untimed: the step's graphs are captured here
    sim.extract_surface_into(grid, 0.5, vert, tri)   # untimed: the extraction's buffers are allocated here
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    ms, its, mesh = timed_run(sim, args.steps, 10)
    mc_total_ms = timed_run.mc_ms
    value = world * n * args.steps / (ms / 1e3)
    ms_nomc, its_nomc, _ = timed_run(sim, args.steps, 0)
    # end to end through the C ABI: host buffers in and out every step, the
    # extractions' meshes copied to the host as in the timed run
    pin = lambda shape: torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()
    h = {"pos": pin((n, 3)), "vel": pin((n, 3)), "vel_half": pin((n, 3)), "density": pin((n,)), "pressure": pin((n,))}
    for k in ("pos", "vel", "vel_half", "pressure"):
        h[k][:] = snap[k]
    barrier()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for k in range(args.steps):
        sim.upload(h["pos"], h["vel"], h["vel_half"], h["pressure"])
        sim.step(1)
        sim.download(h)
        if (k + 1) % 10 == 0:
            sim.extract_surface_into(grid, 0.5, vert, tri)
    e3.record(stream)
    barrier()
    e2e_value = world * n * args.steps / (max_over_ranks(e2.elapsed_time(e3)) / 1e3)
    clk = clocks.stop()
    diag = sim.diagnostics()
    comparison = {}
    if args.eval_steps > 0 and weights is not None:
        comparison["steps"] = "%d..%d" % (start, start + args.eval_steps - 1)
        for name, mode in (("learned", P.WARM_LEARNED), ("zero", P.WARM_ZERO)):
            b = sim if mode == modes[args.warm_start] else make(mode)
            if weights is not None:
                b.mlp_set_weights(weights)
            m_, it_, _ = timed_run(b, args.eval_steps, 0)
            comparison[name] = {"iters_mean": float(it_.mean()), "iters_p50": float(np.median(it_)),
                                "not_converged_steps": int(np.sum(it_ >= sc.max_iters)),
                                "ms_per_step": m_ / args.eval_steps}
            if b is not sim:
                b.close()
        z, l_ = comparison["zero"], comparison["learned"]
        z["iters_ratio_over_learned"] = z["iters_mean"] / max(l_["iters_mean"], 1e-9)
        z["time_ratio_over_learned"] = z["ms_per_step"] / l_["ms_per_step"]
    sim.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # a 20-step sample of 4.2M particles would take minutes on the host:
        # two steps, the same state and start
        try:
            cpu = cpu_baseline_port(sc, snap, min(args.cpu_sample_steps, 2), weights, 0, bnd)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": host_cores(), "kind": "port", "sample": f"failed: {ex}"}
    if rank == 0:
        mc_ms = mc_total_ms / max(1, args.steps // 10)
        out = {
            "metric": "particle-steps/s, 4M-particle PCISPH dam break with a sphere obstacle and MC every 10 steps (C4)",
            "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": sc.name + " + 0.2 m sphere obstacle + MC 256^3 every 10 steps", "particles": n,
                       "boundary_particles": int(bnd.shape[0]), "sphere": {"centre": centre, "radius": radius},
                       "eta": sc.eta, "warm_start": args.warm_start, "dt": sc.dt, "h": sc.h,
                       "timed_steps": "steps %d..%d" % (start, start + args.steps - 1),
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "iters_per_step": {"mean": float(its.mean()), "p50": float(np.median(its)), "max": int(its.max())},
            "mc": {"grid": [256, 256, 256], "level": 0.5, "ms_per_extraction": mc_ms, "vertices": int(mesh[0]),
                   "triangles": int(mesh[1])},
            "ms_per_step_without_mc": ms_nomc / args.steps,
            "iters_per_step_without_mc": float(its_nomc.mean()),
            "diagnostics_fp64": diag,
            "comparison": comparison, "learned_training": train_info, "autotune": tune,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": n * 40, "d2h_bytes_per_step": n * 44},
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(out))
    rep_.close()


def run_c1(args):
    """Config C1: the 262,144-particle PCISPH dam break (eta 1 %, dt 1e-3)
    with 4,096 DEM spheres dropped from above it, coupled two ways through
    boundary particles (psb_project_b200.FluidDemCoupling): each step the
    fluid steps with the spheres as its boundary, its reaction on every
    sphere is the spheres' external force, and the spheres step. `value`
    counts fluid and sphere particle-steps over the device time of the
    coupled steps, the per-step host exchange of sphere positions and forces
    included (that exchange is also the `e2e` traffic). Multi-GPU: replicas."""
    import torch
    import psb_project_b200 as P
    from psb_project_b200 import replicas

    rep_ = replicas.init("nccl")
    rank, world, local = rep_.rank, rep_.world, rep_.local
    torch.cuda.set_device(local)
    fl, sp = P.c1_scenes(seed=1 + (replicas.SEED_STRIDE * rank if world > 1 else 0))
    stream = torch.cuda.current_stream()
    fluid, balls = P.Simulation(fl), P.Simulation(sp)
    for s_ in (fluid, balls):
        s_.set_stream(stream.cuda_stream)
    fluid.upload(P.scene_positions(fl))
    fluid.presolve(args.presolve)
    balls.upload(P.scene_positions(sp))
    coupled = P.FluidDemCoupling(fluid, balls)
    coupled.step(args.warmup)
    fsnap, bsnap = fluid.download(), balls.download()

    def barrier():
        rep_.barrier()
        torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    iters = []
    e0.record(stream)
    for _ in range(args.steps):
        coupled.step(1)
        iters.append(fluid.stats().iters)
    e1.record(stream)
    barrier()
    ms = rep_.max_over_ranks(e0.elapsed_time(e1))
    clk = clocks.stop()
    n_all = fl.n + sp.n
    value = world * n_all * args.steps / (ms / 1e3)
    fluid.profile(True)
    balls.profile(True)
    coupled.step(min(args.steps, 20))
    prof = {("fluid:" + k): v for k, v in fluid.profile_read().items()}
    prof.update({("dem:" + k): v for k, v in balls.profile_read().items()})
    bpos = balls.download()["pos"]
    in_fluid = int(np.sum(bpos[:, 1] < fl.blocks[0].nxyz[1] * fl.blocks[0].spacing))
    diag = fluid.diagnostics()
    fluid.close()
    balls.close()

    def whole_run(implicit):
        """The configured steps from the start, untimed: corrections per
        window of 50 steps and where the spheres are."""
        f_, b_ = P.Simulation(fl), P.Simulation(sp)
        f_.upload(P.scene_positions(fl))
        f_.presolve(args.presolve)
        b_.upload(P.scene_positions(sp))
        c_ = P.FluidDemCoupling(f_, b_, implicit=implicit)
        its_, win = [], []
        t_ = time.perf_counter()
        for k in range(fl.steps):
            c_.step(1)
            its_.append(f_.stats().iters)
            if (k + 1) % 50 == 0:
                w = np.array(its_[-50:])
                y = b_.download()["pos"][:, 1]
                win.append({"steps": f"{k - 48}..{k + 1}", "iters_mean": float(w.mean()), "iters_p50": float(np.median(w)),
                            "not_converged": int(np.count_nonzero(w >= fl.max_iters)), "spheres_y_mean": float(y.mean())})
        f_.close()
        b_.close()
        a_ = np.array(its_)
        return {"steps": fl.steps, "iters_mean": float(a_.mean()), "iters_p50": float(np.median(a_)),
                "not_converged": int(np.count_nonzero(a_ >= fl.max_iters)), "wall_s": round(time.perf_counter() - t_, 1),
                "windows": win}

    runs = {"implicit": whole_run(True), "staggered": whole_run(False)} if not args.c1_no_whole_run else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_c1(fl, sp, fsnap, bsnap, args.cpu_sample_steps)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": host_cores(), "kind": "port", "sample": f"failed: {ex}"}
    if rank == 0:
        tot = sum(v[1] for v in prof.values())
        out = {
            "metric": "particle-steps/s, 262,144-particle PCISPH dam break coupled with 4,096 DEM spheres (C1)",
            "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": fl.name + " + " + sp.name, "fluid_particles": fl.n, "spheres": sp.n,
                       "eta": fl.eta, "dt": fl.dt, "coupling": "spheres as boundary particles, two-way",
                       "timed_steps": "steps %d..%d" % (args.warmup + 1, args.warmup + args.steps),
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "iters_per_step": {"mean": float(np.mean(iters)), "p50": float(np.median(iters)), "max": int(np.max(iters))},
            "spheres_below_fluid_top_at_end": in_fluid,
            "coupling": "implicit: the spheres' motion solved inside the fluid's corrector",
            "whole_run": runs,
            "kernels": {k: {"launches": l, "ms": round(v, 3), "share": round(v / tot, 4)} for k, (l, v) in prof.items()},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 24 * sp.n, "d2h_bytes_per_step": 24 * sp.n},
            "diagnostics_fp64": diag, "clocks": clk, "cpu_baseline": cpu,
        }
        print(json.dumps(out))
    rep_.close()


def run_reference_cuda(args):
    """The reference's own CUDA path on this GPU: its kernel files and its
    pci_SPH_update launcher compiled unchanged for sm_100a
    (oracle/_ref/libpsbref_cuda.so), stepped through PCI_SPHSystem::update's
    (or SPHSystem::update's, C0) call sequence, with the reference's physics
    (three fixed corrections, FP64). Timed on the device over the reference's
    own work (the guards that refuse out-of-bounds steps are not timed).
    Beside it, this build on the same physics (reference profile, same scene
    and start), device-timed the same way. Rank 0 only."""
    from psb_project_b200.replicas import env_ranks
    rank, world, _ = env_ranks()
    if rank != 0:
        return
    import oracle
    import torch
    import psb_project_b200 as P
    sc = P.config_scene(args.scene)
    method = P.WCSPH if sc.method == P.WCSPH else P.PCISPH
    sc_ref = P.dam_break(sc.blocks[0].nxyz, sc.blocks[0].spacing, sc.box_max, sc.h, method=method,
                         profile=P.PROFILE_REF, dt=sc.dt, mass=sc.mass, seed=sc.blocks[0].seed)
    name = "reference-cuda"
    if not oracle.refcuda_available():
        print(json.dumps({"impl": name, "unavailable": "oracle/_ref/libpsbref_cuda.so (the reference's CUDA files "
                          "compiled for this GPU) is not present: build() compiles it where the reference tree "
                          "exists"}))
        return
    pos = oracle.scene_positions(sc_ref).astype(np.float64)
    ref = oracle.RefCudaSim(sc_ref, pos)
    stepf = ref.pcisph_update if method == P.PCISPH else ref.wcsph_update
    try:
        for _ in range(args.warmup):
            stepf()
        t0 = time.perf_counter()
        ms = [stepf() for _ in range(args.steps)]
        wall = time.perf_counter() - t0
    except RuntimeError as ex:
        print(json.dumps({"impl": name, "unavailable": f"the reference's step was refused by the guard: {ex}"}))
        return
    value = sc_ref.n * args.steps / (sum(ms) / 1e3)
    # this build on the same physics from the same start
    stream = torch.cuda.current_stream()
    with P.Simulation(sc_ref) as sim:
        sim.set_stream(stream.cuda_stream)
        sim.upload(pos.astype(np.float32))
        sim.step(args.warmup)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.step(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ours_ms = e0.elapsed_time(e1)
    ours = sc_ref.n * args.steps / (ours_ms / 1e3)
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "impl": name, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sum(ms) / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{sc.name}: reference physics ({'3 fixed corrections' if method == P.PCISPH else 'WCSPH'})",
                   "particles": sc_ref.n, "dt": sc_ref.dt, "parallelism": "single GPU"},
        "wall_ms_per_step": wall * 1e3 / args.steps,
        "same_physics_this_build": {"value": ours, "ms_per_step": ours_ms / args.steps, "dtype": "f32",
                                    "ratio_over_reference": ours / value},
    }))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.impl == "reference-cuda":
        run_reference_cuda(args)
    elif args.scene == "C3":
        run_batch(args)
    elif args.scene == "C4":
        run_c4(args)
    elif args.scene == "C1":
        run_c1(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
