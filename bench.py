"""Benchmark of the B200 pair_style tensormd path: MD atom-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config bcc128k|fcc4k|alloy432k|alloy55k]

Workload (default): BCC a = 2.87 A, 40x40x40 cells = 128,000 atoms, Gaussian
displacements sigma = 0.08 A, 600 K Maxwell velocities, one element, 16
Gaussian radial functions, rc = 6.0 A cosine cutoff, moments of rank <= 3,
MLP 64-64-64-1 tanh (random weights, seeded), NVE dt = 1 fs, neighbor skin
1.0 A.  A step is one velocity-Verlet MD step: half kick + drift, rebuild
check (rebuild when an atom moved more than skin/2), descriptor, MLP and its
backward, pair forces, gather, half kick.

value: atom-steps/s with all state resident in HBM (tmd_nve_run), timed with
CUDA events on the library's stream, max over ranks.  e2e: the same metric
through the reference-facing call pattern with host buffers (per step: H2D of
positions from pinned memory, force evaluation, D2H of forces, velocity
Verlet on the host, as LAMMPS drives PairTensorMD::compute).  N > 1 GPUs run
independent replicas (weak scaling, no collective in the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "lammps-tensormd_b200"))

METRIC = "atom-steps/s on 1 B200, BF16 vs plain FP32 at stated force err; p50/p99 latency"
UNIT = "atom-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="bcc128k")
    ap.add_argument("--e2e-steps", type=int, default=50)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-bf16", action="store_true")
    ap.add_argument("--profile-step", type=int, default=0, metavar="N",
                    help="profiler target: set up the headline workload with the default "
                         "kernel forms, run N force evaluations, print nothing else")
    ap.add_argument("--profile-precision", default="fp32",
                    choices=["fp32", "tf32x3", "bf16x3", "bf16"],
                    help="MLP precision form of the --profile-step target")
    ap.add_argument("--profile-desc", default="", choices=["", "filter4", "wide", "wide2", "split"],
                    help="descriptor form of the --profile-step target (default: the "
                         "library's default form)")
    ap.add_argument("--main-only", action="store_true",
                    help="only the headline workload (no precision forms, cells, serving, "
                         "reference-workload or CPU lines): for profiler launch lists")
    ap.add_argument("--cells-steps", type=int, default=500,
                    help="NVE steps of the 4,096-cell batch line (0 skips it)")
    ap.add_argument("--precision-steps", type=int, default=20,
                    help="NVE steps per MLP form of the 432,000-atom precision line (0 skips it)")
    ap.add_argument("--decomp-steps", type=int, default=0,
                    help="spatial decomposition line: NVE steps of the headline cell cut into "
                         "one slab per rank (tmd_b200.decomp; 0 skips it)")
    ap.add_argument("--drift-steps", type=int, default=0,
                    help="energy-drift line: NVE steps of the shipped W_k32 potential on "
                         "432,000 BCC atoms after 1,000 steps of fix nvt 300 K (0 skips it)")
    ap.add_argument("--serve-rate", type=float, default=2000.0,
                    help="serving line: Poisson arrival rate (jobs/s)")
    ap.add_argument("--serve-sweep", default="250,500,1000",
                    help="serving line: further arrival rates (jobs/s, comma separated; "
                         "empty skips), each served by every MLP form")
    ap.add_argument("--serve-window", type=float, default=2.0,
                    help="serving line: seconds of arrivals (0 skips it)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(value, world, device):
    """The largest of every rank's value, on every rank (the slowest replica's
    time is the job's time)."""
    import torch
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(atoms_per_rank, steps, world, ms_max):
    """Whole-job atom-steps/s of `world` replicas of `atoms_per_rank` atoms that
    each ran `steps` steps, timed by the slowest one (ms_max milliseconds)."""
    return atoms_per_rank * steps * world / (ms_max / 1000.0)


def workload(cfg_name, seed):
    from tmd_b200 import synth
    c = synth.config(cfg_name)
    tmp = Path(tempfile.mkdtemp(prefix="tmdbench"))
    pot = tmp / f"{cfg_name}.npz"
    syms = synth.gaussian_potential(pot, seed=1234, **c["pot"])
    x, t, box, v = synth.build_system(c["kind"], c["a"], c["cells"], sigma=c["sigma"],
                                      T=c["T"], nelt=c["nelt"], seed=seed)
    cfg = {"workload": cfg_name, "natoms": int(len(x)), "lattice": c["kind"], "a": c["a"],
           "cells": list(c["cells"]), "elements": c["nelt"],
           "num_filters": c["pot"]["num_filters"], "rc": c["pot"]["rc"],
           "max_moment": c["pot"]["max_moment"],
           "mlp": [c["pot"]["nelt"] * c["pot"]["num_filters"] * (c["pot"]["max_moment"] + 1)]
           + list(c["pot"]["hidden"]) + [1],
           "actfn": {1: "softplus", 2: "tanh", 3: "squareplus"}[c["pot"]["actfn"]],
           "dt_fs": 1.0, "skin": 1.0, "sigma": c["sigma"], "T": c["T"]}
    return str(pot), syms, x, t, box, v, cfg


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            p = [q.strip() for q in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, val in zip(names, p[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "window": "the whole bench run (every leg), nvidia-smi every 200 ms"}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def fp32_peak_tflops(lib, device):
    """FP32 issue peak measured in this run: the library's packed-FMA (FFMA2)
    microkernel on every SM, best of 5 event-timed launches."""
    import ctypes
    from tmd_b200.lib import check
    tf = ctypes.c_double()
    check(lib.tmd_fp32_peak(int(device), 5, ctypes.byref(tf)))
    return tf.value


def step_bytes_s8d(n, nlist, nin, rebuild_period):
    """Algorithmic HBM bytes of one MD step as the survey's roofline section
    defines them for a fused design: read x (24 B) and type (4 B), write f
    (24 B), read and write v (48 B), write x (24 B), read the neighbor list
    (4 B per entry) and write it once per rebuild period, and the MLP staging
    G + dE/dG written and read (4 x 2 x 2 x nin B).  The design's own staging
    between kernels is not counted."""
    per_atom = 24 + 4 + 24 + 48 + 24 + 16 * nin
    return n * per_atom + nlist * 4 * (1.0 + 1.0 / max(rebuild_period, 1.0))


def ncu_traffic(config, kernel):
    """Per-launch DRAM bytes (read + write) of a kernel, from the committed ncu
    summary of the same workload (profiles/step_kernels_<config>.md, line
    `traffic_bytes_per_launch <kernel>: N`), or None."""
    p = ROOT / "profiles" / f"step_kernels_{config}.md"
    if not p.exists():
        return None
    key = f"traffic_bytes_per_launch {kernel}:"
    for line in p.read_text().splitlines():
        if key in line:
            try:
                return int(line.split(key)[1].split()[0])
            except ValueError:
                return None
    return None


def algorithmic(cfg, npairs_rc, nlist, B, K, D, nin, form):
    """Algorithmic FLOPs and HBM bytes per launch of the force kernel.

    FLOPs, the per-atom work of the force step (everything after the MLP but
    the gather): per pair inside rc the U and V contractions 2 x (2 K D)
    (tensor_ops.cpp kernel_U / kernel_V), the radial functions and their
    derivatives 10 K, F1 2 K + 3, F2 2 D + 3 and the monomial derivatives 6 D;
    per atom and element block dE/dP (2 M + 1) D K (M invariants per filter,
    tensor_ops.cpp kernel_dEdS).  Bytes, each input read once and
    each output written once: P (4 B K D B/atom), G and dE/dG (2 x 4 nin),
    virial partials (48 B/atom), and per pair either (pair-lane forms) the
    descriptor step's compact pair geometry (32 B per pair inside rc) and the
    pair force (16 B), or (filter-lane form) x (24 B/atom), the neighbor row
    (4 B/entry) and the pair force of every entry (16 B)."""
    n = cfg["natoms"]
    M = {1: 1, 4: 2, 10: 3, 20: 4}[D]
    flops = npairs_rc * (4.0 * K * D + 10.0 * K + (2 * K + 3) + (2 * D + 3) + 6.0 * D) \
        + n * B * (2 * M + 1) * D * K
    per_atom = 4 * B * K * D + 8 * nin + 48
    if form == "filter_lane":
        bytes_ = n * (24 + per_atom) + nlist * (4 + 16)
    else:
        bytes_ = n * (per_atom + 4 * B) + npairs_rc * (32 + 16)
    return flops, bytes_


def run_ours(args, rank, world, local):
    # clocks and throttle reasons sampled (nvidia-smi, every 200 ms) over the
    # whole run: the headline's timed region alone is often shorter than one
    # sampling interval
    clk = ClockSampler(local).__enter__()
    try:
        run_ours_sampled(args, rank, world, local, clk)
    finally:
        clk.__exit__(None, None, None)


def run_ours_sampled(args, rank, world, local, clk):
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from tmd_b200 import TensorMDModel, TensorMDSystem
    pot, syms, x, t, box, v, cfg = workload(args.config, seed=42 + rank)
    n = len(x)
    model = TensorMDModel(f"{pot} {' '.join(syms)}", device=local)
    sys_ = TensorMDSystem(model, n, 1.0)
    sys_.set_box(box)
    sys_.set_atoms(x, t, v)
    # setup, outside the timed region: pick the kernel forms for this shape
    tune_ms = sys_.autotune(reps=5)
    tune_dms = sys_.autotune(reps=5, family="descriptor")
    force_form = {"chosen": sys_.force_variant(), "ms_per_launch": tune_ms,
                  "descriptor_chosen": sys_.descriptor_variant(),
                  "descriptor_ms_per_launch": tune_dms}
    stream = torch.cuda.ExternalStream(sys_.stream(), device=dev)
    if world > 1:
        import torch.distributed as dist
        import datetime
        # ranks that wait for one another end with an error within minutes
        dist.init_process_group("nccl", device_id=dev, timeout=datetime.timedelta(seconds=300))
    dt = 0.001

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    # measured FP32 issue peak, the denominator of the FP32 rooflines
    fp32_peak = fp32_peak_tflops(sys_.lib, local)
    # warm-up
    sys_.nve_run(max(args.warmup, 3), dt)
    torch.cuda.synchronize()
    # timed region
    l0 = sys_.launches()
    r0 = sys_.rebuilds()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    sys_.nve_run(args.steps, dt)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    launches = sys_.launches() - l0
    rebuilds = sys_.rebuilds() - r0
    ms_max = max_over_ranks(ms, world, dev)
    value = replicas_value(n, args.steps, world, ms_max)

    # per-kernel device times of the same step sequence (a second, profiled pass)
    sys_.profile(True)
    sys_.profile_read(reset=True)
    nprof = max(10, min(args.steps, 50))
    rp0 = sys_.rebuilds()
    sys_.nve_run(nprof, dt)
    prof = sys_.profile_read(reset=True)
    sys_.profile(False)
    prof_rebuilds = sys_.rebuilds() - rp0

    # force-kernel roofline
    off, ent = sys_.neighbor_list(model.cutmax)
    npairs_rc = len(ent)
    nlist = len(sys_.neighbor_list(model.cutmax + 1.0)[1])
    B, K, D = model.nelt, model.num_filters, {1: 1, 2: 4, 3: 10, 4: 20}[model.mmax]
    flops, abytes = algorithmic(cfg, npairs_rc, nlist, B, K, D, model.n_desc,
                                sys_.force_variant())
    fcnt, fms = prof["force"]
    force_ms = fms / max(fcnt, 1)
    hbm_peak, peak_kind = measured_peaks()
    kname = {"filter_lane": "k_force", "pair_lane8": "k_force_pl<8>",
             "pair_lane16": "k_force_pl<16>", "pair_lane32": "k_force_pl<32>"}[sys_.force_variant()]
    traffic = ncu_traffic(args.config, kname)
    ach_gbs = abytes / (force_ms / 1000.0) / 1e9
    ach_tf = flops / (force_ms / 1000.0) / 1e12
    # the force kernel is bound by FP32 issue (its DRAM traffic is ~20% of
    # peak): the headline roofline is its algorithmic FLOP/s against the FP32
    # peak measured in this run; the HBM view of the same launch beside it
    roofline = {"kernel": kname, "bound": "fp32", "achieved": ach_tf,
                "peak": fp32_peak, "unit": "TFLOP/s", "frac": ach_tf / fp32_peak,
                "traffic": traffic,
                "peak_source": "measured in this run (tmd_fp32_peak: FFMA2 microkernel, "
                               "2 FLOP per FMA, best of 5)",
                "algorithmic_flops_per_launch": flops, "launch_ms": force_ms,
                "hbm": {"achieved_gbs": ach_gbs, "peak_gbs": hbm_peak,
                        "frac": ach_gbs / hbm_peak,
                        "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                        "bytes_per_launch": abytes,
                        "traffic_over_bytes": (traffic / abytes) if traffic else None}}
    kernel_ms = {k: (c, t / max(c, 1)) for k, (c, t) in prof.items()}
    # the other step kernels against their bounds (same profiled pass);
    # algorithmic work per launch: the per-atom operation counts of each step
    Minv = {1: 1, 4: 2, 10: 3, 20: 4}[D]
    sz = cfg["mlp"]
    mlp_macs = sum(a * b for a, b in zip(sz[:-1], sz[1:])) \
        + sum(a * b for a, b in zip(sz[:-2], sz[1:-1]))

    def kms(name):
        c, tt = prof[name]
        return tt / max(c, 1)

    def fp32_row(name, fl):
        ms_ = kms(name)
        tf = fl / (ms_ / 1000.0) / 1e12
        return {"ms": ms_, "bound": "fp32", "flops": fl, "achieved_tflops": tf,
                "frac": tf / fp32_peak}

    desc_flops = npairs_rc * (2.0 * K * D + 10.0 * K + D) + n * B * (2 * Minv + 1) * D * K
    # each pair force is read twice (as an atom's own and as its partner's)
    # but needs to leave HBM once
    gather_bytes = nlist * (16 + 4) + n * (24 + 4)
    g_ms = kms("gather")
    # the whole step against the survey's algorithmic bytes (x, type, list,
    # f, v, MLP staging) and the DRAM bytes the step's kernels move (sum of
    # the committed ncu per-launch traffic of the step kernels)
    steps_all = args.steps + nprof
    period = steps_all / max(rebuilds + prof_rebuilds, 1)
    sbytes = step_bytes_s8d(n, nlist, model.n_desc, period)
    step_traffic = 0
    for kn in ("k_descriptor_w", "k_mlp_fp32w", kname, "k_gather"):
        tr = ncu_traffic(args.config, kn)
        step_traffic = None if (tr is None or step_traffic is None) else step_traffic + tr
    step_roofline = {
        "algorithmic_bytes_per_step": sbytes,
        "algorithmic_bytes_per_atom": sbytes / n,
        "traffic_bytes_per_step": step_traffic,
        "traffic_over_algorithmic": (step_traffic / sbytes) if step_traffic else None,
        "rebuild_period_steps": period,
        "flops_per_step": None,  # filled below
        "note": "bytes as the survey defines them for a fused design; traffic = "
                "committed ncu DRAM bytes per launch of descriptor, MLP, force and gather",
    }
    kernel_roofline = {
        "descriptor": fp32_row("descriptor", desc_flops),
        "mlp": fp32_row("mlp", 2.0 * n * mlp_macs),
        "force": fp32_row("force", flops),
        "gather": {"ms": g_ms, "bound": "hbm", "bytes": gather_bytes,
                   "achieved_gbs": gather_bytes / (g_ms / 1000.0) / 1e9,
                   "frac": gather_bytes / (g_ms / 1000.0) / 1e9 / hbm_peak},
        "fp32_peak_tflops": fp32_peak,
        "work": "descriptor: per pair inside rc P 2KD + radial 10K + monomials D, per atom "
                "and block G (2M+1)DK; mlp: 2 x (forward + backward MACs) per atom; force: "
                "as roofline; gather: per list entry its pair force (16 B, read "
                "once; the partner read is the same array) and partner slot (4 B), per atom "
                "force (24 B) and row length",
    }

    step_roofline["flops_per_step"] = desc_flops + 2.0 * n * mlp_macs + flops
    step_roofline["fp32_frac_of_step"] = (step_roofline["flops_per_step"]
                                          / (ms_max / args.steps / 1000.0) / 1e12 / fp32_peak)

    # e2e through the reference-facing call pattern (host buffers)
    sys_.set_atoms(x, t, v)
    xh = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    vh = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    fh = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    xh[:] = x
    vh[:] = v
    from tmd_b200.synth import MVV2E
    from tmd_b200 import synth
    masses = np.array([synth.MASSES.get(s, 50.0) for s in syms])[t - 1][:, None]
    dtf = 0.5 * dt / MVV2E
    import ctypes
    from tmd_b200.lib import check
    lib = sys_.lib
    pd = ctypes.POINTER(ctypes.c_double)
    xp, fp = xh.ctypes.data_as(pd), fh.ctypes.data_as(pd)
    e = np.zeros(1)
    vir = np.zeros(6)
    # the caller's integrator (LAMMPS FixNVE is a C++ loop over the atoms):
    # in-place multithreaded CPU tensor ops on the same pinned host buffers
    xt, vt, ft = torch.from_numpy(xh), torch.from_numpy(vh), torch.from_numpy(fh)
    dtfm = torch.from_numpy(np.ascontiguousarray(dtf / masses))

    def e2e_step():
        # LAMMPS Verlet step with the pair on the device: initial integrate on
        # the host, positions H2D, pair compute, forces D2H, final integrate
        vt.addcmul_(ft, dtfm)
        xt.add_(vt, alpha=dt)
        check(lib.tmd_system_set_positions(sys_.h, xp))
        check(lib.tmd_compute(sys_.h, 1, 1, 1.0, e.ctypes.data_as(pd), vir.ctypes.data_as(pd),
                              fp, None, None))
        vt.addcmul_(ft, dtfm)

    check(lib.tmd_compute(sys_.h, 1, 1, 1.0, e.ctypes.data_as(pd), vir.ctypes.data_as(pd),
                          fp, None, None))
    for _ in range(3):
        e2e_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        e2e_step()
    t1 = time.perf_counter()
    e2e_val = replicas_value(n, args.e2e_steps, world,
                             1000.0 * max_over_ranks(t1 - t0, world, dev))

    # tensor-core MLP forms of the same workload (same steps, same timing)
    forms = {"fp32": {"value": value, "ms_per_step": ms_max / args.steps,
                      "mlp_ms": prof["mlp"][1] / max(prof["mlp"][0], 1)}}
    for prec in ([] if (args.no_bf16 or args.main_only) else ["tf32x3", "bf16x3", "bf16"]):
        try:
            mb = TensorMDModel(f"{pot} {' '.join(syms)} precision {prec}", device=local)
            sb = TensorMDSystem(mb, n, 1.0)
            sb.set_box(box)
            sb.set_atoms(x, t, v)
            fp = TensorMDSystem(model, n, 1.0)
            fp.set_box(box)
            fp.set_atoms(x, t, v)
            f32 = fp.compute(1, 1)
            fb = sb.compute(1, 1)
            ferr = float(np.sqrt(np.mean((fb["f"] - f32["f"]) ** 2)))
            eerr = abs(fb["energy"] - f32["energy"]) / n
            fp.close()
            sb.nve_run(max(args.warmup, 3), dt)
            torch.cuda.synchronize()
            sb_stream = torch.cuda.ExternalStream(sb.stream(), device=dev)
            b0 = torch.cuda.Event(enable_timing=True)
            b1 = torch.cuda.Event(enable_timing=True)
            barrier()
            torch.cuda.synchronize()
            b0.record(sb_stream)
            sb.nve_run(args.steps, dt)
            b1.record(sb_stream)
            torch.cuda.synchronize()
            bms = max_over_ranks(b0.elapsed_time(b1), world, dev)
            sb.profile(True)
            sb.profile_read(reset=True)
            sb.nve_run(nprof, dt)
            bprof = sb.profile_read(reset=True)
            forms[prec] = {"value": n * args.steps * world / (bms / 1000.0),
                           "ms_per_step": bms / args.steps,
                           "force_rms_err_vs_fp32_eV_per_A": ferr,
                           "energy_err_vs_fp32_eV_per_atom": eerr,
                           "mlp_ms": bprof["mlp"][1] / max(bprof["mlp"][0], 1)}
            sb.close()
            mb.close()
        except Exception as exc:  # report, do not hide
            forms[prec] = {"error": str(exc)}

    cells = None
    if args.cells_steps > 0 and not args.main_only:
        cells = run_cells(args, rank, world, local, dev, barrier)
    serving = None
    if args.serve_window > 0 and not args.main_only:
        serving = run_serving(args, rank, local)
        keys = ("solves_per_s", "p50_ms", "p99_ms", "atom_steps_per_s", "makespan_s",
                "by_kind", "fire_converged_frac")
        precs = [] if args.no_bf16 else ["bf16x3", "bf16"]
        if precs:
            # the same job stream (same seeds) with the MLP in the BF16 forms
            serving["forms"] = {}
            for prec in precs:
                try:
                    sf = run_serving(args, rank, local, precision=prec)
                    serving["forms"][prec] = {k: sf[k] for k in keys}
                except Exception as exc:  # report, do not hide
                    serving["forms"][prec] = {"error": str(exc)}
        # latency against throughput: lower arrival rates, every form
        rates = [float(r) for r in args.serve_sweep.split(",") if r.strip()]
        serving["rate_sweep"] = {}
        for rate in rates:
            row = {}
            for prec in ["fp32"] + precs:
                try:
                    sf = run_serving(args, rank, local, precision=prec, rate=rate)
                    row[prec] = {k: sf[k] for k in keys}
                except Exception as exc:  # report, do not hide
                    row[prec] = {"error": str(exc)}
            serving["rate_sweep"][f"{rate:g}"] = row
        try:
            serving["fire_trained"] = run_fire_trained(rank, local)
        except Exception as exc:  # report, do not hide
            serving["fire_trained"] = {"error": str(exc)}
    decomp = None
    if args.decomp_steps > 0:
        try:
            decomp = run_decomp(args, rank, world, local, dev, barrier)
        except Exception as exc:  # report, do not hide
            decomp = {"error": str(exc)}
    w23k = None if args.main_only else run_w23k(args, rank, world, local, dev, barrier)
    drift = None
    if args.drift_steps > 0:
        try:
            drift = run_w_drift(args, rank, local)
        except Exception as exc:  # report, do not hide
            drift = {"error": str(exc)}
    alloy = None
    if args.precision_steps > 0 and not args.main_only:
        try:
            alloy = run_alloy(args, rank, world, local, dev, barrier)
        except Exception as exc:  # report, do not hide
            alloy = {"error": str(exc)}

    cpu = None
    if rank == 0 and world == 1 and not (args.no_cpu_baseline or args.main_only):
        cpu = cpu_baseline(args.config, samples=2)

    clocks = clk.summary()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32", "data": "synthetic (seeded lattice, random-init potential weights)",
            "config": dict(cfg, parallelism=f"replicas x{world}", precision="plain fp32",
                           l2="working set > 126 MB L2 (neighbor rows, pair forces, P)"),
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": 24 * n,
                    "d2h_bytes_per_step": 24 * n + 7 * 8, "steps": args.e2e_steps,
                    "timing": "host wall clock, includes the host velocity Verlet "
                              "(multithreaded in-place CPU tensor ops)"},
            "gpu_launches": launches,
            "neighbor_rebuilds_in_timed_region": rebuilds,
            "clocks": clocks,
            "roofline": roofline,
            "step_roofline": step_roofline,
            "kernel_roofline": kernel_roofline,
            "kernel_ms": kernel_ms,
            "force_form": force_form,
            "forms": forms,
            "cells4096": cells,
            "alloy432k": alloy,
            "serving": serving,
            "reference_workload_w23k": w23k,
            "w432k_nve_drift": drift,
            "decomposition": decomp,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_alloy(args, rank, world, local, dev, barrier):
    """Precision config: 4-element random FCC alloy a = 3.6 A, 60x60x30 cells =
    432,000 atoms, 32 Gaussians rc 6.5 A, MLP 512-128-128-128-1 softplus.
    Each MLP form (plain FP32, 3xTF32, split BF16, BF16) runs the same NVE steps,
    timed with CUDA events on its system stream after 3 warm-up steps; MLP
    time per step from a profiled pass; force and energy error of the BF16
    forms against the FP32 form on the starting positions."""
    import torch
    from tmd_b200 import TensorMDModel, TensorMDSystem, synth
    pot, syms, x, t, box, v, cfg = workload("alloy432k", seed=42)
    n, dt = len(x), 0.001
    out = {"natoms": n, "steps": args.precision_steps, "config": cfg, "forms": {}}
    ref = None
    for prec in ("fp32", "tf32x3", "bf16x3", "bf16"):
        suffix = "" if prec == "fp32" else f" precision {prec}"
        m = TensorMDModel(f"{pot} {' '.join(syms)}{suffix}", device=local)
        s_ = TensorMDSystem(m, n, 1.0)
        s_.set_box(box)
        s_.set_atoms(x, t, v)
        s_.autotune(reps=3)
        s_.autotune(reps=3, family="descriptor")
        r = s_.compute(1, 1)
        row = {"force_form": s_.force_variant(), "descriptor_form": s_.descriptor_variant()}
        if ref is None:
            ref = r
        else:
            row["force_rms_err_vs_fp32_eV_per_A"] = float(np.sqrt(np.mean((r["f"] - ref["f"]) ** 2)))
            row["energy_err_vs_fp32_eV_per_atom"] = abs(r["energy"] - ref["energy"]) / n
        s_.nve_run(3, dt)
        stream = torch.cuda.ExternalStream(s_.stream(), device=dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        s_.nve_run(args.precision_steps, dt)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
        s_.profile(True)
        s_.profile_read(reset=True)
        s_.nve_run(5, dt)
        prof = s_.profile_read(reset=True)
        row.update({"value": n * args.precision_steps * world / (ms / 1000.0),
                    "ms_per_step": ms / args.precision_steps,
                    "kernel_ms": {k: c_t[1] / max(c_t[0], 1) for k, c_t in prof.items()
                                  if c_t[0] > 0}})
        out["forms"][prec] = row
        s_.close()
        m.close()
    f32 = out["forms"]["fp32"]["value"]
    for prec in ("tf32x3", "bf16x3", "bf16"):
        out["forms"][prec]["speedup_vs_fp32"] = out["forms"][prec]["value"] / f32
    return out


def run_cells(args, rank, world, local, dev, barrier):
    """Multi-cell batch: 4,096 cells x 256 atoms (half FCC, half BCC), two
    elements, per-cell temperatures 300-1200 K, NVE through tmd_batch_nve_run
    (every step one CUDA graph launch), timed with CUDA events on the batch
    stream, max over ranks."""
    import torch
    from tmd_b200 import TensorMDBatch, TensorMDModel, synth
    c = synth.config("cells4096")
    pot = f"/tmp/tmd_bench_cells_{rank}.npz"
    syms = synth.gaussian_potential(pot, seed=2024, **c["pot"])
    data = synth.batch_cells(c["ncells"], c["natoms"], nelt=c["nelt"], sigma=c["sigma"],
                             t_range=c["t_range"], seed=99 + rank)
    model = TensorMDModel(f"{pot} {' '.join(syms)}", device=local)
    b = TensorMDBatch(model, data["natoms"], 1.0)
    b.set_cells(data["boxes"])
    b.set_atoms(data["x"], data["types"], data["v"])
    tune_ms = b.system().autotune(reps=3)
    tune_dms = b.system().autotune(reps=3, family="descriptor")
    n = b.n
    dt = 0.001
    stream = torch.cuda.ExternalStream(b.system().stream(), device=dev)
    b.nve_run(max(args.warmup, 3), dt)
    torch.cuda.synchronize()
    sv = b.system()
    l0 = sv.launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    th = b.nve_run(args.cells_steps, dt, thermo_every=args.cells_steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    launches = sv.launches() - l0
    sv.profile(True)
    sv.profile_read(reset=True)
    b.nve_run(20, dt)
    prof = sv.profile_read(reset=True)
    sv.profile(False)
    etot = th.sum(-1)  # rows x cells
    drift = float(np.abs(etot[-1] - etot[0]).max() / c["natoms"])
    # BF16 MLP forms on the same cells: a shorter timed NVE run each, and the
    # force error of one evaluation against the FP32 form at the starting state
    forms = {}
    if not args.no_bf16:
        b.set_atoms(data["x"], data["types"], data["v"])
        f32 = b.compute()["f"]
        nsteps_f = max(50, args.cells_steps // 5)
        for prec in ("bf16x3", "bf16"):
            try:
                mb = TensorMDModel(f"{pot} {' '.join(syms)} precision {prec}", device=local)
                bb = TensorMDBatch(mb, data["natoms"], 1.0)
                bb.set_cells(data["boxes"])
                bb.set_atoms(data["x"], data["types"], data["v"])
                fe = bb.compute()["f"]
                err = float(np.sqrt(((fe - f32) ** 2).mean()))
                st_b = torch.cuda.ExternalStream(bb.system().stream(), device=dev)
                bb.nve_run(max(args.warmup, 3), dt)
                torch.cuda.synchronize()
                barrier()
                q0 = torch.cuda.Event(enable_timing=True)
                q1 = torch.cuda.Event(enable_timing=True)
                q0.record(st_b)
                bb.nve_run(nsteps_f, dt)
                q1.record(st_b)
                torch.cuda.synchronize()
                barrier()
                msb = max_over_ranks(q0.elapsed_time(q1), world, dev)
                forms[prec] = {"value": n * nsteps_f * world / (msb / 1000.0),
                               "ms_per_step": msb / nsteps_f, "steps": nsteps_f,
                               "force_rms_err_vs_fp32_eV_per_A": err}
                bb.close()
                mb.close()
            except Exception as exc:  # report, do not hide
                forms[prec] = {"error": str(exc)}
    out = {"value": n * args.cells_steps * world / (ms / 1000.0), "unit": UNIT,
           "ms_per_step": ms / args.cells_steps, "steps": args.cells_steps,
           "natoms": n, "ncells": c["ncells"], "gpu_launches": launches,
           "max_cell_energy_drift_eV_per_atom": drift,
           "forms": forms,
           "force_form": {"chosen": sv.force_variant(), "ms_per_launch": tune_ms,
                          "descriptor_chosen": sv.descriptor_variant(),
                          "descriptor_ms_per_launch": tune_dms},
           "kernel_ms": {k: (cnt, t / max(cnt, 1)) for k, (cnt, t) in prof.items()},
           "config": {k: v for k, v in c.items() if k != "pot"} | {"potential": c["pot"]}}
    b.close()
    model.close()
    return out


def run_decomp(args, rank, world, local, dev, barrier):
    """One cell over all ranks: the headline workload cut into one slab per
    rank along x (tmd_b200.decomp.SlabDecomposition over each rank's
    ghost-aware device system; ghosts by all-gather, ghost forces home by
    all-reduce, NCCL between GPUs), args.decomp_steps NVE steps with the
    integrator on the host.  Strong scaling: the cell is fixed, the ranks
    share it.  Host wall clock, max over ranks."""
    from tmd_b200 import TensorMDModel, TensorMDSystem
    from tmd_b200.decomp import SlabDecomposition
    pot, syms, x, t, box, v, cfg = workload(args.config, seed=42)
    model = TensorMDModel(f"{pot} {' '.join(syms)}", device=local)
    n = len(x)
    sysr = TensorMDSystem(model, int(3 * n / world) + 4096, 1.0)
    dec = SlabDecomposition(box, model.cutmax + 1.0, 1.0, sysr, rank=rank, world=world,
                            device=dev)
    dec.set_atoms(x, t, v)
    masses = np.asarray(model.type_mass, dtype=np.float64)
    dec.nve_run(2, 0.001, masses)
    barrier()
    t0 = time.perf_counter()
    dec.nve_run(args.decomp_steps, 0.001, masses)
    wall = time.perf_counter() - t0
    wall = max_over_ranks(wall, world, dev)
    out = {"value": n * args.decomp_steps / wall, "unit": UNIT, "scaling": "strong",
           "natoms": n, "ranks": world, "steps": args.decomp_steps,
           "ms_per_step": 1000.0 * wall / args.decomp_steps,
           "local_atoms_rank0": len(dec.x), "ghosts_rank0": dec.nghost,
           "timing": "host wall clock (host integrator and exchange), max over ranks"}
    sysr.close()
    model.close()
    return out


def run_w23k(args, rank, world, local, dev, barrier):
    """The reference's own speed benchmark, run the same way: W_k32_snapshot.npz
    (shipped trained potential, FNN radial net + rational table, interp
    0.001), BCC a = 3.189 A, 24x24x20 cells = 23,040 atoms, velocities 300 K,
    fix nvt temp 300 300 0.1, 100 steps, skin 1 A
    (examples/tensormd/W/tensormd/speedup/in.lammps).  Published on an A100:
    3.221 M atom-steps/s (log_0114.lammps, the reference's optimized build)."""
    import torch
    from tmd_b200 import TensorMDModel, TensorMDSystem, synth
    model = TensorMDModel(f"{ROOT}/tests/golden/W_k32_snapshot.npz W interp 0.001", device=local)
    x, box = synth.lattice("bcc", 3.189, 24, 24, 20)
    n = len(x)
    t = np.ones(n, dtype=np.int32)
    v = synth.maxwell(np.full(n, model.type_mass[1]), 300.0, np.random.default_rng(984523 + rank))
    s = TensorMDSystem(model, n, 1.0)
    s.set_box(box)
    s.set_atoms(x, t, v)
    tune_ms = s.autotune(reps=5)
    tune_dms = s.autotune(reps=5, family="descriptor")
    stream = torch.cuda.ExternalStream(s.stream(), device=dev)
    s.nvt_run(max(args.warmup, 3), 0.001, 300.0, 300.0, 0.1)
    s.set_atoms(x, t, v)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record(stream)
    s.nvt_run(100, 0.001, 300.0, 300.0, 0.1)
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    value = n * 100 * world / (ms / 1000.0)
    form = {"chosen": s.force_variant(), "ms_per_launch": tune_ms,
            "descriptor_chosen": s.descriptor_variant(), "descriptor_ms_per_launch": tune_dms}
    s.close()
    model.close()
    return {"value": value, "unit": UNIT, "ms_per_step": ms / 100, "natoms": n, "steps": 100,
            "host_wall_s": wall, "force_form": form, "published_a100": 3.221e6, "ratio_vs_published_a100": value / 3.221e6,
            "config": "W_k32_snapshot.npz interp 0.001, bcc 3.189 24x24x20, 300 K, "
                      "fix nvt temp 300 300 0.1, skin 1.0, dt 1 fs"}


def run_w_drift(args, rank, local):
    """Energy conservation on the reference's own trained potential:
    W_k32_snapshot.npz (interp 0.001), BCC a = 3.189 A, 60^3 cells = 432,000
    atoms, velocities 300 K (seeded), 1,000 steps of fix nvt temp 300 300 0.1
    to equilibrate, then args.drift_steps NVE steps at dt = 1 fs with the total
    energy sampled every 100 steps.  The synthetic random-weight potentials are
    not stable lattices (their cells collapse within 10^4 steps), so their drift
    would measure the collapse, not the integrator."""
    from tmd_b200 import TensorMDModel, TensorMDSystem, synth
    model = TensorMDModel(f"{ROOT}/tests/golden/W_k32_snapshot.npz W interp 0.001", device=local)
    x, box = synth.lattice("bcc", 3.189, 60, 60, 60)
    n = len(x)
    t = np.ones(n, dtype=np.int32)
    v = synth.maxwell(np.full(n, model.type_mass[1]), 300.0, np.random.default_rng(20250 + rank))
    s = TensorMDSystem(model, n, 1.0)
    s.set_box(box)
    s.set_atoms(x, t, v)
    s.autotune(reps=3)
    s.autotune(reps=3, family="descriptor")
    t0 = time.perf_counter()
    s.nvt_run(1000, 0.001, 300.0, 300.0, 0.1)
    every = 100
    th = s.nve_run(args.drift_steps, 0.001, thermo_every=every)
    wall = time.perf_counter() - t0
    etot = (th[:, 0] + th[:, 1]) / n
    steps = np.minimum(np.arange(len(etot)) * every, args.drift_steps)
    slope = float(np.polyfit(steps * 1e-6, etot, 1)[0]) if len(etot) > 1 else 0.0  # eV/atom/ns
    temp = 2.0 * th[:, 1] / ((3 * n - 3) * synth.BOLTZ)
    s.close()
    model.close()
    return {"natoms": n, "nve_steps": args.drift_steps, "dt_fs": 1.0, "sample_every": every,
            "max_abs_dE_eV_per_atom": float(np.abs(etot - etot[0]).max()),
            "final_dE_eV_per_atom": float(etot[-1] - etot[0]),
            "slope_eV_per_atom_per_ns": slope,
            "T_first_K": float(temp[0]), "T_last_K": float(temp[-1]),
            "T_mean_K": float(temp.mean()),
            "wall_s": wall, "atom_steps_per_s_wall": n * (1000 + args.drift_steps) / wall,
            "config": "W_k32_snapshot.npz interp 0.001, bcc 3.189 60x60x60, 300 K, "
                      "fix nvt 300 300 0.1 for 1,000 steps, then NVE, skin 1.0, dt 1 fs"}


def run_fire_trained(rank, local, njobs=64):
    """FIRE jobs on a trained potential, whose lattices are real minima (the
    random-weight serving potential has none: its cells collapse under any
    minimiser, so its FIRE jobs run to the iteration cap): the reference's
    MoNi_m3 potential, Mo8Ni8 cells replicated 1-3 times per axis (16-432
    atoms), positions displaced by sigma 0.1 A, min_style fire to max |F_i|
    < 0.01 eV/A, at most 1000 iterations, all submitted at once."""
    from tmd_b200 import TensorMDModel, TensorMDServer
    from tmd_b200.synth import frac_wrap, read_data
    GOLDEN = ROOT / "tests" / "golden"
    x0, t0, box0 = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
    x0 = frac_wrap(x0, box0)
    rng = np.random.default_rng(515 + rank)
    model = TensorMDModel(f"{GOLDEN}/MoNi_m3.npz Mo Ni interp 0.0001", device=local)
    srv = TensorMDServer(model, max_atoms=200000, max_cells=256, steps_per_tick=8)
    a = np.array(box0[3:6])
    tilt = np.array(box0[6:9])
    jobs = []
    for _ in range(njobs):
        r = rng.integers(1, 4, size=3)
        sh = np.stack(np.meshgrid(*(np.arange(k) for k in r), indexing="ij"), -1).reshape(-1, 3)
        off = np.stack([sh[:, 0] * a[0] + sh[:, 1] * tilt[0] + sh[:, 2] * tilt[1],
                        sh[:, 1] * a[1] + sh[:, 2] * tilt[2], sh[:, 2] * a[2]], -1)
        x = (x0[None, :, :] + off[:, None, :]).reshape(-1, 3)
        t = np.tile(t0, len(sh))
        box = np.concatenate([box0[:3], a * r, [tilt[0] * r[1], tilt[1] * r[2],
                                                tilt[2] * r[2]]])
        x = x + rng.normal(0.0, 0.1, size=x.shape)
        jobs.append((x, t, box))
    t_start = time.perf_counter()
    tickets = [srv.submit(2, x, t, box, nsteps=1000, dt=0.001, fmax=0.01) for x, t, box in jobs]
    done = [srv.wait(tk, timeout=600) for tk in tickets]
    t_end = time.perf_counter()
    srv.close()
    model.close()
    it = np.array([d["steps"] for d in done])
    fmax = np.array([np.linalg.norm(d["f"], axis=1).max() for d in done])
    lat = np.array([d["latency"] for d in done]) * 1000.0
    return {"jobs": njobs, "potential": "MoNi_m3.npz interp 0.0001 (trained, shipped)",
            "natoms_range": [int(min(len(j[0]) for j in jobs)), int(max(len(j[0]) for j in jobs))],
            "converged_frac": float(np.mean(fmax < 0.01)), "iteration_cap": 1000,
            "iterations_p50": float(np.percentile(it, 50)),
            "iterations_max": int(it.max()), "makespan_s": t_end - t_start,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))}


def run_serving(args, rank, local, precision="fp32", rate=None):
    """Serving: Poisson arrivals (rate jobs/s, default args.serve_rate, over
    args.serve_window s) of jobs with N log-uniform in [32, 4096] atoms, FCC /
    BCC lattices or random packings (0.085 A^-3, dmin 2 A), 1-4 elements; 60%
    single-point, 25% 200-step NVE, 15% FIRE (min_style fire) to max |F_i| <
    0.01 eV/A (at most 1000 iterations).  Jobs go through tmd_server_submit /
    tmd_server_wait; latency is submit -> completion on the host clock."""
    import threading
    from tmd_b200 import TensorMDModel, TensorMDServer, synth
    rate = args.serve_rate if rate is None else rate
    rng = np.random.default_rng(77 + rank)
    pot = f"/tmp/tmd_bench_serve_{rank}.npz"
    syms = synth.gaussian_potential(pot, seed=4242, nelt=4, num_filters=16, rc=6.0,
                                    max_moment=3, hidden=(64, 64), actfn=2)
    prec = "" if precision == "fp32" else f" precision {precision}"
    model = TensorMDModel(f"{pot} {' '.join(syms)}{prec}", device=local)
    sizes = np.unique(np.round(np.geomspace(32, 4096, 12)).astype(int))
    packings = {int(n): synth.random_packing(int(n), rng) for n in sizes}
    t_arr = np.cumsum(rng.exponential(1.0 / rate, size=int(rate * args.serve_window * 1.5) + 8))
    t_arr = t_arr[t_arr < args.serve_window]
    kinds = rng.choice(3, size=len(t_arr), p=[0.60, 0.25, 0.15])
    jobs = [synth.serving_job(rng, kind=int(k), packings=packings) for k in kinds]
    srv = TensorMDServer(model, max_atoms=2_000_000, max_cells=8192, steps_per_tick=8)
    # warm-up: one job of each kind
    for k in range(3):
        x, t, box, v = jobs[k]
        srv.wait(srv.submit(k, x, t, box, v=v, nsteps=20, dt=0.001, fmax=0.01))
    st0 = srv.stats()
    tickets = [None] * len(jobs)
    done = [None] * len(jobs)

    def submitter():
        t0 = time.perf_counter()
        for i, (ta, k, (x, t, box, v)) in enumerate(zip(t_arr, kinds, jobs)):
            dly = ta - (time.perf_counter() - t0)
            if dly > 0:
                time.sleep(dly)
            tickets[i] = srv.submit(int(k), x, t, box, v=v,
                                    nsteps=(200 if k == 1 else 1000), dt=0.001, fmax=0.01)

    th = threading.Thread(target=submitter)
    t_start = time.perf_counter()
    th.start()
    for i in range(len(jobs)):
        while tickets[i] is None:
            time.sleep(0.0005)
        done[i] = srv.wait(tickets[i])
    t_end = time.perf_counter()
    th.join()
    st1 = srv.stats()
    phases = srv.timing()
    srv.close()
    model.close()
    lat = np.array([d["latency"] for d in done]) * 1000.0
    natoms = np.array([len(j[0]) for j in jobs])
    out = {"precision": precision, "jobs": len(jobs), "arrival_rate_per_s": rate,
           "window_s": args.serve_window, "makespan_s": t_end - t_start,
           "solves_per_s": len(jobs) / (t_end - t_start),
           "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
           "atom_steps_per_s": (st1["atom_steps"] - st0["atom_steps"])
           / max(st1["busy_s"] - st0["busy_s"], 1e-9),
           "mean_atoms": float(natoms.mean()),
           "worker_seconds_by_phase": phases,
           "fire_converged_frac": float(np.mean([d["steps"] < 1000 for d, k in
                                                 zip(done, kinds) if k == 2] or [1.0])),
           "fire_iteration_cap": 1000,
           "by_kind": {}}
    for k, name in enumerate(("single_point", "nve200", "fire")):
        sel = kinds == k
        if sel.any():
            out["by_kind"][name] = {"jobs": int(sel.sum()),
                                    "p50_ms": float(np.percentile(lat[sel], 50)),
                                    "p99_ms": float(np.percentile(lat[sel], 99))}
    return out


def cpu_baseline(cfg_name, samples=2):
    """The FP64 oracle (port of the reference math, OpenMP) on a bounded
    sample: `samples` full MD steps (neighbor build + force) of the workload."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from pack import Oracle, load_npz
    pot, syms, x, t, box, v, cfg = workload(cfg_name, seed=42)
    o = Oracle(load_npz(pot))
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    o.nve(x[:8], v[:8], (t - 1)[:8], box, [1, 1, 1], 0.001, 1)  # load / warm
    t0 = time.perf_counter()
    o.nve(x, v, t - 1, box, [1, 1, 1], 0.001, samples - 1, skin=1.0)
    t1 = time.perf_counter()
    val = len(x) * samples / (t1 - t0)
    out = {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
           "sample": f"{samples} full MD steps (neighbor rebuild + FP64 force) of the "
                     f"{cfg['natoms']}-atom workload, oracle/tmd_oracle.c, OpenMP "
                     f"{cores} threads"}
    # one thread, on the 4,000-atom FCC config (2 MD steps: about 2 s)
    try:
        import ctypes
        gomp = ctypes.CDLL("libgomp.so.1")  # the OpenMP runtime the oracle runs on
        pot1, syms1, x1, t1_, box1, v1, cfg1 = workload("fcc4k", seed=42)
        o1 = Oracle(load_npz(pot1))
        gomp.omp_set_num_threads(1)
        o1.nve(x1[:8], v1[:8], (t1_ - 1)[:8], box1, [1, 1, 1], 0.001, 1)
        s0 = time.perf_counter()
        o1.nve(x1, v1, t1_ - 1, box1, [1, 1, 1], 0.001, 1, skin=1.0)
        s1 = time.perf_counter()
        gomp.omp_set_num_threads(cores)
        out["single_thread"] = {"value": len(x1) * 2 / (s1 - s0), "unit": UNIT, "cores": 1,
                                "sample": "2 full MD steps of the 4,000-atom FCC config "
                                          "(fcc4k), 1 OpenMP thread"}
    except OSError as exc:  # no libgomp under that name: report, do not hide
        out["single_thread"] = {"error": str(exc)}
    return out


def run_reference(args, rank, world):
    """The reference arm: the reference has no CPU pair path and its GPU path
    cannot evaluate this potential (analytic radial basis, tanh MLP), so the
    CPU restatement of its math (oracle, FP64, OpenMP) is timed instead."""
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    sys.path.insert(0, str(ROOT / "oracle"))
    from pack import Oracle, load_npz
    pot, syms, x, t, box, v, cfg = workload(args.config, seed=42)
    o = Oracle(load_npz(pot))
    per = 1
    for _ in range(max(1, min(args.warmup, 1))):
        o.nve(x, v, t - 1, box, [1, 1, 1], 0.001, 0, skin=1.0)
    steps = max(1, min(args.steps, 5))
    t0 = time.perf_counter()
    o.nve(x, v, t - 1, box, [1, 1, 1], 0.001, steps - 1, skin=1.0)
    t1 = time.perf_counter()
    val = len(x) * steps / (t1 - t0)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT,
            "n_gpus": world, "steps": steps, "warmup": 1, "ms_per_step": (t1 - t0) * 1000 / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
            "data": "synthetic", "config": dict(cfg, parallelism="cpu"),
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{steps} MD steps of the {cfg['natoms']}-atom workload "
                                       "(FP64 oracle restatement, OpenMP)"},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def profile_step(args):
    """A short, fixed launch sequence for ncu captures: the headline workload,
    args.profile_step force evaluations (each: neighbor check, descriptor,
    invariants, MLP, force, gather)."""
    from tmd_b200 import TensorMDModel, TensorMDSystem
    pot, syms, x, t, box, v, cfg = workload(args.config, seed=42)
    prec = "" if args.profile_precision == "fp32" else f" precision {args.profile_precision}"
    model = TensorMDModel(f"{pot} {' '.join(syms)}{prec}")
    s = TensorMDSystem(model, len(x), 1.0)
    s.set_box(box)
    s.set_atoms(x, t, v)
    if args.profile_desc:
        s.set_descriptor_variant(args.profile_desc)
    for _ in range(args.profile_step):
        s.compute(1, 1, 1.0)
    print(json.dumps({"profile_step": args.profile_step, "config": args.config,
                      "precision": args.profile_precision,
                      "force_form": s.force_variant(),
                      "descriptor_form": s.descriptor_variant()}), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.profile_step > 0:
        profile_step(args)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
