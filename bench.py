#!/usr/bin/env python
"""Throughput of the D3Q27 thermal LBM time step on B200 (MLUPS and HBM GB/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload inflow|chan|mix|react|tgv] [--N n] [--precision fp64|fp32]

One "step" is one full lattice time step of the workload (collide, stream, boundary,
moments over every fluid cell).  Default workload: config 2 -- the non-reacting
9-species H2/O2/N2 mixing layer, 128^3 interior cells, FP64, characteristic (NSCBC)
inflow and outflow in x, periodic y and z, a seeded sinusoidal interface (Y_H2 0 -> 0.03,
T 300 -> 1000 K, p = 1 atm), dx = 20 um, dt = 1 ns.  The state (about 5 GB in FP64) is far
larger than L2, so no L2 flush is needed between steps.  --workload tgv is config 1 (the
single-component Taylor-Green vortex, 64^3, FP64, Ma 0.1, Re 400); chan is config 3's
reacting channel shape (NSCBC outlets, TMS walls); mix/react are periodic boxes.

* value: MLUPS of K steps with the state resident in HBM, device-timed with CUDA events
  on the library's stream; max over ranks.
* e2e: the same steps through the reference-facing calls of the C ABI: AoS upload and
  Init from host memory, per step the five phase calls and a device->host read of the
  step's result (multicomponent: the conserved totals of lbmgpu_sums; config 1: the
  whole AoS state and the status word every 10 steps, the output cadence of the
  reference's Taylor-Green setup, setup.cpp:146), host wall clock.
* roofline: the dominant kernel's algorithmic bytes per launch / its mean launch time.
* cpu_baseline: the reference's own solver (oracle/_ref; multicomponent on the
  Cantera-API shim) on the host cores, a bounded sample (a slab of the workload).

Under torchrun (N > 1) every rank runs an independent replica of the workload on its own
GPU (the path is not domain-decomposed yet): weak scaling, value = all ranks' cells.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "lattice-boltzmann-method_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "MLUPS & HBM GB/s, D3Q27 reacting, 1 B200; surrogate vs plain chem at ≤1% err"
# algorithmic bytes per cell and launch (one read + one write of every population, plus
# the moment record the stream kernel must store)
BYTES_COLLIDE_FP64 = 2 * 54 * 8          # 864
BYTES_STREAM_FP64 = 54 * 8 + 6 * 8       # 480
BYTES_STEP_FP64 = 2 * 54 * 8             # 864: one read + one write of the populations
OUTPUT_EVERY = 10
# config 4's case: rms velocity (lattice units), hot-side temperature (K), dx (m), dx/dt (m/s)
TURB_DEFAULTS = {"urms": 0.02, "t_hot": 1500.0, "dx": 2e-6, "dxdt": 4000.0}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="default 1000 (tgv) or 200 (multicomponent)")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--N", type=int, default=None, help="interior cells per axis")
    ap.add_argument("--workload", choices=["turb", "tgv", "mix", "react", "inflow", "chan", "flame"], default="turb",
                    help="tgv: config 1 (single component, FP64 Taylor-Green vortex, 64^3); "
                         "mix: 9-species H2/air mixing layer, periodic (config 2 without its NSCBC "
                         "faces, 128^3); react: the same with the reference's explicit chemistry and a "
                         "1800 K slab; inflow: config 2's shape, the mixing layer between a characteristic "
                         "inflow and outflow (N^3); chan: config 3's case, a reacting H2-air channel with "
                         "NSCBC outflow ends and TMS walls, at 2N x N/2 x N/2; flame: config 3 itself, the "
                         "same channel at 4N x N/16 x N/16 (512 x 8 x 8 at the default N); turb (default): "
                         "config 4, the decaying turbulent reacting H2/air layer, N^3 (256), FP32 populations, "
                         "ROS2 stiff chemistry")
    ap.add_argument("--urms", type=float, default=TURB_DEFAULTS["urms"], help="turb: rms velocity, lattice units")
    ap.add_argument("--t-hot", type=float, default=TURB_DEFAULTS["t_hot"], help="turb: hot-side temperature, K")
    ap.add_argument("--dx", type=float, default=TURB_DEFAULTS["dx"], help="turb: lattice spacing, m")
    ap.add_argument("--dxdt", type=float, default=TURB_DEFAULTS["dxdt"], help="turb: dx / dt, m/s")
    ap.add_argument("--cpu-child", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-surrogate", action="store_true", help="turb: skip the surrogate-vs-plain study")
    ap.add_argument("--sur-shape", default="384x96x96",
                    help="turb: the surrogate study's channel (config 5's case; 384x192x192 is config 5 itself)")
    ap.add_argument("--slab-loopback", action="store_true",
                    help="turb on one GPU: run the slab-decomposition path with the rank as its own neighbour "
                         "(halo exchange by device copies) -- the multi-GPU code path without NCCL")
    ap.add_argument("--chem", choices=["ref", "rosenbrock", "surrogate"], default=None,
                    help="reacting workloads: the reference's explicit scheme, the ROS2 stiff integrator, or "
                         "the MLP surrogate trained online from ROS2 (teacher steps, training, then timed "
                         "surrogate steps with a 1 %% audit; plain ROS2 timed on the same lattice beside it)")
    ap.add_argument("--teach", type=int, default=200, help="surrogate: ROS2 teacher steps that collect ~2M samples")
    ap.add_argument("--epochs", type=int, default=16, help="surrogate: training epochs over the samples")
    ap.add_argument("--compare", type=int, default=100,
                    help="surrogate: steps run twice from the same state, with the surrogate and with plain ROS2, "
                         "to compare peak temperature and integrated heat release")
    ap.add_argument("--augment", type=float, default=0.5,
                    help="surrogate: perturbed, integrator-labelled rows added per collected row")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default=None,
                    help="multicomponent population storage (fp32: shifted FP32 populations, FP64 records)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------------------
class Dist:
    """One process per GPU (RANK / LOCAL_RANK / WORLD_SIZE from the launcher): NCCL for the
    benchmark's barrier and max over ranks; gloo on the host for the CPU tests."""

    def __init__(self, backend="nccl"):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                        device_id=torch.device("cuda", self.local))
            else:
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
            self.pg = dist

    def _device(self):
        return "cuda" if self.backend == "nccl" else "cpu"

    def barrier(self):
        if self.pg:
            import torch
            t = torch.zeros(1, device=self._device())
            self.pg.all_reduce(t)
            if self.backend == "nccl":
                torch.cuda.synchronize()

    def max(self, x):
        if not self.pg:
            return x
        import torch
        t = torch.tensor([float(x)], device=self._device(), dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def whole_job_mlups(world, cells, steps, seconds):
    """Replicas (the path is not domain-decomposed): every rank updates its own lattice of
    `cells` for `steps`; the job's rate is all ranks' cell updates over the slowest rank's
    time (`seconds`, already the max over ranks)."""
    return world * cells * steps / seconds / 1e6


# ---------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------------------
def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel, cells, case):
    """DRAM bytes of one launch of `kernel` over `cells` fluid cells in the workload family
    `case`, scaled from the committed ncu capture (profiles/ncu_traffic.txt: bytes of one
    captured launch, the cells it processed and the case captured; the traffic of these
    kernels grows in proportion to the cells), or None."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        for line in open(p):
            parts = line.split()
            if (len(parts) >= 7 and parts[0] == "traffic" and parts[1] == kernel and parts[3] == "cells"
                    and parts[5] == "case" and parts[6] == case):
                return float(parts[2]) / float(parts[4]) * cells
    except OSError:
        pass
    return None


def workload(N):
    import workloads
    cells, prm = workloads.tgv_sc(N)
    return cells, prm


def fluid_cells(cells):
    return int((cells["type"] == 0).sum())


class stdout_to_stderr:
    """Routes the process's file-descriptor-level stdout to stderr (the reference's own
    solver prints progress with std::cout; the bench's stdout carries one JSON line)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def cpu_reference_run(cells, prm, steps, warmup, threads):
    """Times the reference's own solver (oracle/_ref) -- or, where it was not built, the C
    oracle port -- for `steps` steps after `warmup`; returns (seconds, kind)."""
    from oracle import refsc, sc
    N3 = [s - 2 for s in cells.shape]
    if refsc.available():
        refsc.set_threads(threads)
        ref = refsc.RefSC(*N3, prm["nu"], prm["R"], prm["gamma"], prm["prtl"], cells.dtype)
        ref.cells[...] = cells
        ref.init()
        if warmup:
            ref.loop(warmup)
        t0 = time.perf_counter()
        ref.loop(steps)
        dt = time.perf_counter() - t0
        ref.close()
        return dt, "reference"
    sc.set_threads(threads)
    a = cells.copy()
    o = sc.OracleSC(a, prm["nu"], prm["R"], prm["gamma"], prm["prtl"])
    o.init()
    if warmup:
        o.loop(warmup)
    t0 = time.perf_counter()
    o.loop(steps)
    return time.perf_counter() - t0, "port"


def cpu_baseline(cells, prm, target_s=10.0):
    threads = os.cpu_count() or 1
    t1, kind = cpu_reference_run(cells, prm, 1, 1, threads)
    n = max(2, min(200, int(target_s / max(t1, 1e-3))))
    dt, kind = cpu_reference_run(cells, prm, n, 0, threads)
    ncell = fluid_cells(cells)
    return {"value": ncell * n / dt / 1e6, "unit": "MLUPS", "cores": threads, "kind": kind,
            "sample": f"{n} steps of the same 64^3 state after Init + 1 warm-up step, "
                      f"{threads} OpenMP threads, {dt:.1f} s"}


# ---------------------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------------------
def run_reference_mc(args, dist):
    """The reference's multicomponent solver (reference LBM + Cantera-API shim) on the
    host cores, each step over a slab of the workload sized so that the whole
    --steps/--warmup run takes about two minutes."""
    threads = os.cpu_count() or 1
    budget = 120.0 / max(1, args.steps + args.warmup)
    cross, m = mc_cpu_sample(args, budget, threads)
    m, mix, sp = mc_workload(args, cross=cross)
    ncell = fluid_cells(mix)
    with stdout_to_stderr():
        dt = mc_cpu_run(m, mix, sp, args.steps, args.warmup, threads, mc_reaction(args))
    v = ncell * args.steps / dt / 1e6
    shape = "x".join(str(s_ - 2) for s_ in mix.shape)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "MLUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded sinusoidal H2/air interface, numpy PCG64 seed 20261203)",
        "config": {"workload": mc_workload_name(args, ncell_shape=shape), "cells": ncell, "threads": threads},
        "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": threads, "kind": "reference",
                         "sample": f"{shape} slab of the {args.N}-cell-long workload, {args.steps} steps after "
                                   f"{args.warmup} warm-up steps, reference multicomponent LBM + Cantera-API shim"},
        "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def mc_workload_name(args, ncell_shape):
    reaction = mc_reaction(args)
    chem = ""
    if reaction:
        chem = {"rosenbrock": "ROS2 stiff chemistry",
                "surrogate": "MLP chemistry surrogate trained online from ROS2 (1 % audit)"}.get(
                    args.chem, "reference explicit chemistry")
    return (f"{args.workload}{args.N}_mc9_{args.precision}"
            + ({"rosenbrock": "_ros2", "surrogate": "_surrogate"}.get(args.chem, "") if reaction else "")
            + f": 9-species H2/O2/N2 D3Q27, {ncell_shape} {MC_SHAPES[args.workload]}, dx 20 um, dt 1 ns, "
            + (chem if reaction else "non-reacting"))


def run_reference(args, dist):
    if dist.rank != 0:
        return
    if args.workload != "tgv":
        run_reference_mc(args, dist)
        return
    cells, prm = workload(args.N)
    threads = os.cpu_count() or 1
    with stdout_to_stderr():
        dt, kind = cpu_reference_run(cells, prm, args.steps, args.warmup, threads)
    ncell = fluid_cells(cells)
    v = ncell * args.steps / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "MLUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Taylor-Green vortex)",
        "config": {"workload": f"tgv{args.N}_sc_fp64", "cells": ncell, "threads": threads},
        "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": threads, "kind": kind,
                         "sample": f"{args.steps} steps after {args.warmup} warm-up steps"},
        "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)




def mc_bytes(kernel, pop_bytes, reaction=False):
    """Algorithmic bytes per fluid cell of one multicomponent launch (9 species): every
    population (270 planes of `pop_bytes`) read once and, by the update, written once;
    the FP64 record, parameter and sum planes each kernel must read or write once per cell.
      k_mc_relax : 270 populations in and out; per species rho_a, the 3 face terms and
                   the parameters om_a, F_a (3) [, drho_a]; shared u (3), T, rho; the
                   energy set's 7 parameters -> 9 * (4 + 4) + 5 + 7 = 84 planes [+ 9]
      k_mc_gather: 270 populations pulled, 91 sum planes written (per species rho_a, j_a,
                   its P-tensor share; the energy sum)
      k_mc_solve : the 91 sum planes, 21 record planes (rho, T, p, rho_a, X_a) and the 36
                   D_ab read, 88 record planes written
      k_mc_props : 58 record planes of the cell, 86 parameter planes written (49 + the 36
                   D_ab + R/W) [+ HRR]
      k_mc_eflux : 53 record planes of the cell (rho, u, T, p, rho_a, u_a, the P tensor, the
                   heat flux) + 3 rates read, 40 read once by its neighbours, 3 written"""
    if kernel == "k_mc_relax":
        return 2 * 270 * pop_bytes + (84 + (9 if reaction else 0)) * 8
    if kernel == "k_mc_props":
        return (58 + 86 + (1 if reaction else 0)) * 8
    if kernel == "k_mc_eflux":
        return (53 + 3 + 40 + 3) * 8
    if kernel == "k_mc_solve":
        return (91 + 21 + 36 + 88) * 8
    return 270 * pop_bytes + 91 * 8  # k_mc_gather


MC_SHAPES = {"mix": "periodic", "react": "periodic", "inflow": "TYPE_I_C inflow / TYPE_O_C outflow in x, periodic y z",
             "chan": "TYPE_O_C outflow at both x ends, TMS solid y walls, periodic z",
             "flame": "TYPE_O_C outflow at both x ends, TMS solid y walls, periodic z"}


def mc_workload(args, cross=None):
    """The multicomponent workload; `cross` shrinks the two transverse axes (a slab of the
    same case, for the bounded CPU samples)."""
    import mech
    import workloads
    m = mech.h2_air_9()
    N = args.N
    if args.workload == "inflow":
        c = cross or N
        mix, sp = workloads.inflow_layer_mc(m, NX=N, NY=c, NZ=c)
    elif args.workload == "chan":
        c = cross or N // 2
        mix, sp = workloads.flame_channel_mc(m, NX=2 * N, NY=c, NZ=c)
    elif args.workload == "flame":
        c = min(cross or N // 16, N // 16)
        mix, sp = workloads.flame_channel_mc(m, NX=4 * N, NY=c, NZ=c)
    else:
        c = cross or N
        kw = {"T_hi": 1800.0} if args.workload == "react" else {}
        mix, sp = workloads.mixing_layer_mc(m, N=N, NY=c, NZ=c, **kw)
    return m, mix, sp


def mc_reaction(args):
    return args.workload in ("react", "chan", "flame")


def mc_cpu_sample(args, budget_s, threads):
    """The reference's multicomponent solver on a slab of the workload (full extent along
    x, the transverse axes shrunk so that one step takes about budget_s): returns
    (slab cells, seconds per step measured over `steps`, description)."""
    m, mix, sp = mc_workload(args, cross=8)
    reaction = mc_reaction(args)
    with stdout_to_stderr():
        t8 = mc_cpu_run(m, mix, sp, 1, 1, threads, reaction)
    rate = fluid_cells(mix) / max(t8, 1e-6)  # cells per second
    nx = mix.shape[0] - 2
    cross = int(max(4, min(args.N, (rate * budget_s / nx) ** 0.5)))
    if args.workload == "chan":
        cross = min(cross, args.N // 2)
    if args.workload == "flame":
        cross = min(cross, args.N // 16)
    return cross, m


def mc_cpu_run(m, mix, sp, steps, warmup, threads, reaction):
    """The reference's own multicomponent solver on the Cantera-API shim (oracle/_ref)."""
    import workloads
    from oracle import refmc
    fast = refmc.available(reaction, fast=True)  # the reference's own -O3 -ffast-math build
    refmc.set_threads(threads, reaction, fast)
    N3 = [s_ - 2 for s_ in mix.shape]
    ref = refmc.RefMC(*N3, m, workloads.FLAME_UNITS, workloads.MIXTURE_MC, workloads.SPECIES, reaction=reaction,
                      fast=fast)
    ref.cells[...] = mix
    for a in range(len(sp)):
        ref.species[a][...] = sp[a]
    ref.init()
    if warmup:
        ref.loop(warmup)
    t0 = time.perf_counter()
    ref.loop(steps)
    dt = time.perf_counter() - t0
    ref.close()
    return dt


def surrogate_vs_plain(lat, mix, sp, K, refresh_s, cap):
    """From the lattice's current state, K steps with the surrogate (1 % audit; the audited
    states collected and the network refreshed from them every 50 steps, timed into
    refresh_s) and, after restoring the state, K steps of plain ROS2: the comparison the
    surrogate is held to -- peak temperature and heat release integrated over the cells and
    the K steps -- from the device diagnostics (lbmgpu_diagnostics) after every step."""
    import lbmgpu
    import workloads
    c0 = mix.copy()
    s0 = [a.copy() for a in sp]
    lat.download(c0, s0)
    d0 = lat.diagnostics()
    runs, status = {}, {}
    for name, on in (("surrogate", True), ("plain", False)):
        lat.upload(c0, s0)
        lat.surrogate_enable(on, audit_period=100)
        lat.surrogate_collect(on, stride=100, capacity=cap)
        hrr, tpk = 0.0, d0["T_max"]
        for k in range(K):
            if on and k > 0 and k % 50 == 0:
                t0 = time.perf_counter()
                lat.surrogate_train(epochs=2, batch=4096, lr=5e-4, seed=20261204 + k)
                refresh_s.append(time.perf_counter() - t0)
            lat.step(1)
            d = lat.diagnostics()
            hrr += d["hrr"]
            tpk = max(tpk, d["T_max"])
        runs[name] = (hrr, tpk, d["T_max"])
        status[name] = lat.synchronize()
        if on:
            st = lat.surrogate_stats()
            audit = {"audit_rel_err": st["audit_rel_err"],
                     "integrated_frac": st["cells_integrated"] / max(1, st["cells_predicted"] + st["cells_integrated"]
                                                                     + st["cells_audited"])}
    kelvin = lbmgpu.units_from_dx_dt(*workloads.FLAME_UNITS)[3]
    (hs, ps, fs), (hp, pp, fp) = runs["surrogate"], runs["plain"]
    return {"compare_steps": K,
            "peak_T_K": {"surrogate": ps * kelvin, "plain": pp * kelvin, "start": d0["T_max"] * kelvin},
            "peak_T_rel_err": abs(ps - pp) / abs(pp),
            "peak_T_rise_rel_err": abs(ps - pp) / max(abs(pp - d0["T_max"]), 1e-300),
            "final_T_max_rel_err": abs(fs - fp) / abs(fp),
            "heat_release_integrated": {"surrogate": hs, "plain": hp, "unit": "lattice (sum over cells and steps)"},
            "heat_release_rel_err": abs(hs - hp) / max(abs(hp), 1e-300), "compare_status": status,
            "compare_audit": audit}


def run_ours_mc(args, dist):
    import numpy as np

    import lbmgpu
    import workloads
    device = dist.local
    reaction = mc_reaction(args)
    m, mix, sp = mc_workload(args)
    ncell = fluid_cells(mix)
    chem = lbmgpu.CHEM_OFF
    if reaction:
        chem = lbmgpu.CHEM_ROSENBROCK if args.chem in ("rosenbrock", "surrogate") else lbmgpu.CHEM_REF_EXPLICIT
    use_sur = reaction and args.chem == "surrogate"

    prec = lbmgpu.FP32 if args.precision == "fp32" else lbmgpu.FP64
    pop_bytes = 4 if args.precision == "fp32" else 8

    def lattice():
        return lbmgpu.Lattice(*mix.shape, mech=m, dtype=workloads.MIXTURE_MC, species_dtype=workloads.SPECIES,
                              dx_dt=workloads.FLAME_UNITS, chem=chem, device=device, precision=prec)

    lat = lattice()
    lat.upload(mix, sp)
    lat.init()
    sur = None
    if use_sur:
        # teacher steps (ROS2) writing samples, training, then the surrogate with a 1 % audit
        cap = 1 << 21
        stride = max(1, -(-mix.size * args.teach // cap))
        lat.surrogate_collect(True, stride=stride, capacity=cap)
        t0 = time.perf_counter()
        lat.step(args.teach)
        lat.synchronize()
        t_teach = time.perf_counter() - t0
        lat.surrogate_collect(False)
        t0 = time.perf_counter()
        n_aug = int(args.augment * lat.surrogate_stats()["samples"])
        if n_aug > 0:
            lat.surrogate_augment(n_aug, span_y=1.5, span_t=0.01, y_trace=1e-3, seed=20261203)
        lat.synchronize()
        t_aug = time.perf_counter() - t0
        t0 = time.perf_counter()
        loss = lat.surrogate_train(epochs=args.epochs, batch=4096, lr=2e-3, seed=20261203)
        t_train = time.perf_counter() - t0
        n_samples = lat.surrogate_stats()["samples"]
        lat.surrogate_enable(True, audit_period=100)
        sur_params = lat.surrogate_params()
        # online: from here on the audited states are collected, and the network is refreshed
        # from them between the measurements and every 50 steps of the comparison run
        sur_cap = n_samples + (200 + args.compare) * (-(-mix.size // 100))
        lat.surrogate_collect(True, stride=100, capacity=sur_cap)
        sur = {"teacher_steps": args.teach, "sample_stride": stride, "samples_rows": n_samples,
               "teacher_s": t_teach, "augmented_rows": n_aug, "augment_s": t_aug, "train_epochs": args.epochs, "train_s": t_train, "train_loss": loss}
    lat.time_steps(max(3, args.warmup))
    if use_sur:
        lat.surrogate_enable(True, audit_period=100)  # the audit report covers the timed steps
    dist.barrier()
    clk = Clocks(device)
    clk.start()
    ms = lat.time_steps(args.steps)
    clocks = clk.stop()
    status = lat.synchronize()
    ms = dist.max(ms)
    if use_sur:
        st = lat.surrogate_stats()
        tot = max(1, st["cells_predicted"] + st["cells_integrated"] + st["cells_audited"])
        sur.update({"audit_rel_err": st["audit_rel_err"], "audit_max_abs_err": st["audit_max_abs_err"],
                    "predicted_frac": st["cells_predicted"] / tot, "integrated_frac": st["cells_integrated"] / tot,
                    "audited_frac": st["cells_audited"] / tot})
    kk = min(args.steps, 20)
    lat.profile(True)
    lat.time_steps(kk)
    launches, kms = lat.kernel_times()
    lat.profile(False)
    if use_sur:
        t0 = time.perf_counter()
        lat.surrogate_train(epochs=2, batch=4096, lr=5e-4, seed=20261204)
        sur["refresh_s"] = [time.perf_counter() - t0]
        # plain ROS2 on the same lattice and state, for the comparison
        lat.surrogate_collect(False)
        lat.surrogate_enable(False)
        kp = min(args.steps, 10)
        ms_plain = lat.time_steps(kp)
        sur["plain_chem_mlups"] = ncell * kp / (ms_plain * 1e-3) / 1e6
        sur["surrogate_ms_per_step"] = kms[4] / max(kk, 1)
        # the chemistry part of a step: the chemistry kernel (ROS2, or the surrogate's use of
        # its prediction) plus, with the surrogate, its features, network and integrator
        # list; plain ROS2 profiled over a few more plain steps; the transport kernel, the
        # same in both, is not chemistry
        lat.profile(True)
        lat.time_steps(kp)
        _, kms_plain = lat.kernel_times()
        lat.profile(False)
        chem_sur = (kms[4] + kms[7]) / max(kk, 1)
        chem_plain = kms_plain[7] / max(kp, 1)
        sur["chemistry_ms_per_step"] = {"surrogate": chem_sur, "plain": chem_plain,
                                        "speedup": chem_plain / max(chem_sur, 1e-12)}
        sur["network_flops_per_cell"] = 2 * (12 * 128 + 2 * 128 * 128 + 128 * 10)
        if args.compare > 0:
            sur.update(surrogate_vs_plain(lat, mix, sp, args.compare, sur["refresh_s"], sur_cap))
    lat.close()
    avg = {"k_mc_relax": kms[0] / max(launches[0], 1), "k_mc_gather": kms[1] / max(launches[1], 1),
           "k_mc_solve": kms[5] / max(launches[5], 1), "k_mc_props": kms[3] / max(launches[3], 1),
           "k_mc_eflux": kms[6] / max(launches[6], 1)}
    hbm_kernels = ("k_mc_relax", "k_mc_gather")
    dom = max(hbm_kernels, key=avg.get)  # the dominant population-moving kernel
    alg = mc_bytes(dom, pop_bytes, reaction) * ncell
    peak, peak_kind = peaks()
    achieved = alg / (avg[dom] * 1e-3) / 1e9

    # end to end through the reference-facing calls: AoS upload + Init from host memory,
    # the five phase calls per step with the step's conserved totals read back
    # (lbmgpu_sums), one AoS download at the end (the reference's flame setups write
    # output every 1000 steps, setup.cpp:2852); host wall clock
    hm = mix.copy()
    hs = [a.copy() for a in sp]
    lat = lattice()
    if use_sur:  # the network trained above, loaded through the API
        lat.surrogate_params(sur_params)
        lat.surrogate_enable(True, audit_period=100)
    dist.barrier()
    t0 = time.perf_counter()
    lat.upload(hm, hs)
    lat.init()
    for s_ in range(args.steps):
        lat.collide_species()
        lat.collide()
        lat.streaming()
        lat.tms_bc()
        lat.calculate_moment()
        tot = lat.sums()
    lat.synchronize()
    lat.download(hm, hs)
    wall = dist.max(time.perf_counter() - t0)
    lat.close()
    nbytes = mix.nbytes + sum(a.nbytes for a in sp)
    e2e = {"value": whole_job_mlups(dist.world, ncell, args.steps, wall), "unit": "MLUPS",
           "h2d_bytes_per_step": nbytes / args.steps,
           "d2h_bytes_per_step": nbytes / args.steps + 8 * len(tot),
           "note": "AoS upload + Init, per step the five phase calls and the conserved totals read back, "
                   "one AoS download"}
    if dist.rank != 0:
        return
    value = whole_job_mlups(dist.world, ncell, args.steps, ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": dist.world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded H2/air cases of the reference's flame setups, numpy PCG64 seed 20261203)",
        "config": {"workload": mc_workload_name(args, "x".join(str(s_ - 2) for s_ in mix.shape)),
                   "cells": ncell, "parallelism": f"replicas{dist.world}", "l2": "state larger than L2, no flush",
                   "storage": ("FP32 populations (shifted), FP64 records; transport properties in FP32, the "
                               "chemistry, moment solve and temperature recovery in FP64") if pop_bytes == 4
                   else "FP64"},
        "hbm_gbs_step": ncell * sum(mc_bytes(k, pop_bytes, reaction) for k in ("k_mc_relax", "k_mc_gather", "k_mc_solve", "k_mc_props", "k_mc_eflux"))
        / (ms / args.steps * 1e-3) / 1e9,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": ncu_traffic(dom, ncell, f"{args.workload}_{args.precision}"),
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "alg_bytes_per_launch": alg, "mean_launch_ms": avg[dom], "kernel_ms": avg},
        "gpu_launches": int(round(sum(launches) / kk * args.steps)),
        "status": status, "clocks": clocks, "e2e": e2e,
        **({"surrogate": sur} if sur else {}),
    }
    if dist.world == 1 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            n = 5
            cross, _ = mc_cpu_sample(args, 3.0, threads)
            m2, mix2, sp2 = mc_workload(args, cross=cross)
            with stdout_to_stderr():
                dt = mc_cpu_run(m2, mix2, sp2, n, 1, threads, reaction)
            line["cpu_baseline"] = {"value": fluid_cells(mix2) * n / dt / 1e6, "unit": "MLUPS", "cores": threads,
                                    "kind": "reference",
                                    "sample": f"{'x'.join(str(s_ - 2) for s_ in mix2.shape)} slab of the workload, "
                                              f"{n} steps after 1 warm-up step, reference multicomponent LBM + "
                                              f"Cantera-API shim, {threads} OpenMP threads, {dt:.1f} s"}
        except Exception as exc:
            line["cpu_baseline"] = {"value": None, "error": str(exc)}
    print(json.dumps(line), flush=True)


def run_ours(args, dist):
    import numpy as np

    import lbmgpu
    device = dist.local
    cells, prm = workload(args.N)
    Nx, Ny, Nz = cells.shape
    ncell = fluid_cells(cells)
    lat = lbmgpu.Lattice(Nx, Ny, Nz, prm["nu"], prm["R"], prm["gamma"], prm["prtl"], device=device)
    lat.upload(cells)
    lat.init()
    lat.time_steps(max(3, args.warmup))

    # ---- device-timed resident run
    dist.barrier()
    clk = Clocks(device)
    clk.start()
    ms = lat.time_steps(args.steps)
    clocks = clk.stop()
    status = lat.synchronize()
    ms = dist.max(ms)

    # ---- per-kernel times (separate short run with per-launch events)
    kk = min(args.steps, 200)
    lat.profile(True)
    lat.time_steps(kk)
    launches, kms = lat.kernel_times()
    lat.profile(False)
    per_step_launches = (launches[0] + launches[1] + launches[2]) / kk
    avg = {"k_sc_collide": kms[0] / max(launches[0], 1), "k_sc_stream_moment": kms[1] / max(launches[1], 1)}
    dom = max(avg, key=avg.get)
    alg = (BYTES_COLLIDE_FP64 if dom == "k_sc_collide" else BYTES_STREAM_FP64) * ncell
    peak, peak_kind = peaks()
    achieved = alg / (avg[dom] * 1e-3) / 1e9
    lat.close()

    # ---- end to end through the reference-facing phase calls, host buffers
    e2e = None
    try:
        import torch
        pinned = torch.empty(cells.nbytes, dtype=torch.uint8, pin_memory=True)
        host = np.frombuffer(pinned.numpy(), dtype=cells.dtype).reshape(cells.shape)
    except Exception:
        host = np.empty_like(cells)
    host[...] = cells
    lat = lbmgpu.Lattice(Nx, Ny, Nz, prm["nu"], prm["R"], prm["gamma"], prm["prtl"], device=device)
    lat.upload(host)
    lat.init()
    for _ in range(max(3, args.warmup)):
        lat.collide(); lat.streaming(); lat.tms_bc(); lat.calculate_moment()
    lat.synchronize()
    host[...] = cells
    dist.barrier()
    t0 = time.perf_counter()
    lat.upload(host)
    lat.init()
    nread = 0
    for s in range(1, args.steps + 1):
        lat.collide()
        lat.streaming()
        lat.tms_bc()
        lat.calculate_moment()
        if s % OUTPUT_EVERY == 0:
            lat.status()
            lat.download(host)
            nread += 1
    lat.synchronize()
    wall = dist.max(time.perf_counter() - t0)
    lat.close()
    e2e = {"value": whole_job_mlups(dist.world, ncell, args.steps, wall), "unit": "MLUPS",
           "h2d_bytes_per_step": cells.nbytes / args.steps,
           "d2h_bytes_per_step": (cells.nbytes + 4) * nread / args.steps,
           "note": f"upload of the AoS state once, phase calls per step, AoS download + status every {OUTPUT_EVERY} steps"}

    if dist.rank != 0:
        return
    value = whole_job_mlups(dist.world, ncell, args.steps, ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": dist.world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Taylor-Green vortex, numpy PCG64 seed 20261203)",
        "config": {"workload": f"tgv{args.N}_sc_fp64: single-component thermal D3Q27, {args.N}^3 periodic, "
                               f"Ma 0.1, Re 400, FP64 (config 1)",
                   "cells": ncell, "parallelism": f"replicas{dist.world}",
                   "l2": "state larger than L2 (248 MB of populations), no flush"},
        "hbm_gbs_step": ncell * BYTES_STEP_FP64 / (ms / args.steps * 1e-3) / 1e9,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": ncu_traffic(dom, ncell, "tgv_fp64"),
                     "peak_source": f"{peak_kind} hbm_gbs", "alg_bytes_per_launch": alg,
                     "mean_launch_ms": avg[dom], "kernel_ms": avg},
        "gpu_launches": int(round(per_step_launches * args.steps)),
        "status": status,
        "clocks": clocks,
        "e2e": e2e,
    }
    if dist.world == 1 and not args.no_cpu_baseline:
        try:
            with stdout_to_stderr():
                line["cpu_baseline"] = cpu_baseline(cells, prm)
        except Exception as exc:  # the baseline never decides the GPU number
            line["cpu_baseline"] = {"value": None, "error": str(exc)}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# config 4: the decaying turbulent reacting H2/air layer, 256^3, FP32 populations, stiff
# chemistry -- generated and uploaded plane range by plane range (its AoS copy is 83 GB)
# ---------------------------------------------------------------------------------------
TURB_CHUNK = 8  # x-planes per upload / download call


def turb_units(args):
    return (args.dx, args.dx / args.dxdt)


def turb_gen(args, m, N, field, i0, i1):
    import workloads
    return workloads.turbulent_layer_mc(m, N=N, i0=i0, i1=i1, field=field, T_hi=args.t_hot, u_rms=args.urms,
                                        units=turb_units(args))


def turb_name(args, N):
    chem = {"rosenbrock": "ROS2 stiff chemistry", "ref": "the reference's explicit chemistry",
            "surrogate": "MLP chemistry surrogate"}[args.chem]
    return (f"turb{N}_mc9_{args.precision}_{ {'rosenbrock': 'ros2', 'ref': 'refchem', 'surrogate': 'sur'}[args.chem]}: "
            f"decaying turbulent reacting H2/air layer (config 4), 9-species D3Q27, {N}^3, periodic x z, TYPE_O_C "
            f"y faces, u' {args.urms} l.u. (k0 4), air 300 K / H2-air {args.t_hot:g} K, dx {args.dx:g} m, "
            f"dx/dt {args.dxdt:g} m/s, {chem}")


def turb_cpu_child(args):
    """Runs in a child process (bench.py --cpu-child): the reference's own solver on an N^3
    instance of the turbulent layer, printing one JSON line {cells, steps, seconds}.  A child,
    because the reference aborts the whole process when its temperature iteration fails."""
    import mech
    import workloads
    from oracle import refmc
    m = mech.h2_air_9()
    N = args.N
    mix, sp = turb_gen(args, m, N, None, 0, N + 2)
    threads = os.cpu_count() or 1
    fast = refmc.available(True, fast=True)
    refmc.set_threads(threads, True, fast)
    with stdout_to_stderr():
        ref = refmc.RefMC(N, N, N, m, turb_units(args), workloads.MIXTURE_MC, workloads.SPECIES, reaction=True,
                          fast=fast)
        ref.cells[...] = mix
        for a in range(len(sp)):
            ref.species[a][...] = sp[a]
        ref.init()
        if args.warmup:
            ref.loop(args.warmup)
        t0 = time.perf_counter()
        ref.loop(args.steps)
        dt = time.perf_counter() - t0
        ref.close()
    print(json.dumps({"cells": N ** 3, "steps": args.steps, "seconds": dt, "threads": threads,
                      "kind": "reference" if fast else "reference (oracle build)"}), flush=True)


def turb_cpu_sample(args, N, steps, warmup):
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-child", "--N", str(N), "--steps", str(steps),
           "--warmup", str(warmup), "--urms", str(args.urms), "--t-hot", str(args.t_hot), "--dx", str(args.dx),
           "--dxdt", str(args.dxdt)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    for line in r.stdout.splitlines()[::-1]:
        if line.startswith("{"):
            return json.loads(line)
    raise RuntimeError(f"reference solver exited with {r.returncode}: {r.stderr.strip().splitlines()[-1:]}")


def run_reference_turb(args, dist):
    if dist.rank != 0:
        return
    Ns = 64  # a bounded instance of the case: about 10 s of the reference's solver for 20 steps
    try:
        d = turb_cpu_sample(args, Ns, args.steps, args.warmup)
        v = d["cells"] * d["steps"] / d["seconds"] / 1e6
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "MLUPS", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": d["seconds"] * 1e3 / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded turbulence field and H2/air layer, numpy PCG64 seed 20261203)",
                "config": {"workload": turb_name(args, args.N), "cells": args.N ** 3, "threads": d["threads"]},
                "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": d["threads"], "kind": "reference",
                                 "sample": f"{Ns}^3 instance of the same case, {args.steps} steps after {args.warmup} "
                                           f"warm-up steps, reference multicomponent LBM + Cantera-API shim with "
                                           f"its explicit chemistry, built with the reference's flags"},
                "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    except Exception as exc:
        line = {"impl": "reference", "unavailable": f"the reference solver failed on the workload: {exc}"}
    print(json.dumps(line), flush=True)


def surrogate_block(args, device):
    """Config 5's case -- the reacting H2/air channel of config 3 (NSCBC outflow ends, TMS
    walls, 1800 K ignition kernel), FP32 populations, ROS2 chemistry -- at args.sur_shape:
    ROS2 teacher steps writing ~2 M sample rows, augmentation and training, then the
    surrogate (1 % audit, online collection) against plain ROS2 on the same GPU and state:
    the chemistry kernels' time per step, and over args.compare steps from the same state
    (network refreshed every 50) the peak temperature and the integrated heat release."""
    import lbmgpu
    import mech
    import workloads
    m = mech.h2_air_9()
    NX, NY, NZ = (int(x) for x in args.sur_shape.split("x"))
    mix, sp = workloads.flame_channel_mc(m, NX=NX, NY=NY, NZ=NZ)
    ncell = fluid_cells(mix)
    lat = lbmgpu.Lattice(*mix.shape, mech=m, dtype=workloads.MIXTURE_MC, species_dtype=workloads.SPECIES,
                         dx_dt=workloads.FLAME_UNITS, chem=lbmgpu.CHEM_ROSENBROCK, device=device,
                         precision=lbmgpu.FP32)
    lat.upload(mix, sp)
    lat.init()
    cap = 1 << 21
    stride = max(1, -(-mix.size * args.teach // cap))
    lat.surrogate_collect(True, stride=stride, capacity=cap)
    t0 = time.perf_counter()
    lat.step(args.teach)
    lat.synchronize()
    out = {"case": f"config 5's case at {NX}x{NY}x{NZ}: reacting H2/air channel, NSCBC outflow ends, TMS walls, "
                   f"1800 K ignition kernel, FP32 populations", "cells": ncell, "teacher_steps": args.teach,
           "teacher_s": time.perf_counter() - t0}
    lat.surrogate_collect(False)
    n_rows = lat.surrogate_stats()["samples"]
    lat.surrogate_augment(int(args.augment * n_rows), span_y=1.5, span_t=0.01, y_trace=1e-3, seed=20261203)
    t0 = time.perf_counter()
    out["train_loss"] = lat.surrogate_train(epochs=args.epochs, batch=4096, lr=2e-3, seed=20261203)
    out.update({"train_s": time.perf_counter() - t0, "sample_rows": lat.surrogate_stats()["samples"],
                "teacher_rows": n_rows, "train_epochs": args.epochs})
    sur_cap = lat.surrogate_stats()["samples"] + (40 + args.compare) * (-(-mix.size // 100))
    kk = 20
    lat.surrogate_enable(True, audit_period=100)
    lat.surrogate_collect(True, stride=100, capacity=sur_cap)
    lat.profile(True)
    ms_sur = lat.time_steps(kk)
    _, kms = lat.kernel_times()
    lat.profile(False)
    st = lat.surrogate_stats()
    tot = max(1, st["cells_predicted"] + st["cells_integrated"] + st["cells_audited"])
    out.update({"audit_rel_err": st["audit_rel_err"], "predicted_frac": st["cells_predicted"] / tot,
                "integrated_frac": st["cells_integrated"] / tot, "audited_frac": st["cells_audited"] / tot,
                "surrogate_step_mlups": ncell * kk / (ms_sur * 1e-3) / 1e6})
    refresh = []
    t0 = time.perf_counter()
    lat.surrogate_train(epochs=2, batch=4096, lr=5e-4, seed=20261204)
    refresh.append(time.perf_counter() - t0)
    lat.surrogate_collect(False)
    lat.surrogate_enable(False)
    kp = 10
    lat.profile(True)
    ms_plain = lat.time_steps(kp)
    _, kmp = lat.kernel_times()
    lat.profile(False)
    chem_sur, chem_plain = (kms[4] + kms[7]) / kk, kmp[7] / kp
    out.update({"plain_step_mlups": ncell * kp / (ms_plain * 1e-3) / 1e6,
                "chemistry_ms_per_step": {"surrogate": chem_sur, "plain": chem_plain,
                                          "speedup": chem_plain / max(chem_sur, 1e-12),
                                          "kernels": "surrogate: features, network, the prediction's use and the "
                                                     "integrator list; plain: the ROS2 kernel; the transport kernel "
                                                     "both share is not counted"},
                "network_flops_per_cell": 2 * (12 * 128 + 2 * 128 * 128 + 128 * 10)})
    if args.compare > 0:
        out.update(surrogate_vs_plain(lat, mix, sp, args.compare, refresh, sur_cap))
    out["refresh_s"] = refresh
    out["status"] = lat.synchronize()
    lat.close()
    return out


class SlabStepper:
    """World > 1 (or the loopback check): one slab per rank along x, the rank's 256^3 box of
    the turbulent layer (the global domain is `world` such boxes in a row, periodic in x),
    halo planes exchanged every step (slab.exchange) -- over NCCL, issued on the library's own
    stream so that the exchange, the kernels and the timing events share one ordering."""

    def __init__(self, lat, dist, loopback=False):
        import torch

        import slab
        self.torch, self.slab, self.lat, self.dist = torch, slab, lat, dist
        self.world, self.rank = (1, 0) if loopback else (dist.world, dist.rank)
        self.ext = torch.cuda.ExternalStream(lat.stream())
        self.bufs = {w: [torch.empty(lat.halo_bytes(w) // 8, dtype=torch.float64, device="cuda") for _ in range(2)]
                     for w in (slab.POPULATIONS, slab.RECORD)}
        self.comm = LoopbackComm(torch) if loopback else slab.TorchComm(dist.pg)

    def pack(self, face, what):
        buf = self.bufs[what][face]
        self.lat.halo_pack(face, what, buf.data_ptr())
        return buf

    def unpack(self, face, what, t):
        self.lat.halo_unpack(face, what, t.data_ptr())

    def exchange(self, what):
        with self.torch.cuda.stream(self.ext):
            self.slab.exchange(what, self.pack, self.unpack, self.comm, self.world, self.rank)

    def steps(self, k, after=None):
        lat = self.lat
        for _ in range(k):
            lat.collide_species()
            lat.collide()
            self.exchange(self.slab.POPULATIONS)
            lat.streaming()
            lat.tms_bc()
            lat.calculate_moment()
            self.exchange(self.slab.RECORD)
            if after:
                after()

    def time_steps(self, k):
        """Device milliseconds of k steps, CUDA events on the library's stream."""
        t = self.torch
        e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        e0.record(self.ext)
        self.steps(k)
        e1.record(self.ext)
        e1.synchronize()
        return e0.elapsed_time(e1)


class LoopbackComm:
    """exchange() transport of a single slab that is its own neighbour: each receive takes
    the send with the matching tag (device copies on the current stream)."""

    def __init__(self, torch):
        self.torch = torch

    def empty_like(self, t):
        return self.torch.empty_like(t)

    def sendrecv(self, ops):
        sent = {tag: buf for kind, buf, peer, tag in ops if kind == "send"}
        for kind, buf, peer, tag in ops:
            if kind == "recv":
                buf.copy_(sent[tag])


def run_ours_turb(args, dist):
    import lbmgpu
    import mech
    import workloads
    device = dist.local
    m = mech.h2_air_9()
    N = args.N
    ncell = N ** 3
    field = workloads.turbulence_field(N, u_rms=args.urms)
    chem = {"rosenbrock": lbmgpu.CHEM_ROSENBROCK, "ref": lbmgpu.CHEM_REF_EXPLICIT}[args.chem]
    prec = lbmgpu.FP32 if args.precision == "fp32" else lbmgpu.FP64
    pop_bytes = 4 if args.precision == "fp32" else 8
    lat = lbmgpu.Lattice(N + 2, N + 2, N + 2, mech=m, dtype=workloads.MIXTURE_MC, species_dtype=workloads.SPECIES,
                         dx_dt=turb_units(args), chem=chem, device=device, precision=prec)
    slabs = dist.world > 1 or args.slab_loopback
    st = None
    if slabs:  # the rank's box between two halo planes; the domain: world boxes in a row
        lat.set_halo(1, 1, N * dist.world + 2)
        st = SlabStepper(lat, dist, loopback=args.slab_loopback)

    # host buffers of one plane range (TURB_CHUNK x-planes), page-locked where torch can
    # allocate them so: the end-to-end copies start from pinned host memory
    def host_buffer(dtype, rows):
        import numpy as np
        shape = (rows, N + 2, N + 2)
        try:
            import torch
            nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
            t = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
            return np.frombuffer(t.numpy(), dtype=dtype).reshape(shape), t
        except Exception:
            return np.zeros(shape, dtype=dtype), None

    hb_mix = host_buffer(workloads.MIXTURE_MC, TURB_CHUNK)
    hb_sp = [host_buffer(workloads.SPECIES, TURB_CHUNK) for _ in range(len(m.species_names()))]

    def upload_all():
        """Generates and uploads the state plane range by plane range; returns the seconds
        spent inside the upload calls and the bytes they copied.  Each range is generated
        into the host buffers (outside the timed calls), then uploaded from them.  Slabs: the
        halo planes hold the box's last and first plane (the neighbouring boxes' edge
        planes)."""
        api, nbytes = 0.0, 0
        ranges = [(i0, i0, min(N + 2, i0 + TURB_CHUNK)) for i0 in range(0, N + 2, TURB_CHUNK)]
        if slabs:
            ranges = ([(0, N, N + 1)] + [(i0, i0, min(N + 1, i0 + TURB_CHUNK)) for i0 in range(1, N + 1, TURB_CHUNK)]
                      + [(N + 1, 1, 2)])
        for dst, g0, g1 in ranges:
            gm, gs = turb_gen(args, m, N, field, g0, g1)
            rows = g1 - g0
            mix = hb_mix[0][:rows]
            mix[...] = gm
            sp = [b[0][:rows] for b in hb_sp]
            for d_, s_ in zip(sp, gs):
                d_[...] = s_
            t0 = time.perf_counter()
            lat.upload_planes(dst, mix, sp)
            api += time.perf_counter() - t0
            nbytes += mix.nbytes + sum(a.nbytes for a in sp)
        return api, nbytes

    def init():
        lat.init()
        if slabs:
            st.exchange(1)  # the halo planes' records from the neighbours

    def time_steps(k):
        return st.time_steps(k) if slabs else lat.time_steps(k)

    upload_all()
    init()
    time_steps(max(3, args.warmup))
    dist.barrier()
    clk = Clocks(device)
    clk.start()
    ms = time_steps(args.steps)
    clocks = clk.stop()
    status = lat.synchronize()
    ms = dist.max(ms)
    # per-kernel device times over a few more steps (every launch bracketed by events)
    kk = min(args.steps, 5)
    lat.profile(True)
    time_steps(kk)
    launches, kms = lat.kernel_times()
    lat.profile(False)
    names = {0: "k_mc_relax", 1: "k_mc_gather", 2: "k_mc_special (+ other; slabs: + halo pack/unpack)",
             3: "k_mc_props", 5: "k_mc_solve", 6: "k_mc_eflux", 7: "k_mc_chem"}
    per_step = {names[k]: kms[k] / kk for k in names}
    prof_step = sum(per_step.values())
    step_ms = ms / args.steps
    alg_step = 2 * 27 * 10 * pop_bytes + 16  # survey 8(d): one read + one write of every population, FP64 T
    peak, peak_kind = peaks()
    achieved = alg_step * ncell / (step_ms * 1e-3) / 1e9
    kern = {}
    case = f"turb_{args.precision}"
    step_kernels = ("k_mc_props", "k_mc_chem", "k_mc_eflux", "k_mc_relax", "k_mc_special", "k_mc_gather", "k_mc_solve")
    # the boundary kernel's cells are the two planes next to the outflow faces (2 N^2 per box)
    parts = [ncu_traffic(name, 2 * N * N if name == "k_mc_special" else ncell, case)
             for name in step_kernels]
    step_traffic = sum(parts) if all(p_ is not None for p_ in parts) else None
    for k, name in ((0, "k_mc_relax"), (1, "k_mc_gather")):
        alg = mc_bytes(name, pop_bytes, True) * ncell
        t = kms[k] / max(launches[k], 1)
        kern[name] = {"alg_bytes_per_launch": alg, "mean_launch_ms": t, "achieved_gbs": alg / (t * 1e-3) / 1e9,
                      "frac": alg / (t * 1e-3) / 1e9 / peak, "traffic": ncu_traffic(name, ncell, case)}
    # end to end through the reference-facing calls: plane-range uploads from host memory
    # and Init, per step the five phase calls and the conserved totals read back, the
    # plane-range download of the final state; the time inside those calls
    api_up, nbytes = upload_all()
    dist.barrier()
    t0 = time.perf_counter()
    tot = []

    def read_sums():  # the step's conserved totals; slabs: FP64 all-reduce over the ranks
        tot[:] = lat.sums()
        if dist.world > 1:
            import torch
            t = torch.tensor(tot, dtype=torch.float64, device="cuda")
            dist.pg.all_reduce(t)
            tot[:] = t.tolist()

    init()
    if slabs:
        st.steps(args.steps, after=read_sums)
    else:
        for _ in range(args.steps):
            lat.collide_species()
            lat.collide()
            lat.streaming()
            lat.tms_bc()
            lat.calculate_moment()
            read_sums()
    lat.synchronize()
    api_steps = time.perf_counter() - t0
    api_down = 0.0
    gm, gs = turb_gen(args, m, N, field, 0, TURB_CHUNK)  # the cell types the download keeps
    mix = hb_mix[0]
    mix[...] = gm
    sp = [b[0] for b in hb_sp]
    for d_, s_ in zip(sp, gs):
        d_[...] = s_
    for i0 in range(0, N + 2, TURB_CHUNK):
        i1 = min(N + 2, i0 + TURB_CHUNK)
        mv, sv = mix[: i1 - i0], [a[: i1 - i0] for a in sp]
        t0 = time.perf_counter()
        lat.download_planes(i0, mv, sv)
        api_down += time.perf_counter() - t0
    wall = dist.max(api_up + api_steps + api_down)
    e2e_status = lat.synchronize()
    if st:
        st = None
        import torch
        torch.cuda.synchronize()
    lat.close()
    e2e = {"value": whole_job_mlups(dist.world, ncell, args.steps, wall), "unit": "MLUPS",
           "h2d_bytes_per_step": nbytes / args.steps, "d2h_bytes_per_step": nbytes / args.steps + 8 * len(tot),
           "seconds": {"upload": api_up, "init_steps_sums": api_steps, "download": api_down},
           "note": "time inside the C-ABI calls: plane-range AoS uploads from pinned host buffers + Init, per step "
                   "the five phase calls and the conserved totals read back, the plane-range AoS download into the "
                   "host buffers (host-side generation of the initial state between upload calls excluded)"}
    if dist.rank != 0:
        return
    value = whole_job_mlups(dist.world, ncell, args.steps, ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": dist.world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded turbulence field and H2/air layer, numpy PCG64 seed 20261203)",
        "config": {"workload": turb_name(args, N), "cells": ncell,
                   "parallelism": (f"x-slabs{dist.world} (one {N}^3 box per GPU, halos over NCCL)" if dist.world > 1
                                   else ("x-slab loopback check" if slabs else "single GPU")),
                   "l2": "state larger than L2 (86 GB at 258^3 FP32), no flush",
                   "storage": ("FP32 populations (shifted), FP64 records; transport properties in FP32, the "
                               "chemistry, moment solve and temperature recovery in FP64") if pop_bytes == 4
                   else "FP64"},
        "chemistry": {"ms_per_step": per_step["k_mc_chem"], "fraction_of_step": per_step["k_mc_chem"] / step_ms,
                      "integrator": "ROS2, rtol 1e-5" if args.chem == "rosenbrock" else args.chem},
        "hbm_gbs_step": achieved,
        "roofline": {"bound": "hbm", "kernel": "whole step (all kernels)", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": step_traffic,
                     "traffic_note": "DRAM bytes of one step: the sum over the step's kernels of ncu's "
                                     "dram__bytes_read + write per launch, captured at 64^3 and scaled by cells",
                     "peak_source": f"{peak_kind} hbm_gbs", "alg_bytes_per_cell": alg_step,
                     "alg_bytes_note": "one read + one write of the 270 populations + FP64 T read and write",
                     "kernel_ms_per_step": per_step, "profiled_ms_per_step": prof_step, "kernels": kern},
        "gpu_launches": int(round(sum(launches) / kk * args.steps)),
        "status": status, "e2e_status": e2e_status, "clocks": clocks, "e2e": e2e,
    }
    if dist.world == 1 and not args.no_surrogate:
        try:
            line["surrogate"] = surrogate_block(args, device)
        except Exception as exc:  # the surrogate study never decides the step's number
            line["surrogate"] = {"error": str(exc)}
    if dist.world == 1 and not args.no_cpu_baseline:
        try:
            # ~5 M cell updates: about 10 s of the reference's solver on the box's host cores
            d = turb_cpu_sample(args, 64, 20, 1)
            line["cpu_baseline"] = {"value": d["cells"] * d["steps"] / d["seconds"] / 1e6, "unit": "MLUPS",
                                    "cores": d["threads"], "kind": "reference",
                                    "sample": f"64^3 instance of the same case, {d['steps']} steps after 1 warm-up "
                                              f"step, reference multicomponent LBM + Cantera-API shim with its "
                                              f"explicit chemistry, reference flags, {d['seconds']:.1f} s"}
        except Exception as exc:
            line["cpu_baseline"] = {"value": None, "error": str(exc)}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.N is None:
        args.N = {"tgv": 64, "turb": 256}.get(args.workload, 128)
    if args.steps is None:
        args.steps = {"tgv": 1000, "turb": 20}.get(args.workload, 200)
    if args.chem is None:
        args.chem = "rosenbrock" if args.workload == "turb" else "ref"
    if args.precision is None:
        args.precision = "fp32" if args.workload == "turb" else "fp64"
    if args.cpu_child:
        turb_cpu_child(args)
        return
    dist = Dist()
    try:
        if args.impl == "reference" and args.workload == "turb":
            run_reference_turb(args, dist)
        elif args.impl == "reference":
            run_reference(args, dist)
        elif args.workload == "turb":
            run_ours_turb(args, dist)
        elif args.workload == "tgv":
            run_ours(args, dist)
        else:
            run_ours_mc(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
