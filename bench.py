"""Benchmark of the PhP_FDTD time-step loop on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload cfg1] [--precision fp64|fp32|fp64-strict]

One step = one FDTD time step (H sweep, fused D/source/E/ADE/ion sweep,
monitor probe, running DFT) over the whole domain of the workload.  The
default workload is the 256^3 tensor-ADE configuration (Drude-Lorentz tip
over a rotated lossy anisotropic slab, 12-cell CPML, sine source at
900 cm^-1, running DFT 2 cells above the slab), synthetic inputs from a
fixed seed.  The field state (9 x 16.8 M cells, 1.2 GB in FP64) is far larger
than L2, so no flush is needed between steps.

Prints one JSON line on rank 0.  With --gpus N (torchrun) every rank advances
its own replica of the domain (weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {"cfg0": 0, "cfg1": 1, "cfg2": 2, "cfg3": 3, "cfg4": 4}
# what the solver computes where the workload texts name parameters the
# reference's loop has no input for
REFERENCE_FORM = ("CPML graded as the reference hard-codes it (m = 3, kappa_max = 7, alpha_max = 0.05, "
                  "fdtd.c:975-977; the cfg0 text names kappa_max = 5); ion equations of motion without a damping "
                  "term, as fdtd.c:3521-3528 integrate them (the cfg0 text names gamma = 5 cm^-1)")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=400)
    p.add_argument("--warmup", type=int, default=20)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="cfg1", choices=sorted(WORKLOADS))
    p.add_argument("--precision", default="fp64", choices=["fp64", "fp32", "fp64-strict"])
    p.add_argument("--scale", type=float, default=1.0, help="grid scale (1.0 = the configuration's grid)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-mixed", action="store_true", help="skip the FP32 leg beside the FP64 line")
    p.add_argument("--acc-steps", type=int, default=None,
                   help="steps of the FP32-vs-FP64 error run (default: the configuration's tsteps; 0 = skip)")
    p.add_argument("--case-dir", default=None)
    p.add_argument("--no-largest", action="store_true", help="skip the 1024 x 1024 x 512 (cfg4) sub-object")
    p.add_argument("--no-serving", action="store_true", help="skip the serving (cfg3) sub-object")
    p.add_argument("--no-configs", action="store_true", help="skip the cfg0 / cfg2 sub-object")
    p.add_argument("--slabs", type=int, default=0, help="time the workload as this many z slabs on one GPU")
    p.add_argument("--z-chunk", type=int, default=0, help="planes per sweep block (0 = the library's choice)")
    p.add_argument("--largest-steps", type=int, default=2000,
                   help="steps of the cfg4 runs whose FP32-vs-FP64 error is reported")
    p.add_argument("--requests", type=int, default=256, help="cfg3: number of requests")
    p.add_argument("--max-active", type=int, default=16, help="cfg3: simulations running at once")
    p.add_argument("--baseline-sample", type=int, default=16, help="cfg3: requests run alone for the baselines")
    p.add_argument("--concurrency", action="store_true",
                   help="cfg3 requests of fixed edges, alone and many at once through the serving loop")
    return p.parse_args()


def run_concurrency(args, local):
    """Does running many small simulations at once fill the GPU?  Serving
    requests (FP32, two-atom slab, tip, 8-cell CPML, running DFT) of a fixed
    cubic edge: one alone (its own stream, device-timed steps), and N at once
    through the serving loop (aggregate cell-updates over the makespan on the
    server clock); against the rate of one 192^3 request alone.  A batched
    launch over all running jobs could only recover the gap between the
    concurrent small grids and the large one."""
    import torch
    from php_fdtd_b200 import Simulation
    from php_fdtd_b200.serving import DftSpec, Server
    from php_fdtd_b200.workloads import request_desc

    def req(edge, steps):
        return {"index": 0, "arrival": 0.0, "grid": (edge, edge, edge), "pml": 8, "steps": steps,
                "wavenumber": 1400.0, "tip_height_nm": 20.0}

    def alone(edge, steps):
        holder, dft = request_desc(req(edge, steps), "fp32", device=local)
        with Simulation(holder) as sim:
            sim.dft_add(dft["component"], dft["z_plane"], dft["freqs"])
            sim.step(64)
            sim.sync()
            st = torch.cuda.ExternalStream(sim.stream, device=torch.device("cuda", local))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            sim.step(steps)
            e1.record(st)
            e1.synchronize()
            return edge ** 3 * steps / (e0.elapsed_time(e1) * 1e-3) / 1e9

    def together(edge, steps, n):
        built = [request_desc(req(edge, steps), "fp32", device=local) for _ in range(n)]
        with Server(memory_budget=150 * 10 ** 9, device=local, max_active=n) as srv:
            for q, (holder, dft) in enumerate(built):
                srv.submit(holder, steps, DftSpec(dft["component"], dft["z_plane"], dft["freqs"]), tag=q)
            infos = []
            while len(infos) < n:
                for info in srv.poll(timeout_ms=200):
                    infos.append(info)
                    srv.release(info["job"])
        bad = sum(i["status"] != 0 for i in infos)
        # device-busy span: first job started stepping to last job done
        span = max(i["t_done"] for i in infos) - min(i["t_start"] for i in infos)
        return n * edge ** 3 * steps / span / 1e9, bad

    out = {"metric": "Gcell-updates/s, serving requests of one edge, FP32", "unit": "Gcell-updates/s",
           "big_alone": {"edge": 192, "value": round(alone(192, 2000), 3)}, "edges": {}}
    for edge, steps, n in ((64, 40000, 32), (96, 20000, 24), (128, 10000, 16)):
        agg, bad = together(edge, steps, n)
        out["edges"][str(edge)] = {"alone": round(alone(edge, steps), 3), "together": round(agg, 3), "jobs": n,
                                   "steps": steps, "failed": bad}
    return out


# ----------------------------------------------------------------- plumbing


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append({"sm": float(f[1]), "max": float(f[2]), "power": float(f[3]), "hw": f[5], "hwt": f[6],
                             "swt": f[7], "swp": f[8]})
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        reasons = set()
        for r in rows:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"), ("swt", "sw_thermal_slowdown"),
                              ("swp", "sw_power_cap")):
                if r[key].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in rows), "sm_max_mhz": max(r["max"] for r in rows),
                "power_w_max": max(r["power"] for r in rows), "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------------------ workload


def make_case(workload: str, scale: float, tsteps: int, case_dir: Path) -> Path:
    from php_fdtd_b200.workloads import baseline_case, write_case
    spec = baseline_case(WORKLOADS[workload], tsteps=tsteps, scale=scale)
    cfg = case_dir / "case.cfg"
    stamp = case_dir / "stamp.json"
    key = {"workload": workload, "scale": scale, "tsteps": tsteps}
    if cfg.exists() and stamp.exists() and json.loads(stamp.read_text()) == key:
        return cfg
    write_case(spec, case_dir)
    stamp.write_text(json.dumps(key))
    return cfg


def census(cfg, medium: np.ndarray):
    """Cell counts per material class and PML membership (algorithmic bytes)."""
    nx, ny, nz, L = cfg.nx, cfg.ny, cfg.nz, cfg.pml_thickness
    mats = cfg.materials
    ade = np.array([m.use_ade == 1 for m in mats])
    lossy = np.array([(m.use_ade == 0) and any(m.eps_im[q] != 0 for q in range(9)) for m in mats])
    natom = np.array([m.natom for m in mats])
    counts = np.bincount(medium.ravel(), minlength=len(mats))
    c = {k: int(v) for k, v in enumerate(counts.tolist()) if v}
    n_ade = sum(v for k, v in c.items() if ade[k])
    n_lossy = sum(v for k, v in c.items() if lossy[k])
    atom_words = sum(v * 12 * natom[k] for k, v in c.items())
    n_atom_cells = sum(v for k, v in c.items() if natom[k] > 0)

    def pml_count(n):
        idx = np.arange(n)
        return int(np.sum((idx < L) | (idx >= n - L))) if L > 0 else 0
    px, py, pz = pml_count(nx), pml_count(ny), pml_count(nz)
    # PML axis memberships summed over cells (H sweep covers i<nx-1, j<ny-1)
    pml_e = px * ny * nz + nx * py * nz + nx * ny * pz
    pml_h = (min(px, nx - 1) * (ny - 1) * nz + (nx - 1) * min(py, ny - 1) * nz + (nx - 1) * (ny - 1) * pz)
    return {"cells": nx * ny * nz, "h_cells": (nx - 1) * (ny - 1) * nz, "ade_cells": n_ade, "lossy_cells": n_lossy,
            "atom_cells": n_atom_cells, "atom_words": int(atom_words), "pml_e": pml_e, "pml_h": pml_h}


def algorithmic_bytes(c: dict, s: int, ion_pass: bool = False):
    """Compulsory state traffic per launch: H sweep reads E, H and writes H
    (9 words), plus 4 psi words per PML axis; the fused sweep reads H, D and
    writes D, E (12 words), plus old E in lossy/ADE cells (3), P and P_old
    (12) in ADE cells, r and v (12 N) in atom cells -- or, when the ion pass
    updates the lattice apart, P_ion (3) -- 4 psi words per PML axis, and the
    1-byte material id."""
    h = s * (9 * c["h_cells"] + 4 * c["pml_h"])
    atoms = 3 * c["atom_cells"] if ion_pass else c["atom_words"]
    e = s * (12 * c["cells"] + 3 * (c["ade_cells"] + c["lossy_cells"]) + 12 * c["ade_cells"] + atoms
             + 4 * c["pml_e"]) + c["cells"]
    return h, e


def step_bytes(c: dict, s: int, ion_pass: bool = False):
    """Compulsory state traffic of the one-launch step (he_sweep_tma): reads E,
    H, D and writes E, H, D (18 words per cell: H crosses HBM once each way,
    and the old E of lossy and ADE cells comes with the staged E), P and P_old
    (12) in ADE cells, r and v (12 N) in atom cells -- or P_ion (3) with the
    ion pass apart -- 4 psi words per PML axis of the H and of the D update,
    and the 1-byte material id."""
    atoms = 3 * c["atom_cells"] if ion_pass else c["atom_words"]
    return s * (18 * c["cells"] + 12 * c["ade_cells"] + atoms + 4 * (c["pml_h"] + c["pml_e"])) + c["cells"]


def sweep_rooflines(prof: dict, c: dict, s: int, peak: float, ion_pass: bool = False, dft_cells: int = 0,
                    dft_freqs: int = 0) -> dict:
    """Per-launch rate of each sweep kernel that ran (the one-launch step, or
    the H sweep and the fused D/E sweep) against the copy bandwidth.  When no
    dft_sample launch ran, the E sweep sampled the running DFT itself: per
    sampled cell the value read back (1 word) and 16 bytes read + 16 written
    per frequency of its FP64 accumulators."""
    hb, eb = algorithmic_bytes(c, s, ion_pass)
    dft = dft_cells * (s + 32 * dft_freqs) if prof["dft"]["launches"] == 0 else 0
    eb += dft
    out = {}
    for k, b, name in (("step", step_bytes(c, s, ion_pass) + dft,
                        "he_sweep_tma (one-launch step: H, D, sources, E, ADE, ions)"),
                       ("e_sweep", eb, "e_sweep_tma (fused D/source/E/ADE/ion sweep)"),
                       ("h_sweep", hb, "h_sweep_tma")):
        if prof[k]["launches"]:
            ms = prof[k]["ms"] / prof[k]["launches"]
            gbs = b / (ms * 1e-3) / 1e9
            out[k] = {"kernel": name, "achieved": round(gbs, 1), "frac": round(gbs / peak, 4),
                      "avg_launch_ms": round(ms, 5), "algorithmic_bytes_per_launch": int(b)}
    return out


# ------------------------------------------------------------------ our arm


def run_ours(args, ws, rank, local, precision):
    import torch
    from php_fdtd_b200 import Config, Simulation

    case_dir = Path(args.case_dir or tempfile.gettempdir()) / f"php_bench_{args.workload}_{args.scale}_r{rank}"
    case_dir.mkdir(parents=True, exist_ok=True)
    tsteps = args.warmup + 4 * args.steps + 8
    cfg_path = make_case(args.workload, args.scale, tsteps, case_dir)
    old = os.getcwd()
    os.chdir(case_dir)
    try:
        cfg = Config.load("case.cfg")
        medium = cfg.load_medium()
    finally:
        os.chdir(old)
    holder = cfg.desc(medium, precision)
    holder.desc.device = local
    holder.desc.z_chunk = args.z_chunk
    sim = Simulation(holder)
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    V = nx * ny * nz
    oi = cfg.output_interval
    # per-step extras of the configuration: monitor probe and running DFT
    sim.probe_set(cfg.monitor_x, cfg.monitor_y, cfg.monitor_z + 1, cfg.monitor_z)
    dft_plane = cfg.output_slice_position + 1
    f_src = cfg.unique_source_frequency
    sim.dft_add("Ez", dft_plane, [f_src], first_step=0, interval=1)
    stream = torch.cuda.ExternalStream(sim.stream, device=torch.device("cuda", local))

    # warm-up: W steps, then one untimed pass of the timed step pattern so that
    # every step graph the timed region launches is already instantiated
    sim.step(args.warmup)
    sim.probe_read()
    sim.step(min(args.steps, 4096))
    sim.probe_read()
    sim.sync()

    # ---- device-resident timed region
    barrier(ws)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        remaining = args.steps
        while remaining > 0:  # the probe ring holds 8192 rows; drain between blocks
            n = min(remaining, 4096)
            sim.step(n)
            remaining -= n
            if remaining > 0:
                sim.probe_read()
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    barrier(ws)
    ms = ev0.elapsed_time(ev1)
    sim.probe_read()
    ms_max = max_over_ranks(ms, ws)
    value = V * args.steps * ws / (ms_max * 1e-3) / 1e9

    # ---- per-kernel device time (event nodes inside the step graphs)
    sim.profile(True)
    sim.step(min(args.steps, 200))
    prof = sim.profile_read()
    sim.profile(False)
    sim.probe_read()

    # ---- end to end through the C ABI with host buffers, over at least four
    # output intervals (a run's steps between its outputs, as the drop-in
    # executable takes them)
    e2e = None
    if not args.no_e2e:
        e2e_steps = max(args.steps, 4 * oi)
        for n in sorted({min(oi, e2e_steps), e2e_steps % oi} - {0}):
            sim.prepare(n)                    # the step graphs, recorded before the clock
        sim.probe_read()
        sim.sync()
        barrier(ws)
        t0 = time.perf_counter()
        done = 0
        d2h = 0
        h2d = 0
        pending = []
        while done < e2e_steps:
            n = min(oi, e2e_steps - done)
            sim.step(n)                       # per-step source values and DFT phasors copied host -> device
            h2d += n * 8 * (cfg.num_sources + 3)
            # the output frame of this interval (monitor rows, |E|max / r max,
            # the slice) copied device -> host behind the steps; the host
            # takes it while the device runs the next interval
            pending.append(sim.frame_begin(diag=True, probe=True,
                                           slice=("Ez", cfg.output_slice_axis, cfg.output_slice_position)))
            if len(pending) > 1:
                fr = sim.frame_wait(pending.pop(0))
                d2h += fr["rows"].nbytes + 32 + fr["slice"].nbytes
            done += n
        for tk in pending:
            fr = sim.frame_wait(tk)
            d2h += fr["rows"].nbytes + 32 + fr["slice"].nbytes
        sim.sync()
        t1 = time.perf_counter()
        barrier(ws)
        e2e_s = max_over_ranks(t1 - t0, ws)
        e2e = {"value": round(V * e2e_steps * ws / e2e_s / 1e9, 4), "unit": "Gcell-updates/s",
               "h2d_bytes_per_step": round(h2d / e2e_steps, 1), "d2h_bytes_per_step": round(d2h / e2e_steps, 1),
               "steps": e2e_steps,
               "path": "php_step + php_frame_begin/php_frame_wait (monitor rows, diagnostics, slice) per output "
                       f"interval ({oi} steps), page-locked host buffers, one frame in flight; wall clock over "
                       f"{e2e_steps} steps"}

    s = 4 if precision == "fp32" else 8
    c = census(cfg, medium)
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    sweeps = sweep_rooflines(prof, c, s, peak, ion_pass=prof["ion"]["launches"] > 0, dft_cells=nx * ny, dft_freqs=1)
    top = "step" if "step" in sweeps else "e_sweep"   # the dominant kernel
    traffic = None
    tf = ROOT / "profiles" / f"traffic_{args.workload}_{precision}.json"
    if tf.exists() and args.scale == 1.0:
        traffic = json.loads(tf.read_text()).get(f"{top}_dram_bytes_per_launch")
    launches_per_step = sum(v["launches"] for v in prof.values()) / max(1, prof[top]["launches"])
    return sim, cfg, {
        "value": value, "ms": ms_max, "V": V, "clocks": clocks.summary(), "prof": prof, "e2e": e2e,
        "launches_per_step": launches_per_step, "census": c, "roofline": {
            "bound": "hbm", "kernel": sweeps[top]["kernel"],
            "achieved": sweeps[top]["achieved"], "peak": peak, "unit": "GB/s", "frac": sweeps[top]["frac"],
            "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured" else "fallback 6650",
            "traffic": traffic, "algorithmic_bytes_per_launch": sweeps[top]["algorithmic_bytes_per_launch"],
            "avg_launch_ms": sweeps[top]["avg_launch_ms"], "sweeps": sweeps,
            "kernel_share": {k: round(v["ms"] / max(1e-9, sum(x["ms"] for x in prof.values())), 4)
                             for k, v in prof.items() if v["launches"]}}}


def run_largest(args, local):
    """The largest single domain (1024 x 1024 x 512 cells of 8 nm, 16-cell
    CPML, two-atom polar slab with anglex = 20 deg under a Drude-Lorentz tip,
    z-dipole Gaussian at 1400 cm^-1, FP64 running DFT at 1370, 1400 and
    1450 cm^-1 on the plane z = 66), FP64 and FP32: rate over --steps
    device-timed steps, roofline of both sweeps, and the FP32 error against
    the FP64 path on the z slice and the three DFT planes after
    --largest-steps steps.  One context per precision, each run from step 0
    to the same step count."""
    import torch
    from php_fdtd_b200 import Config, Simulation
    from php_fdtd_b200.workloads import C_CM
    n_total = max(args.largest_steps, args.warmup + 2 * args.steps + 40)
    case_dir = Path(args.case_dir or tempfile.gettempdir()) / "php_bench_cfg4_largest"
    case_dir.mkdir(parents=True, exist_ok=True)
    t_gen = time.perf_counter()
    make_case("cfg4", 1.0, n_total, case_dir)
    old = os.getcwd()
    os.chdir(case_dir)
    try:
        cfg = Config.load("case.cfg")
        medium = cfg.load_medium()
    finally:
        os.chdir(old)
    t_gen = time.perf_counter() - t_gen
    V = cfg.nx * cfg.ny * cfg.nz
    c = census(cfg, medium)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    wn = (1370.0, 1400.0, 1450.0)
    plane = cfg.output_slice_position + 1
    out, state = {}, {}
    for prec in ("fp64", "fp32"):
        holder = cfg.desc(medium, prec)
        holder.desc.device = local
        t_create = time.perf_counter()
        sim = Simulation(holder)
        t_create = time.perf_counter() - t_create
        pid = sim.dft_add("Ez", plane, [w * C_CM for w in wn], first_step=0, interval=1)
        sim.probe_set(cfg.monitor_x, cfg.monitor_y, cfg.monitor_z + 1, cfg.monitor_z)
        stream = torch.cuda.ExternalStream(sim.stream, device=torch.device("cuda", local))
        sim.step(args.warmup)
        sim.step(args.steps)          # records the timed region's graphs
        sim.probe_read()
        sim.sync()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clocks:
            ev0.record(stream)
            sim.step(args.steps)
            ev1.record(stream)
            ev1.synchronize()
        ms = ev0.elapsed_time(ev1)
        sim.probe_read()
        sim.profile(True)
        sim.step(20)
        prof = sim.profile_read()
        sim.profile(False)
        done = args.warmup + 2 * args.steps + 20
        while done < n_total:
            n = min(4096, n_total - done)
            sim.step(n)
            sim.probe_read()
            done += n
        sim.sync()
        # the configuration's own z slice (position 65: plane 66, the DFT plane)
        state[prec] = {"slice": sim.read_slice("Ez", "z", cfg.output_slice_position, f64=True),
                       "dft": sim.dft_read(pid)[0]}
        census_blocks = sim.block_census()
        sim.close()
        s = 4 if prec == "fp32" else 8
        out[prec] = {
            "value": round(V * args.steps / (ms * 1e-3) / 1e9, 4), "unit": "Gcell-updates/s",
            "ms_per_step": round(ms / args.steps, 4), "create_s": round(t_create, 2),
            "roofline": {"bound": "hbm", "peak": peak, "unit": "GB/s",
                         **sweep_rooflines(prof, c, s, peak, dft_cells=cfg.nx * cfg.ny, dft_freqs=len(wn))},
            "kernel_profile": prof, "blocks": census_blocks, "clocks": clocks.summary()}
    a, b = state["fp32"], state["fp64"]
    err = {"steps": n_total, "reference": "FP64 GPU path (same inputs, same steps)",
           "slice_rel_l2": float(np.linalg.norm(a["slice"] - b["slice"]) / max(np.linalg.norm(b["slice"]), 1e-300)),
           "slice": f"Ez, z plane {plane}"}
    for q, w in enumerate(wn):
        f32, f64 = a["dft"][q], b["dft"][q]
        wgt = np.abs(f64) ** 2
        dphi = np.angle(f32 * np.conj(f64))
        err[f"dft_{int(w)}cm-1"] = {
            "rel_l2": float(np.linalg.norm(f32 - f64) / np.linalg.norm(f64)),
            "amplitude_rel_l2": float(np.linalg.norm(np.abs(f32) - np.abs(f64)) / np.linalg.norm(f64)),
            "phase_rms_rad": float(math.sqrt(np.sum(wgt * dphi ** 2) / np.sum(wgt)))}
    return {
        "workload": "cfg4_largest_1024x1024x512", "grid": [cfg.nx, cfg.ny, cfg.nz], "cells": V,
        "reference_form": REFERENCE_FORM,
        "atom_cells": c["atom_cells"], "ade_cells": c["ade_cells"], "inputs_s": round(t_gen, 1),
        "fp64": out["fp64"], "fp32": out["fp32"],
        "fp32_speedup_vs_fp64": round(out["fp32"]["value"] / out["fp64"]["value"], 3),
        "error_fp32_vs_fp64": err,
        "cpu_baseline": largest_reference_sample(case_dir / "case.cfg", cfg.nz, V) if not args.no_cpu_baseline else None,
    }


def largest_reference_sample(case_cfg: Path, nz: int, V: int, steps: int = 3):
    """The reference on the largest domain: a few time steps on every host
    core (its own loop timer), extrapolated per step.  It needs about 75 GB
    of host memory (fields, z-psi, per-cell pointer arrays, r/v of 67 M atom
    cells); skipped with the reason when the host has less."""
    need = 110 * 10 ** 9
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except ImportError:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    if avail < need:
        return {"value": None, "unit": "Gcell-updates/s", "kind": "reference",
                "sample": f"skipped: the reference needs about 75 GB of host memory here, {avail / 1e9:.0f} GB available"}
    ranks = reference_ranks(nz)
    t0 = time.perf_counter()
    res, err = reference_rate(case_cfg, steps, ranks, timeout=1500)
    wall = time.perf_counter() - t0
    if res is None:
        return {"value": None, "unit": "Gcell-updates/s", "kind": "reference", "sample": err}
    return {"value": round(V * steps / res["loop_s"] / 1e9, 6), "unit": "Gcell-updates/s", "cores": res["ranks"],
            "kind": "reference", "extrapolated": True,
            "sample": f"{steps} time steps of the full 1024x1024x512 domain, reference solver {res['exe']} "
                      f"({res['ranks']} MPI ranks as processes through the shared-memory MPI stand-in), its own loop "
                      f"timer, rate per step extrapolated to the workload; set-up and run {wall:.0f} s wall; "
                      f"CPU {cpu_model()}"}


def run_other_configs(args, ws, rank, local):
    """The other single-domain workloads at their full size: config 0 (96^3,
    two-atom slab) and config 2 (512 x 512 x 256, 16-atom lattice through the
    ion pass), FP64 and FP32, device-timed over --steps steps; for config 2
    the ion pass's roofline beside the sweeps'."""
    import copy
    out = {}
    for wl in ("cfg0", "cfg2"):
        entry = {}
        for prec in ("fp64", "fp32"):
            a = copy.copy(args)
            a.workload, a.no_e2e, a.z_chunk = wl, True, 0
            # the 96^3 step takes ~0.06 ms: time at least 400 of its 2000 steps so that
            # the fixed cost of a graph launch does not set the rate
            if wl == "cfg0":
                a.steps = max(args.steps, 400)
            sim, cfg, r = run_ours(a, ws, rank, local, prec)
            sim.close()
            prof = r["prof"]
            e = {"value": round(r["value"], 4), "unit": "Gcell-updates/s", "steps": a.steps,
                 "ms_per_step": round(r["ms"] / a.steps, 5),
                 "kernel_ms": {k: round(v["ms"] / max(1, v["launches"]), 5) for k, v in prof.items() if v["launches"]},
                 **{f"{k}_frac": v["frac"] for k, v in r["roofline"]["sweeps"].items()}}
            c = r["census"]
            if prof["ion"]["launches"]:
                s = 4 if prec == "fp32" else 8
                ion_bytes = s * (c["atom_words"] + 6 * c["atom_cells"]) + 13 * c["atom_cells"]
                ion_ms = prof["ion"]["ms"] / prof["ion"]["launches"]
                e["ion_pass"] = {"achieved": round(ion_bytes / (ion_ms * 1e-3) / 1e9, 1), "unit": "GB/s",
                                 "frac": round(ion_bytes / (ion_ms * 1e-3) / 1e9 / r["roofline"]["peak"], 4),
                                 "avg_launch_ms": round(ion_ms, 4), "algorithmic_bytes_per_launch": int(ion_bytes)}
            entry[prec] = e
        entry["fp32_speedup_vs_fp64"] = round(entry["fp32"]["value"] / entry["fp64"]["value"], 3)
        from php_fdtd_b200.workloads import CONFIG_NAMES
        entry["workload"] = CONFIG_NAMES[WORKLOADS[wl]]
        entry["grid"] = [cfg.nx, cfg.ny, cfg.nz]
        out[wl] = entry
    return out


def run_slabs(args, local, nslabs: int):
    """The default workload split into nslabs z slabs on one GPU (LocalSlabs:
    each step in parts on two streams per slab, halo planes copied device to
    device, no graphs): wall-clock rate over --steps steps."""
    import torch
    from php_fdtd_b200 import Config
    from php_fdtd_b200.slab import LocalSlabs
    case_dir = Path(args.case_dir or tempfile.gettempdir()) / f"php_bench_{args.workload}_{args.scale}_slabs"
    case_dir.mkdir(parents=True, exist_ok=True)
    make_case(args.workload, args.scale, args.warmup + args.steps + 8, case_dir)
    old = os.getcwd()
    os.chdir(case_dir)
    try:
        cfg = Config.load("case.cfg")
        medium = cfg.load_medium()
    finally:
        os.chdir(old)
    holder = cfg.desc(medium, args.precision)
    holder.desc.device = local
    slabs = LocalSlabs(holder, nslabs, devices=(local,))
    slabs.step(args.warmup)
    slabs.sync()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    slabs.step(args.steps)
    slabs.sync()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    slabs.close()
    V = cfg.nx * cfg.ny * cfg.nz
    return {"metric": f"Gcell-updates/s, {nslabs} z slabs on one GPU, {args.precision.upper()} path",
            "value": round(V * args.steps / dt / 1e9, 4), "unit": "Gcell-updates/s", "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 4), "timer": "wall clock",
            "config": {"workload": workload_name(args), "slabs": [n for _, n in slabs.ranges]}}


def accuracy_vs_fp64(args, local, steps: int):
    """Error of the FP32 path against the FP64 path on the workload after
    `steps` time steps: relative L2 of (Ex, Ey, Ez) over the volume, and of
    the running-DFT near-field plane (complex, amplitude, and the
    amplitude-weighted RMS phase difference).  The FP64 path is the one that
    matches the reference to 1e-10 on the parity cases."""
    from php_fdtd_b200 import Config, Simulation
    case_dir = Path(args.case_dir or tempfile.gettempdir()) / f"php_bench_{args.workload}_{args.scale}_r0"
    old = os.getcwd()
    os.chdir(case_dir)
    try:
        cfg = Config.load("case.cfg")
        medium = cfg.load_medium()
    finally:
        os.chdir(old)
    out = {}
    for prec in ("fp64", "fp32"):
        holder = cfg.desc(medium, prec)
        holder.desc.device = local
        with Simulation(holder) as sim:
            pid = sim.dft_add("Ez", cfg.output_slice_position + 1, [cfg.unique_source_frequency])
            sim.step(steps)
            sim.sync()
            out[prec] = {"E": [sim.read_volume(c) for c in ("Ex", "Ey", "Ez")], "dft": sim.dft_read(pid)[0][0]}
    num = sum(float(np.sum((a - b) ** 2)) for a, b in zip(out["fp32"]["E"], out["fp64"]["E"]))
    den = sum(float(np.sum(b ** 2)) for b in out["fp64"]["E"])
    f32, f64 = out["fp32"]["dft"], out["fp64"]["dft"]
    w = np.abs(f64) ** 2
    dphi = np.angle(f32 * np.conj(f64))
    return {
        "steps": steps, "reference": "FP64 GPU path (same inputs)",
        "field_rel_l2": math.sqrt(num / den) if den > 0 else None,
        "nearfield_rel_l2": float(np.linalg.norm(f32 - f64) / np.linalg.norm(f64)),
        "nearfield_amplitude_rel_l2": float(np.linalg.norm(np.abs(f32) - np.abs(f64)) / np.linalg.norm(f64)),
        "nearfield_phase_rms_rad": float(math.sqrt(np.sum(w * dphi ** 2) / np.sum(w))),
        "targets": {"field_rel_l2": 1e-4, "nearfield": 1e-3},
    }


# ------------------------------------------------------ reference / baseline


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def reference_ranks(nz: int) -> int:
    """MPI ranks for the reference on this host: every core it may use, at
    most one per two z planes (the reference splits z across ranks)."""
    return max(1, min(host_cores(), nz // 2))


def reference_rate(case_cfg: Path, steps: int, ranks: int = 1, timeout: int = 900):
    """Runs the reference solver (compiled from its own sources with its
    release flags) on the workload for `steps` time steps, as `ranks` MPI
    ranks (forked processes through the shared-memory MPI stand-in); its own
    loop timer on rank 0 (fdtd.c:3110, 3915) gives the throughput."""
    from oracle import reference_binary
    exe = reference_binary("mp")
    env = dict(os.environ, PHP_MPI_NP=str(ranks))
    if not exe.exists():
        exe, ranks = reference_binary("fast"), 1
    if not exe.exists():
        return None, "reference binary not built (make -C oracle ref)"
    case_dir = case_cfg.parent
    text = case_cfg.read_text()
    text = re.sub(r"(?m)^tsteps = \d+", f"tsteps = {steps}", text)
    text = re.sub(r"(?m)^output_interval = \d+", f"output_interval = {max(1, steps)}", text)
    run_dir = case_dir / "refrun"
    run_dir.mkdir(exist_ok=True)
    for p in case_dir.iterdir():
        if p.is_file() and p.name not in ("case.cfg",):
            dst = run_dir / p.name
            if not dst.exists():
                os.symlink(p, dst)
    (run_dir / "case.cfg").write_text(text)
    t0 = time.perf_counter()
    pr = subprocess.run([str(exe), "case.cfg"], cwd=run_dir, capture_output=True, text=True, timeout=timeout, env=env)
    wall = time.perf_counter() - t0
    m = re.search(r"Simulation completed in ([\d.]+) seconds", pr.stdout)
    if pr.returncode != 0 or not m:
        return None, f"reference run failed rc={pr.returncode}: {pr.stdout[-300:]} {pr.stderr[-300:]}"
    return {"loop_s": float(m.group(1)), "wall_s": wall, "steps": steps, "exe": exe.name, "ranks": ranks}, None


def cpu_model():
    try:
        for l in open("/proc/cpuinfo"):
            if l.startswith("model name"):
                return l.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def ref_sample_steps(V: int, k: int, ranks: int = 1) -> int:
    # about 2e8 cell updates per rank (~10-30 s of the reference's loop)
    return int(max(2, min(k, round(2e8 * ranks / V))))


def run_reference_arm(args, ws, rank):
    if rank != 0:
        return
    if args.workload == "cfg3":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving mode (one simulation per "
                          "mpirun); the serving line carries its sequential plain-FP64 baseline"}))
        return
    case_dir = Path(args.case_dir or tempfile.gettempdir()) / f"php_bench_{args.workload}_{args.scale}_ref"
    case_dir.mkdir(parents=True, exist_ok=True)
    cfg_path = make_case(args.workload, args.scale, 10, case_dir)
    from php_fdtd_b200.workloads import baseline_case
    spec = baseline_case(WORKLOADS[args.workload], scale=args.scale)
    V = spec.nx * spec.ny * spec.nz
    ranks = reference_ranks(spec.nz)
    steps = ref_sample_steps(V, args.steps, ranks)
    # warm-up sample (page cache, allocator) then the timed sample
    if args.warmup > 0:
        reference_rate(cfg_path, 1, ranks)
    res, err = reference_rate(cfg_path, steps, ranks)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    rate = V * steps / res["loop_s"] / 1e9
    line = {
        "metric": metric_name(args), "value": round(rate, 6), "unit": "Gcell-updates/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(res["loop_s"] / steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": workload_name(args), "grid": [spec.nx, spec.ny, spec.nz], "cells": V,
                   "reference_form": REFERENCE_FORM},
        "cpu_baseline": {"value": round(rate, 6), "unit": "Gcell-updates/s", "cores": res["ranks"], "kind": "reference",
                         "sample": f"{steps} time steps of the full {spec.nx}x{spec.ny}x{spec.nz} domain, reference "
                                   f"solver ({res['exe']}, -Ofast -funroll-loops, {res['ranks']} MPI ranks as processes "
                                   f"through the shared-memory MPI stand-in, {host_cores()} host cores usable), timed "
                                   f"by its own loop timer; CPU {cpu_model()}"},
        "e2e": {"value": round(rate, 6), "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def metric_name(args):
    return f"Gcell-updates/s, {args.precision.upper()} path"


def workload_name(args):
    from php_fdtd_b200.workloads import CONFIG_NAMES
    return CONFIG_NAMES[WORKLOADS[args.workload]] + ("" if args.scale == 1.0 else f" (scale {args.scale})")


def run_serving(args, ws, rank, local):
    """cfg3: the request stream submitted at its Poisson arrival times to the
    serving loop (FP32 mixed kernels, 150 GB budget); latency = completion
    minus submission on the server clock.  Baseline: the same requests run
    one after another with the plain FP64 path, timed on a sample and
    extrapolated by cell-steps (a + b * cells * steps fitted on the sample)."""
    from php_fdtd_b200 import Simulation
    from php_fdtd_b200.serving import DftSpec, Server
    from php_fdtd_b200.workloads import request_desc, serving_requests
    reqs = serving_requests(args.requests, seed=rank)
    built = [request_desc(r, "fp32", device=local) for r in reqs]  # host-side inputs, before the clock
    cells = np.array([r["grid"][0] * r["grid"][1] * r["grid"][2] for r in reqs], dtype=np.float64)
    steps = np.array([r["steps"] for r in reqs], dtype=np.float64)
    # the baseline sample: requests at evenly spaced ranks of their work
    # (cells x steps), so that it spans the stream's sizes
    by_work = np.argsort(cells * steps, kind="stable")
    sample = sorted(set(by_work[np.linspace(0, len(reqs) - 1, min(args.baseline_sample, len(reqs))).round()
                                .astype(int)].tolist()))
    served = {}
    infos = {}
    done_evt = threading.Event()
    budget = 150 * 10 ** 9

    with ClockSampler(local) as clocks, Server(memory_budget=budget, device=local, max_active=args.max_active) as srv:
        def collector():
            while len(infos) < len(reqs):
                for info in srv.poll(timeout_ms=200):
                    q = info["tag"]
                    infos[q] = info
                    if q in sample and info["status"] == 0:
                        served[q] = srv.fetch_dft(info)
                    else:
                        srv.release(info["job"])
            done_evt.set()
        th = threading.Thread(target=collector, daemon=True)
        th.start()
        t0 = srv.clock()
        for q, (r, (holder, dft)) in enumerate(zip(reqs, built)):
            wait = t0 + r["arrival"] - srv.clock()
            if wait > 0:
                time.sleep(wait)
            srv.submit(holder, r["steps"], DftSpec(dft["component"], dft["z_plane"], dft["freqs"]), tag=q)
        done_evt.wait()
        th.join()
        stats = srv.stats()
    bad = [i for i in infos.values() if i["status"] != 0]
    lat = np.array([infos[q]["t_done"] - infos[q]["t_submit"] for q in range(len(reqs))])
    queue_wait = np.array([infos[q]["t_admit"] - infos[q]["t_submit"] for q in range(len(reqs))])
    build = np.array([infos[q]["t_start"] - infos[q]["t_admit"] for q in range(len(reqs))])
    t_first = min(i["t_submit"] for i in infos.values())
    t_last = max(i["t_done"] for i in infos.values())
    makespan = t_last - t_first
    sims_h = len(reqs) / makespan * 3600.0

    # baselines on the sample: plain FP64 alone (timed) and FP32 alone (identity check)
    seq_t, err, same = [], [], 0
    for q in sample:
        h64, dft = request_desc(reqs[q], "fp64", device=local)
        t1 = time.perf_counter()
        with Simulation(h64) as sim:
            pid = sim.dft_add(dft["component"], dft["z_plane"], dft["freqs"])
            sim.step(reqs[q]["steps"])
            f64 = sim.dft_read(pid)[0]
        seq_t.append(time.perf_counter() - t1)
        with Simulation(built[q][0]) as sim:
            pid = sim.dft_add(dft["component"], dft["z_plane"], dft["freqs"])
            sim.step(reqs[q]["steps"])
            f32 = sim.dft_read(pid)[0]
        if q in served:
            same += int(np.array_equal(served[q], f32))
            err.append(float(np.linalg.norm(served[q] - f64) / max(np.linalg.norm(f64), 1e-300)))
    cs = cells * steps
    A = np.vstack([np.ones(len(sample)), cs[sample]]).T
    coef, *_ = np.linalg.lstsq(A, np.array(seq_t), rcond=None)
    seq_total = float(np.sum(np.maximum(coef[0] + coef[1] * cs, 0.0)))
    seq_sims_h = len(reqs) / seq_total * 3600.0
    # the sample itself, timed: its requests one after another in plain FP64
    sample_sims_h = len(sample) / float(np.sum(seq_t)) * 3600.0
    sample_work = float(np.mean(cs[sample]) / np.mean(cs))
    h2d = float(np.sum(cells) * 5 + np.sum(steps) * 8 * 4)
    d2h = float(sum(16 * r["grid"][0] * r["grid"][1] for r in reqs))
    line = {
        "metric": "sims/h, serving loop (FP32 mixed, continuous batching)", "value": round(sims_h, 2), "unit": "sims/h",
        "n_gpus": ws, "steps": int(steps.sum()), "warmup": 0, "ms_per_step": round(makespan / steps.sum() * 1e3, 6),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "ours",
        "config": {"workload": "cfg3_serving_request stream", "requests": len(reqs), "arrivals": "Poisson 4/s",
                   "reference_form": REFERENCE_FORM,
                   "edges": "log-uniform 64-192 per axis", "steps": "3000-12000", "pml": 8,
                   "memory_budget_bytes": budget, "max_active": args.max_active, "chunk_steps": 256},
        "latency_s": {"p50": round(float(np.percentile(lat, 50)), 3), "p95": round(float(np.percentile(lat, 95)), 3),
                      "p99": round(float(np.percentile(lat, 99)), 3), "max": round(float(lat.max()), 3),
                      "queue_wait_p50": round(float(np.percentile(queue_wait, 50)), 3),
                      "build_p50": round(float(np.percentile(build, 50)), 4),
                      "build_p99": round(float(np.percentile(build, 99)), 4)},
        "makespan_s": round(makespan, 3), "gcell_updates_per_s": round(float(cs.sum()) / makespan / 1e9, 3),
        "failed": len(bad), "server": stats,
        "baseline_sequential_fp64": {"sims_per_h": round(seq_sims_h, 2), "sample": len(sample),
                                     "method": "the sample's requests run one after another in plain FP64 "
                                               "(timed); the stream's total from a + b * cells * steps "
                                               "fitted on them",
                                     "fit_s": [float(coef[0]), float(coef[1])],
                                     "sample_sims_per_h": round(sample_sims_h, 2),
                                     "sample_mean_work_vs_stream": round(sample_work, 3),
                                     "speedup": round(sims_h / seq_sims_h, 3)},
        "results": {"identical_to_alone": f"{same}/{len(served)}",
                    "nearfield_rel_l2_vs_fp64_max": round(max(err), 9) if err else None,
                    "target": 1e-3},
        "e2e": {"value": round(sims_h, 2), "unit": "sims/h", "h2d_bytes_per_step": round(h2d / steps.sum(), 1),
                "d2h_bytes_per_step": round(d2h / steps.sum(), 3),
                "path": "php_batch_submit host descriptions -> php_batch_poll/fetch_dft, whole stream timed"},
        "clocks": clocks.summary(),
        # per job step: the two sweeps (the one-launch step with PHP_FUSED=1), which also sample
        # the running DFT (a launch of its own with PHP_DFT_FOLD=0)
        "gpu_launches": int(steps.sum()) * ((1 if os.environ.get("PHP_FUSED") == "1" else 2) +
                                            (1 if os.environ.get("PHP_DFT_FOLD") == "0" else 0)),
    }
    return line


def main():
    args = parse()
    ws, rank, local = dist_init()
    if args.impl == "reference":
        run_reference_arm(args, ws, rank)
        barrier(ws)
        return
    if args.workload == "cfg3":
        line = run_serving(args, ws, rank, local)
        if rank == 0:
            print(json.dumps(line))
        barrier(ws)
        return
    if args.slabs > 0:
        print(json.dumps(run_slabs(args, local, args.slabs)))
        return
    if args.concurrency:
        print(json.dumps(run_concurrency(args, local)))
        return
    sim, cfg, r = run_ours(args, ws, rank, local, args.precision)
    sim.close()
    mixed = None
    if args.precision == "fp64" and not args.no_mixed:
        sim32, _, r32 = run_ours(args, ws, rank, local, "fp32")
        sim32.close()
        mixed = {"precision": "fp32", "value": round(r32["value"], 4), "unit": "Gcell-updates/s",
                 "ms_per_step": round(r32["ms"] / args.steps, 5), "speedup_vs_fp64": round(r32["value"] / r["value"], 3),
                 "e2e": r32["e2e"], "roofline": r32["roofline"], "clocks": r32["clocks"], "kernel_profile": r32["prof"]}
        from php_fdtd_b200.workloads import baseline_case
        acc_steps = args.acc_steps if args.acc_steps is not None else baseline_case(WORKLOADS[args.workload]).tsteps
        if acc_steps > 0 and ws == 1:
            mixed["error_vs_fp64"] = accuracy_vs_fp64(args, local, acc_steps)
    largest = serving = configs = None
    if args.precision == "fp64" and args.workload == "cfg1" and args.scale == 1.0 and ws == 1 and not args.no_configs:
        configs = run_other_configs(args, ws, rank, local)
    if args.precision == "fp64" and args.workload == "cfg1" and args.scale == 1.0 and ws == 1 and not args.no_largest:
        largest = run_largest(args, local)
    if args.precision == "fp64" and args.workload == "cfg1" and ws == 1 and not args.no_serving:
        sv = run_serving(args, ws, rank, local)
        serving = {k: sv[k] for k in ("metric", "value", "unit", "latency_s", "makespan_s", "gcell_updates_per_s",
                                      "failed", "baseline_sequential_fp64", "results", "e2e", "clocks")}
        serving["config"] = sv["config"]
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and ws == 1:
            case_dir = Path(args.case_dir or tempfile.gettempdir()) / f"php_bench_{args.workload}_{args.scale}_r{rank}"
            ranks = reference_ranks(cfg.nz)
            steps = ref_sample_steps(r["V"], args.steps, ranks)
            res, err = reference_rate(case_dir / "case.cfg", steps, ranks)
            if res:
                cpu = {"value": round(r["V"] * steps / res["loop_s"] / 1e9, 6), "unit": "Gcell-updates/s",
                       "cores": res["ranks"], "kind": "reference",
                       "sample": f"{steps} time steps of the full domain, reference solver {res['exe']} "
                                 f"({res['ranks']} MPI ranks as processes through the shared-memory MPI stand-in, its "
                                 f"own loop timer); CPU {cpu_model()}"}
            else:
                cpu = {"value": None, "unit": "Gcell-updates/s", "cores": 1, "kind": "reference", "sample": err}
        line = {
            "metric": metric_name(args), "value": round(r["value"], 4), "unit": "Gcell-updates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(r["ms"] / args.steps, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp64": "f64", "fp32": "f32", "fp64-strict": "f64"}[args.precision], "data": "synthetic",
            "config": {"workload": workload_name(args), "grid": [cfg.nx, cfg.ny, cfg.nz], "cells": r["V"],
                       "precision": args.precision, "parallelism": f"replicas x{ws}" if ws > 1 else "single domain",
                       "l2": "state 9 fields x cells > L2 (126 MB); no flush needed",
                       "per_step": ("one-launch step (H, D, sources, E, ADE) + monitor probe + running DFT (1 plane)"
                                    if "step" in r["roofline"]["sweeps"] else
                                    "H sweep + fused D/source/E/ADE sweep + monitor probe + running DFT (1 plane)"),
                       "reference_form": REFERENCE_FORM},
            "hbm_gbs": r["roofline"]["achieved"],
            "roofline": r["roofline"], "cpu_baseline": cpu, "e2e": r["e2e"], "clocks": r["clocks"],
            "gpu_launches": int(round(r["launches_per_step"] * args.steps)),
            "kernel_profile": r["prof"],
        }
        if mixed is not None:
            line["mixed"] = mixed
        if largest is not None:
            line["largest"] = largest
        if serving is not None:
            line["serving"] = serving
        if configs is not None:
            line["configs"] = configs
        print(json.dumps(line))
    barrier(ws)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
