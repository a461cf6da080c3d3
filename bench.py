"""Benchmark: Coulomb shift+force evaluations per second at 32k atoms (B200).

Workload: 10,923 rigid 3-site waters = 32,769 charges at 1.0 g/cm^3 in a
68.91 A cubic cell (seeded synthetic input, converted to Bohr).  One step is one
shift+force evaluation of the reference's fast Ewald method
(ewald_potential_force with force, src/dftbp/extlibs/fftewald/fft/ewald_fft_3d.f90:36-134):
parameters re-derived from the charges, real-space pair sum, adjoint NFFT, four
forward NFFTs (potential and ik force), self term.

Our arm (default):
  value   plain FP64 form at tol 1e-10 (the reference chain: 280^3 grid, m=12),
          inputs and outputs resident in HBM, device-timed with CUDA events on
          the launching stream; L2 flushed between steps (flush not timed).
  e2e     the same through the C ABI with pinned host buffers: every step copies
          positions and charges in and potential and force out.
  fp64_ad the plain form with forces by window differentiation (one inverse
          FFT instead of four), with its deviation from the i k forces.
  mixed   the mixed-precision form (FP32 stencils, FFT and pair terms, FP64
          accumulation) with force scheme and parameters from the library's
          autotuner (ewg_tune) for an RMS force error of at most 5e-7 against
          the FP64 form, with its measured error.
  roofline, cpu_baseline, clocks, gpu_launches as the measurement contract asks.
Reference arm (--impl reference): the CPU restatement of the reference's own
algorithm (oracle/), all host threads, one full evaluation per step.

Multi-GPU (torchrun): the single cell does not shard; every rank runs its own
replica ("replicas only"), value = all ranks' evaluations / max-over-ranks time.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "dftb_fast-ewald_3d_b200")
ORACLE = os.path.join(ROOT, "oracle")
for _p in (PKG, ORACLE):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import workloads  # noqa: E402

METRIC = "Coulomb shift+force evals/s at 32k atoms, mixed vs FP64; rel. err vs FP64"
TOL_FP64 = 1e-10
TOL_MIXED = 1e-7
MIXED_TARGET = 1e-6  # mixed form: RMS relative force error <= MIXED_TARGET / 2 vs FP64
L2_FLUSH_BYTES = 256 << 20


# Single-cell workloads: name -> (generator, label).  C3 is the headline; the
# others fill the per-configuration table (seeded synthetic inputs, Bohr).
SINGLE_CELL = {
    "c3": (lambda: workloads.c3_water_32k(), "water_32769_atoms_68.91A_tol1e-10"),
    "c1": (lambda: workloads.c1_small_cubic(), "random_64_atoms_12A_cubic_tol1e-10"),
    "c2": (lambda: workloads.c2_random_4096(), "random_4096_atoms_35A_cubic_tol1e-10"),
    "c5": (lambda: workloads.c5_rock_salt_216k(), "rock_salt_216000_sites_169.2A_tol1e-10"),
}


def metric_for(name, natoms):
    if name == "c3":
        return METRIC
    return f"Coulomb shift+force evals/s at {natoms} atoms ({name}), mixed vs FP64; rel. err vs FP64"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        loaded = [x for x in sm if smax is None or x > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# algorithmic bytes per stage launch (one evaluation), for the roofline
# ---------------------------------------------------------------------------
def stage_bytes(params, natoms, real_bytes, nc=4):
    M = params["n_modes"]
    n = [2 * m for m in M]
    H = [m - m // 2 for m in M]
    K1, K2, K3 = H[0] + 1, 2 * H[1] + 1, 2 * H[2] + 1
    s, c = real_bytes, 2 * real_bytes
    G = n[0] * n[1] * n[2] * s
    # force grids in the fractional-derivative basis: the z pass writes 2
    # spectra, the y inverse 3, the x C2R 4 real grids
    nz, ny = (2, 3) if nc == 4 else (1, 1)
    return {
        "spread": G,
        "fft_x_r2c": G + n[1] * n[2] * K1 * c,
        "fft_y_fwd": n[2] * n[1] * K1 * c + n[2] * K2 * K1 * c,
        "fft_z_influence": n[2] * K2 * K1 * c * (1 + nz),
        "fft_y_inv": nz * n[2] * K2 * K1 * c + ny * n[2] * n[1] * K1 * c,
        "fft_x_c2r": ny * n[2] * n[1] * K1 * c + nc * G,
        "gather": nc * G + natoms * (8 * 4 + 8 * 4),
    }


def stage_flops(params, natoms, nc=4):
    """Algorithmic FP64 flops of the tensor-core stages: one multiply-add per
    stencil point and component (gather: nc components; spread: one)."""
    w = (2 * params["window_cutoff"] + 1) ** 3
    return {"spread": 2 * natoms * w, "gather": 2 * natoms * w * nc}


# DRAM bytes (read + write) per launch from one ncu capture of the 32,769-atom
# workload (profiles/c3_water_32k_fp64_top_kernels.md), keyed by (workload, real
# bytes, grids through the inverse passes and the gather, stage); other
# workloads report null.
DRAM_TRAFFIC = {
    ("c3", 8, 4, "gather"): 746.37e6 + 62.96e6,
}


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# reference arm and CPU baseline: the oracle's port of the reference algorithm
# ---------------------------------------------------------------------------
def cpu_evals(pos, q, lat, tol, steps, warmup, threads):
    import oracle

    oracle.build()
    oracle.set_threads(threads)
    for _ in range(warmup):
        oracle.fft_potential_force(pos, q, lat, tol)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        oracle.fft_potential_force(pos, q, lat, tol)
        times.append(time.perf_counter() - t0)
    cpu_evals.split = oracle.last_stage_seconds()  # of the last evaluation
    return times


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    if args.workload not in SINGLE_CELL:
        print(json.dumps({"impl": "reference", "unavailable":
                          f"the reference arm times single-cell workloads only, not {args.workload}"}))
        return 0
    gen, label = SINGLE_CELL[args.workload]
    pos, q, lat = gen()
    threads = os.cpu_count() or 1
    times = cpu_evals(pos, q, lat, TOL_FP64, args.steps, args.warmup, threads)
    total = sum(times)
    value = args.steps / total
    line = {
        "metric": metric_for(args.workload, len(q)), "value": value, "unit": "evals/s",
        "impl": "reference", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": label, "natoms": len(q), "tol": TOL_FP64},
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full {args.workload} shift+force evaluations (oracle/ C++ "
                                   f"restatement, OpenMP, project FFT in place of FFTW)",
                         "split_s": cpu_evals.split},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
class Arm:
    """One precision form on one device: device-resident and end-to-end timing."""

    def __init__(self, eb, torch, device, precision, tol, pos, q, lat, scheme=None, ov=None,
                 want_force=True):
        self.eb, self.torch = eb, torch
        self.tol = tol
        self.want_force = want_force  # False: SCC-style shift (potential) only
        self.ov = dict(ov or {})
        self.ctx = eb.Context(device, precision)
        if scheme is not None:
            self.ctx.set_force_scheme(scheme)
        self.cfg = (pos, q, lat)
        self.shape = None
        # A dedicated (non-default) stream: the library launches on it and the
        # CUDA events that time the steps are recorded on it.
        # High priority: the library's real-space side stream (lowest priority)
        # then fills the gaps between the mesh kernels.
        self.stream = torch.cuda.Stream(device=device, priority=-1)
        self.ctx.set_stream(self.stream.cuda_stream)
        dev = f"cuda:{device}"
        self.n = len(q)
        self.lat = np.asfortranarray(lat)
        self.x = torch.tensor(pos, dtype=torch.float64, device=dev).contiguous()
        self.q = torch.tensor(q, dtype=torch.float64, device=dev).contiguous()
        self.pot = torch.empty(self.n, dtype=torch.float64, device=dev)
        self.force = torch.empty((self.n, 3), dtype=torch.float64, device=dev)
        self.flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
        # pinned host buffers for the end-to-end path (Fortran positions(N,3))
        self.h_pos = torch.empty((3, self.n), dtype=torch.float64, pin_memory=True).numpy()
        self.h_pos[:] = np.asarray(pos).T
        self.h_q = torch.empty(self.n, dtype=torch.float64, pin_memory=True).numpy()
        self.h_q[:] = q
        self.h_pot = torch.empty(self.n, dtype=torch.float64, pin_memory=True).numpy()
        self.h_force = torch.empty((self.n, 3), dtype=torch.float64, pin_memory=True).numpy()
        torch.cuda.synchronize()

    def tune_shapes(self):
        """The library's kernel-shape autotuner on this arm's configuration
        (untimed, once): later evaluations of the bucket run its choice."""
        pos, q, lat = self.cfg
        shape, (ms0, ms1) = self.ctx.tune_kernels(pos, q, lat, self.tol, self.want_force, **self.ov)
        self.shape = dict(shape, default_ms=ms0, tuned_ms=ms1)
        return self.shape

    def step_device(self):
        self.ctx.potential_force_device(self.x, self.q, self.lat, self.tol, self.pot,
                                        self.force if self.want_force else None, **self.ov)

    def step_e2e(self):
        L = self.eb.lib()
        dp = C.POINTER(C.c_double)
        ov = self.eb._overrides(**self.ov)
        rc = L.ewg_potential_force(self.ctx.handle, self.n, self.h_pos.ctypes.data_as(dp),
                                   self.h_q.ctypes.data_as(dp), self.lat.ctypes.data_as(dp),
                                   float(self.tol), self.h_pot.ctypes.data_as(dp),
                                   self.h_force.ctypes.data_as(dp) if self.want_force else None,
                                   C.byref(ov))
        if rc:
            raise self.eb.EwaldError(rc, self.eb.status_string(rc))

    def time_device(self, steps, warmup, profile=False):
        torch = self.torch
        for _ in range(warmup):
            self.step_device()
        if profile:
            self.ctx.stage_times(reset=True)
            self.ctx.set_profiling(True)
        launches0 = self.ctx.kernel_launches
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        torch.cuda.synchronize()
        for i in range(steps):
            with torch.cuda.stream(self.stream):
                self.flush.zero_()  # L2 flush, outside the timed interval
            evs[i][0].record(self.stream)
            self.step_device()
            evs[i][1].record(self.stream)
        torch.cuda.synchronize()
        ms = [a.elapsed_time(b) for a, b in evs]
        launches = self.ctx.kernel_launches - launches0
        stages = None
        if profile:
            stages = self.ctx.stage_times(reset=True)
            self.ctx.set_profiling(False)
        return ms, launches, stages

    def time_e2e(self, steps, warmup):
        for _ in range(warmup):
            self.step_e2e()
        self.torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            self.step_e2e()
        self.torch.cuda.synchronize()
        return time.perf_counter() - t0


def run_batched(args, eb, torch, device, dist, ws, rank):
    """Batched cells through ewg_batch_potential_force from host arrays (copies
    inside the timed region), every stage of all cells in one segmented launch
    (the default; the one-lane figure, cells one after another, beside it).  Weak scaling: the job
    holds 256 cells (c4) or 8 boxes (c3_batch) per GPU, partitioned over the
    ranks by sharding.shard_of (LPT on the cost model; no collective in the
    data path), and each rank times its own share with CUDA events on the
    library's stream; the step time is the max over ranks.  The one gather of
    the results (sharding.gather_results) follows the timed region.
    c4:       independent triclinic cells (50-2000 atoms each), reference chain
              per cell (FP64 tol 1e-10, mixed tol 1e-7); N = 1 is C4's 256 cells;
    c3_batch: independent 32,769-atom water boxes (seeds 3, 4, ...); FP64 with the
              reference chain at tol 1e-10, mixed with the autotuner's parameters
              and force scheme for the first box applied to all."""
    import sharding

    if args.workload == "c4":
        cells = workloads.c4_batched_cells(256 * ws)
        metric = "C4 batched cells: cell shift+force evals/s (256 cells per GPU, 50-2000 atoms)"
        label = "c4_256_triclinic_cells_per_gpu"
    else:
        cells = [workloads.water_box(10923, seed=3 + k) for k in range(8 * ws)]
        metric = "batched 32k-atom cells: shift+force evals/s (8 water boxes of 32,769 atoms per GPU)"
        label = "c3_batch_8_water_32769_per_gpu"
    natoms = sum(len(c[1]) for c in cells)
    mine = sharding.shard_of(cells, TOL_FP64, sharding.library_parameters, rank, ws)
    my_cells = [cells[i] for i in mine]

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def maxrank(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    out = {}
    gather_s = None
    for name, prec, tol in (("fp64", eb.FP64, TOL_FP64), ("mixed", eb.MIXED, TOL_MIXED)):
        ctx = eb.Context(device, prec)
        stream = torch.cuda.Stream(device=device)
        ctx.set_stream(stream.cuda_stream)
        kw, note = {}, None
        if name == "mixed" and args.workload == "c3_batch":
            kw, scheme, rep = ctx.tune(*cells[0], MIXED_TARGET)
            ctx.set_force_scheme(scheme)
            note = {"force_scheme": "ik" if scheme == eb.FORCE_IK else "window differentiation",
                    "r_cut_bohr": kw["r_cut_in"], "window_cutoff": kw["windowCutoff_in"],
                    "tuner_force_rms": rep["force_rms"]}
        res = {}
        launches = 0
        # Host arrays packed once in the C ABI's layout, page-locked; each step is
        # one ewg_batch_potential_force_ov call (uploads, all cells, downloads).
        packed = eb.PackedCells(my_cells, alloc=lambda shape: torch.empty(
            shape, dtype=torch.float64, pin_memory=True).numpy())
        for lanes in (0, 1):
            ctx.set_batch_lanes(lanes)
            for _ in range(args.warmup):
                packed.evaluate(ctx, tol, **kw)
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            l0 = ctx.kernel_launches
            e0.record(stream)
            for _ in range(args.steps):
                packed.evaluate(ctx, tol, **kw)
            e1.record(stream)
            torch.cuda.synchronize()
            if lanes == 0:
                launches = ctx.kernel_launches - l0
            res[lanes] = maxrank(e0.elapsed_time(e1) / 1e3) / args.steps
        if name == "fp64":
            pots, forces = ctx.batch_potential_force(my_cells, tol)
            barrier()
            t0 = time.perf_counter()
            sharding.gather_results(mine, pots, forces, len(cells), ws)
            gather_s = maxrank(time.perf_counter() - t0)
        out[name] = {"value": len(cells) / res[0], "ms_per_step": 1e3 * res[0],
                     "one_lane_value": len(cells) / res[1], "gpu_launches": launches}
        if note:
            out[name]["params"] = note
        ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    h2d = sum(len(c[1]) * 4 * 8 + 9 * 8 for c in cells)
    d2h = natoms * 4 * 8
    line = {"metric": metric,
            "value": out["fp64"]["value"], "unit": "cells/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": out["fp64"]["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "timing": "CUDA events on the library's stream around each rank's batched C-ABI calls on "
                      "page-locked host arrays packed once (host checks, uploads, all cells and "
                      "downloads inside), max over ranks; segmented launches (one per stage for all "
                      "cells of a rank)",
            "config": {"workload": label, "cells": len(cells), "natoms_total": natoms,
                       "tol": TOL_FP64, "parallelism": f"cells sharded over {ws} ranks (LPT)",
                       "l2": "working set of a batch > L2 for c3_batch; c4 cells fit in L2"},
            "e2e": {"value": out["fp64"]["value"], "unit": "cells/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": out["fp64"]["gpu_launches"],
            "one_lane_value": out["fp64"]["one_lane_value"],
            "result_gather_s": gather_s,
            "mixed": dict(out["mixed"], unit="cells/s", tol=TOL_MIXED,
                          speedup_vs_fp64=out["mixed"]["value"] / out["fp64"]["value"])}
    print(json.dumps(line), flush=True)
    return 0


def run_scc(args, eb, torch, device, dist, ws, rank):
    """SCC on fixed geometry: 30 charge updates per step, each followed by a
    shift (potential) evaluation through the TCoulomb-style resident calls
    (ewg_set_charges + ewg_shift, host arrays).  c5_scc: the 216,000-site rock
    salt; c3_scc: the 32,769-atom water box.  One cell does not shard: under
    torchrun every rank runs a replica, each timed with CUDA events on the
    library's stream, max over ranks."""
    if args.workload == "c5_scc":
        pos, q, lat = workloads.c5_rock_salt_216k()
        charges = [workloads.c5_charge_update(q, k) for k in range(30)]
        label, metric = "c5_rock_salt_216000_scc30", "C5 SCC: shift evals/s at 216,000 sites, fixed geometry, 30 charge updates"
        grids = "working set (512^3 grids) > L2"
    else:
        pos, q, lat = workloads.c3_water_32k()
        charges = [workloads.charge_update(q, k, seed=3) for k in range(30)]
        label, metric = "c3_water_32769_scc30", "C3 SCC: shift evals/s at 32,769 atoms, fixed geometry, 30 charge updates"
        grids = "working set (280^3 grids) > L2"

    def maxrank(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    out = {}
    for name, prec, tol in (("fp64", eb.FP64, TOL_FP64), ("mixed", eb.MIXED, TOL_MIXED)):
        ctx = eb.Context(device, prec)
        stream = torch.cuda.Stream(device=device)
        ctx.set_stream(stream.cuda_stream)
        ctx.set_lattice(np.asarray(lat).T)
        ctx.set_coords(np.ascontiguousarray(np.asarray(pos)))
        for k in range(min(args.warmup, 30)):
            ctx.set_charges(charges[k])
            ctx.shift(tol, len(q))
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = ctx.kernel_launches
        e0.record(stream)
        nev = 0
        for _ in range(args.steps):
            for k in range(30):
                ctx.set_charges(charges[k])
                ctx.shift(tol, len(q))
                nev += 1
        e1.record(stream)
        torch.cuda.synchronize()
        dt = maxrank(e0.elapsed_time(e1) / 1e3)
        out[name] = {"value": ws * nev / dt, "ms_per_eval": 1e3 * dt / nev,
                     "gpu_launches": ctx.kernel_launches - l0}
        # The same 30 updates in one submission each step (ewg_shift_batch):
        # one upload, one download, no host wait between the updates.
        qs = np.ascontiguousarray(np.stack(charges))
        res = np.empty_like(qs)
        for _ in range(max(args.warmup, 1)):
            ctx.shift_batch(tol, qs, out=res)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            ctx.shift_batch(tol, qs, out=res)
        e1.record(stream)
        torch.cuda.synchronize()
        dtb = maxrank(e0.elapsed_time(e1) / 1e3)
        out[name]["batched"] = {"value": ws * nev / dtb, "ms_per_eval": 1e3 * dtb / nev}
        ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    n = len(q)
    line = {"metric": metric,
            "value": out["fp64"]["value"], "unit": "evals/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 30 * out["fp64"]["ms_per_eval"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "timing": "CUDA events on the library's stream around set_charges + shift, host arrays "
                      "in and out, max over ranks",
            "config": {"workload": label, "natoms": n, "tol": TOL_FP64,
                       "parallelism": f"replicas x{ws}", "l2": grids},
            "e2e": {"value": out["fp64"]["value"], "unit": "evals/s", "h2d_bytes_per_step": 30 * n * 8,
                    "d2h_bytes_per_step": 30 * n * 8},
            "gpu_launches": out["fp64"]["gpu_launches"],
            "batched": {"value": out["fp64"]["batched"]["value"], "unit": "evals/s",
                        "what": "the 30 updates of a step in one ewg_shift_batch call"},
            "mixed": {"value": out["mixed"]["value"], "unit": "evals/s", "tol": TOL_MIXED,
                      "batched": out["mixed"]["batched"]["value"]}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch

    import ewald_b200 as eb

    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    device = local
    torch.cuda.set_device(device)
    eb.lib()
    if args.workload in ("c4", "c3_batch"):
        return run_batched(args, eb, torch, device, dist, ws, rank)
    if args.workload in ("c5_scc", "c3_scc"):
        return run_scc(args, eb, torch, device, dist, ws, rank)
    gen, label = SINGLE_CELL[args.workload]
    pos, q, lat = gen()

    if args.profile_only:
        # For profiler captures: warm-up + steps evaluations of one form, nothing
        # timed, no JSON line (numbers taken under a profiler are not results).
        prec, tol = (eb.MIXED, TOL_MIXED) if args.profile_only == "mixed" else (eb.FP64, TOL_FP64)
        scheme = eb.FORCE_AD if args.profile_only == "fp64_ad" else None
        ov = None
        if args.profile_only == "mixed" and args.mixed_params:
            # the tuned parameters of a previous bench line: mixed.params
            mp = json.loads(args.mixed_params)
            ov = {"alpha_in": mp["alpha"], "r_cut_in": mp["r_cut_bohr"], "k_cut_in": mp["k_cut"],
                  "windowCutoff_in": mp["window_cutoff"]}
            scheme = eb.FORCE_AD if mp["forces"] == "window differentiation" else eb.FORCE_IK
        arm = Arm(eb, torch, device, prec, tol, pos, q, lat, scheme=scheme, ov=ov)
        for _ in range(args.warmup + args.steps):
            arm.step_device()
        torch.cuda.synchronize()
        print(f"profile-only: {args.warmup + args.steps} {args.profile_only} evaluations", flush=True)
        return 0

    # Three arms on the same inputs:
    #   fp64     the plain form: FP64, the reference's parameters and its i k forces;
    #   fp64_ad  the same with forces by window differentiation (one inverse FFT);
    #   mixed    the mixed form (FP32 stencils, FFT and pair terms), with the
    #            force scheme and parameters from the library's autotuner for an
    #            RMS force error of at most MIXED_TARGET / 2 against fp64.
    fp64 = Arm(eb, torch, device, eb.FP64, TOL_FP64, pos, q, lat)
    fp64_ad = Arm(eb, torch, device, eb.FP64, TOL_FP64, pos, q, lat, scheme=eb.FORCE_AD)
    tuner = eb.Context(device, eb.MIXED)
    tuned_ov, tuned_scheme, tune_report = tuner.tune(pos, q, lat, MIXED_TARGET)  # untimed, once
    tuner.close()
    mixed = Arm(eb, torch, device, eb.MIXED, TOL_MIXED, pos, q, lat, scheme=tuned_scheme,
                ov=tuned_ov)
    # SCC-style shift evaluations (potential only: one spread, one inverse
    # transform, one gather), reported beside the force evaluations.
    shift64 = Arm(eb, torch, device, eb.FP64, TOL_FP64, pos, q, lat, want_force=False)
    shift32 = Arm(eb, torch, device, eb.MIXED, TOL_MIXED, pos, q, lat, ov=tuned_ov,
                  want_force=False)
    scheme_name = {eb.FORCE_IK: "ik", eb.FORCE_AD: "window differentiation"}
    for a in (fp64, fp64_ad, mixed, shift64, shift32):
        a.tune_shapes()  # untimed, once per arm

    # accuracy of the other arms against the plain form (same inputs)
    for a in (fp64, fp64_ad, mixed):
        a.step_device()
    torch.cuda.synchronize()
    p64, f64 = fp64.pot.cpu().numpy(), fp64.force.cpu().numpy()

    def rel(a, b):
        return {"max": float(np.abs(a - b).max() / np.abs(b).max()),
                "rms": float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))}

    err = {"potential": rel(mixed.pot.cpu().numpy(), p64), "force": rel(mixed.force.cpu().numpy(), f64)}
    err_ad = {"potential": rel(fp64_ad.pot.cpu().numpy(), p64),
              "force": rel(fp64_ad.force.cpu().numpy(), f64)}
    # FP64 direct-Ewald ground truth (the direct engine with its splitting
    # pinned: cell-list real space, structure-factor sum over the k sphere),
    # against which the mixed form's bar (RMS force <= 1e-6) is defined.
    pd, fd = fp64.ctx.direct_ground_truth(pos, q, lat)
    err_direct = {"potential": rel(mixed.pot.cpu().numpy(), pd),
                  "force": rel(mixed.force.cpu().numpy(), fd)}
    err64_direct = {"potential": rel(p64, pd), "force": rel(f64, fd)}
    params64 = fp64.ctx.last_params()
    params32 = mixed.ctx.last_params()

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    tensor_peak = fp64.ctx.fp64_mma_peak()
    sampler = ClockSampler(device)
    barrier()
    sampler.start()
    time.sleep(0.3)  # the sampler's first reading lands inside the timed regions
    ms64, launches64, _ = fp64.time_device(args.steps, args.warmup)
    barrier()
    msad, launchesad, _ = fp64_ad.time_device(args.steps, args.warmup)
    barrier()
    ms32, launches32, _ = mixed.time_device(args.steps, args.warmup)
    barrier()
    mss64, _, _ = shift64.time_device(args.steps, args.warmup)
    barrier()
    mss32, _, _ = shift32.time_device(args.steps, args.warmup)
    clocks = sampler.stop()
    barrier()
    # Per-stage device times come from a separate profiled pass: with stage
    # events on, the library runs the real-space sum in line instead of beside
    # the mesh pipeline, so these stages add up to more than the step time.
    _, _, stages = fp64.time_device(args.steps, 0, profile=True)
    _, _, stagesad = fp64_ad.time_device(args.steps, 0, profile=True)
    _, _, stages32 = mixed.time_device(args.steps, 0, profile=True)
    barrier()
    e2e64 = fp64.time_e2e(args.steps, args.warmup)
    barrier()
    e2ead = fp64_ad.time_e2e(args.steps, args.warmup)
    barrier()
    e2e32 = mixed.time_e2e(args.steps, args.warmup)
    barrier()
    e2es64 = shift64.time_e2e(args.steps, args.warmup)
    barrier()
    e2es32 = shift32.time_e2e(args.steps, args.warmup)
    barrier()

    def maxrank(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    t64 = maxrank(sum(ms64) / 1e3)
    tad = maxrank(sum(msad) / 1e3)
    t32 = maxrank(sum(ms32) / 1e3)
    te64 = maxrank(e2e64)
    tead = maxrank(e2ead)
    te32 = maxrank(e2e32)
    ts64, ts32 = maxrank(sum(mss64) / 1e3), maxrank(sum(mss32) / 1e3)
    tes64, tes32 = maxrank(e2es64), maxrank(e2es32)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        times = cpu_evals(pos, q, lat, TOL_FP64, 1, 0, threads)
        cpu = {"value": 1.0 / times[0], "unit": "evals/s", "cores": threads, "kind": "port",
               "sample": f"1 full {len(q)}-atom shift+force evaluation at tol 1e-10 (oracle/ C++ "
                         "restatement of the reference, OpenMP, project FFT in place of FFTW)",
               "split_s": cpu_evals.split}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    peak, peak_kind = load_peaks()
    natoms = len(q)

    def roofline(stages_ms, params, real_bytes, steps, tensor_peak=None, nc=4):
        """Per-stage rates; the roofline entry is the stage with the largest time.
        HBM-type stages (the FFT passes; every stage in the FP32 form) use
        algorithmic bytes / time against the measured copy bandwidth.  The FP64
        spread and gather run on the FP64 tensor cores (DMMA): algorithmic FP64
        flops / time against the FP64 tensor rate measured live on this GPU.
        nc: grids through the inverse passes and the gather (4 for i k, 1 for
        window differentiation)."""
        sb = stage_bytes(params, natoms, real_bytes, nc)
        fl = stage_flops(params, natoms) if tensor_peak else {}
        per = {}
        for name, (ms, _) in stages_ms.items():
            if ms <= 0:
                continue
            dur = ms / steps / 1e3
            entry = {"ms": ms / steps}
            if name in fl:
                entry["tflops"] = fl[name] / dur / 1e12
                entry["flops"] = fl[name]
            elif name in sb:
                entry["gbs"] = sb[name] / dur / 1e9
                entry["bytes"] = sb[name]
            per[name] = entry
        top = max((k for k in per if k in sb or k in fl), key=lambda k: per[k]["ms"])
        traffic = DRAM_TRAFFIC.get((args.workload, real_bytes, nc, top))
        if top in fl:
            ach = per[top]["tflops"]
            roof = {"bound": "tensor", "kernel": top, "achieved": ach, "peak": tensor_peak,
                    "unit": "TFLOP/s", "frac": ach / tensor_peak,
                    "peak_source": "measured live: dense FP64 DMMA m8n8k4 rate (ewg_fp64_mma_peak)",
                    "traffic": traffic}
        else:
            ach = per[top]["gbs"]
            roof = {"bound": "hbm", "kernel": top, "achieved": ach, "peak": peak, "unit": "GB/s",
                    "frac": ach / peak, "peak_source": f"{peak_kind} hbm_gbs", "traffic": traffic}
        return top, per, roof

    def whole_eval(params, real_bytes, t_step, nc=4):
        """Algorithmic bytes of one evaluation (the sum of the stage counts)
        against the measured HBM rate."""
        b = sum(stage_bytes(params, natoms, real_bytes, nc).values())
        return {"bytes": b, "achieved_gbs": b / t_step / 1e9, "frac": b / t_step / 1e9 / peak}

    def grid_of(params):
        return "x".join(str(2 * m) for m in params["n_modes"])

    top64, per64, roof64 = roofline(stages, params64, 8, args.steps, tensor_peak)
    _, perad, roofad = roofline(stagesad, params64, 8, args.steps, tensor_peak, nc=1)
    nc32 = 1 if tuned_scheme == eb.FORCE_AD else 4
    top32, per32, roof32 = roofline(stages32, params32, 4, args.steps, nc=nc32)
    h2d = natoms * 3 * 8 + natoms * 8
    d2h = natoms * 8 + natoms * 3 * 8
    value = ws * args.steps / t64
    e2e_io = {"h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
    line = {
        "metric": metric_for(args.workload, natoms), "value": value, "unit": "evals/s", "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t64 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": label, "natoms": natoms,
                   "tol": TOL_FP64, "grid": grid_of(params64),
                   "window_cutoff": params64["window_cutoff"], "alpha": params64["alpha"],
                   "r_cut_bohr": params64["r_cut"], "forces": "ik (the reference's scheme)",
                   "kernel_shape": fp64.shape,
                   "parallelism": f"replicas x{ws}",
                   "l2": "flushed between steps (256 MiB write, untimed); working set > L2"},
        "e2e": dict(value=ws * args.steps / te64, unit="evals/s", **e2e_io),
        "rel_err_vs_direct": err64_direct,
        "roofline": roof64,
        "whole_eval_hbm": whole_eval(params64, 8, t64 / args.steps),
        "stages_ms": per64,
        "fp64_ad": {
            "value": ws * args.steps / tad, "unit": "evals/s", "forces": "window differentiation",
            "speedup_vs_fp64": (ws * args.steps / tad) / value,
            "e2e": dict(value=ws * args.steps / tead, unit="evals/s", **e2e_io),
            "rel_err_vs_fp64": err_ad, "roofline": roofad, "kernel_shape": fp64_ad.shape,
            "whole_eval_hbm": whole_eval(params64, 8, tad / args.steps, nc=1), "stages_ms": perad,
            "gpu_launches": launchesad,
        },
        "mixed": {
            "value": ws * args.steps / t32, "unit": "evals/s", "forces": scheme_name[tuned_scheme],
            "params": {"source": f"ewg_tune, target {MIXED_TARGET:g} (RMS force error <= "
                                 f"{MIXED_TARGET / 2:g} vs the FP64 form)",
                       "forces": scheme_name[tuned_scheme], "alpha": params32["alpha"],
                       "r_cut_bohr": params32["r_cut"], "k_cut": params32["k_cut"],
                       "grid": grid_of(params32), "window_cutoff": params32["window_cutoff"],
                       "tuner_report": tune_report, "kernel_shape": mixed.shape},
            "speedup_vs_fp64": (ws * args.steps / t32) / value,
            "e2e": dict(value=ws * args.steps / te32, unit="evals/s", **e2e_io),
            "rel_err_vs_fp64": err, "rel_err_vs_direct": err_direct, "roofline": roof32,
            "whole_eval_hbm": whole_eval(params32, 4, t32 / args.steps, nc=nc32), "stages_ms": per32,
            "gpu_launches": launches32,
        },
        "shift_only": {
            "what": "SCC-style shift evaluations: potential only (one spread, one inverse "
                    "transform, one gather) plus the real-space potential",
            "fp64": {"value": ws * args.steps / ts64, "unit": "evals/s",
                     "e2e": {"value": ws * args.steps / tes64, "unit": "evals/s",
                             "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": natoms * 8}},
            "mixed": {"value": ws * args.steps / ts32, "unit": "evals/s",
                      "e2e": {"value": ws * args.steps / tes32, "unit": "evals/s",
                              "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": natoms * 8}},
        },
        "gpu_launches": launches64,
        "clocks": clocks,
    }
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["c3", "c1", "c2", "c5", "c4", "c5_scc", "c3_scc", "c3_batch"],
                    default="c3",
                    help="c3 (default, the headline) or another configuration of the table")
    ap.add_argument("--profile-only", choices=["fp64", "fp64_ad", "mixed"], default=None,
                    help="run warm-up + steps evaluations of one form for a profiler; no timing")
    ap.add_argument("--mixed-params", default=None,
                    help="with --profile-only mixed: a bench line's mixed.params (JSON) to run "
                         "the tuned parameters instead of the reference chain at tol 1e-7")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
