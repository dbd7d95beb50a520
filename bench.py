#!/usr/bin/env python
"""Benchmark of the MOLDY Fe EAM hot path on B200.

Metric: atom-steps/s of the 2,000,000-atom bcc Fe workload (100^3 cells,
a0 = 2.8665 A, Gaussian displacements sigma = 0.05 A, 1200 K Maxwell-Boltzmann
velocities, Parrinello-Rahman NPT at 0 GPa, dt = 1 fs, FETRANSMETAL Fe-Fe
lookup tables, rnear = 6.3 A, neighbour list rebuilt every 100 steps).  One
"step" is one mdloop iteration: velocity Verlet (drift, force = link-cell
relink on schedule, half-list build on schedule, density pass, embedding,
pair-force pass, virial, box update) and update_therm_avs.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value   -- device-resident throughput of the mixed-precision path (state in
           HBM; CUDA events on the library's stream; max over ranks); the FP64
           path is timed beside it ("fp64", "speedup_mixed_over_fp64") and the
           mixed path's force, energy, stress and NVE-drift errors against FP64
           are in "accuracy_mixed_vs_fp64"
e2e     -- the same K steps through the C ABI with host buffers: state upload
           from pinned memory, K mdloop calls returning their thermodynamics to
           the host, state and forces read back
Multi-GPU runs are independent replicas (the path does not shard across GPUs).

  --workload batch    1024 supercells (config 3): batched force evaluations and the CG quench
  --workload adjoint  256 x 1024-atom force-matching gradients (config 4)
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s, 2M-atom Fe EAM: mixed vs FP64 GPU at <=1e-5 eV/A force err"
UNIT = "atom-steps/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=100, help="bcc cells per box side (2 n^3 atoms)")
    ap.add_argument("--precision", choices=["both", "fp64", "mixed"], default="both",
                    help="both: the mixed path is the headline value, the FP64 path is timed beside it")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--skins", default=None,
                    help="md: intermediate/outer list skins in A (e.g. 0.15/0.8) instead of the sweep")
    ap.add_argument("--nve-steps", type=int, default=1000)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-quench", action="store_true", help="batch: skip the quench")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--ref-seconds", type=float, default=150.0)
    ap.add_argument("--workload", choices=["md", "batch", "adjoint", "liquid", "rdf", "small"], default="md",
                    help="md: the 2M-atom NPT step (headline); batch: 1024 supercells, force "
                         "evaluations and the CG quench; adjoint: force-matching gradients; liquid: "
                         "the 1.024M-atom heating ramp 300 -> 2500 K with scalev; rdf: the structure "
                         "analysis of the 2M-atom cell; small: the 2000-atom NVE case against the oracle")
    ap.add_argument("--nsys", type=int, default=1024, help="batch: number of supercells")
    ap.add_argument("--nconf", type=int, default=256, help="adjoint: number of configurations")
    ap.add_argument("--adj-engines", type=int, default=4, help="adjoint: engines (host threads) per rank")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def workload(n, seed):
    from moldy_b200 import workloads as wl
    return wl.config_large_npt(n=n, seed=seed)


def config_dict(w, precision, extra=None):
    d = {
        "workload": w.name, "atoms": w.nm, "cells": [w.meta["n"]] * 3, "a0": w.meta["a0"],
        "sigma_A": w.meta["sigma"], "temperature_K": w.meta["temperature"],
        "ensemble": "NPT Parrinello-Rahman, P=0 GPa, boxmass 50" if w.ivol == 0 else "NVE",
        "dt_fs": w.meta["dt_fs"], "potential": "FETRANSMETAL Fe-Fe, lookup tables nlookup=5000",
        "rnear_A": w.rnear, "nbrupdate": w.ntcm, "precision": precision,
        "l2": "inputs larger than L2 (per-step working set > 1 GB vs 126 MB L2)",
        "parallelism": "replicas",
    }
    if extra:
        d.update(extra)
    return d


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML (read only)."""

    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
        0x8: "hw_slowdown", 0x10: "sync_boost", 0x20: "sw_thermal_slowdown",
        0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
        0x100: "display_clock_setting",
    }

    def __init__(self, torch_device: int):
        self.samples = []
        self.reasons = 0
        self.max_mhz = None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml as nv
            import torch
            nv.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(torch_device).uuid)
            for i in range(nv.nvmlDeviceGetCount()):
                h = nv.nvmlDeviceGetHandleByIndex(i)
                u = nv.nvmlDeviceGetUUID(h)
                u = u.decode() if isinstance(u, bytes) else u
                if u.replace("GPU-", "") == uuid.replace("GPU-", ""):
                    self._h = h
                    break
            if self._h is None and nv.nvmlDeviceGetCount() == 1:
                self._h = nv.nvmlDeviceGetHandleByIndex(0)
            if self._h is not None:
                self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(self._h, nv.NVML_CLOCK_SM)
            self._nv = nv
        except Exception:
            self._h = None

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                self.samples.append((mhz, r))
                self.reasons |= r
            except Exception:
                pass
            self._stop.wait(0.05)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._h is not None:
            self._t.join(timeout=2)

    def summary(self):
        if self._h is None or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        busy = [m for m, r in self.samples if not (r & 0x1)] or [m for m, _ in self.samples]
        names = [v for k, v in self.REASONS.items() if self.reasons & k and k != 0x1]
        return {"sm_mhz": float(statistics.median(busy)), "sm_max_mhz": self.max_mhz,
                "reasons": names, "samples": len(self.samples)}


# ---------------------------------------------------------------- roofline --
def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def kernel_bytes_per_atom(name, n_half, n_full, n_screen, mixed=True):
    """Algorithmic DRAM bytes per atom of one launch.
    n_half: mean half-list length; n_full: mean interacting (directed) pairs;
    n_screen: mean intermediate-row entries the screening pass reads; mixed:
    the fixed-point position records (16 bytes) instead of the FP64 ones (32)."""
    own = 16 if mixed else 32
    table = {
        # intermediate row + count, own position; compact-row writes + count, F and F'
        # writes, position record with F' (rho is stored on the last step of a call only)
        "screen_density": 4.0 * n_screen + 4 + own + 4.0 * n_full + 4 + 16 + own,
        # compact row + count, own position record, mass; forces; x1 and x2 read + write, del2, Z
        "forces": 4.0 * n_full + 4 + own + 8 + 24 + 48 + 48 + 8 + 4,
        # pos read + write, x1, x2, build snapshot (fixed point), mass, Z, fixed-point positions
        "drift": 64 + 48 + 16 + 8 + 4 + 16,
        "therm": 48 + 8 + 4,
        "build_nlist": 4.0 * n_half + 4 + 32 + 16,
    }
    return table.get(name)


def load_traffic():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return None
    return None


# ------------------------------------------------------------ CPU baseline --
def cpu_baseline(w, seconds):
    """Times the oracle (the C restatement of the reference) on the host cores."""
    import oracle
    oracle.build()
    nthreads = oracle.max_threads()
    o = oracle.from_workload(w, uselookup=True, threads=nthreads)
    o.md_init()
    t0 = time.perf_counter()
    steps = 0
    while True:
        o.md_step()
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds or steps >= 1000:
            break
    o.close()
    return {"value": w.nm * steps / el, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"{steps} mdloop steps of the {w.nm}-atom workload after set-up "
                      f"(linkup, list build, md_init untimed), {nthreads} OpenMP threads, "
                      f"{el:.1f} s"}


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    import oracle
    oracle.build()
    w = workload(args.n, seed=2)
    nthreads = oracle.max_threads()
    o = oracle.from_workload(w, uselookup=True, threads=nthreads)
    o.md_init()
    for _ in range(min(args.warmup, 2)):
        o.md_step()
    t0 = time.perf_counter()
    steps = 0
    while steps < args.steps:
        o.md_step()
        steps += 1
        if time.perf_counter() - t0 > args.ref_seconds:
            break
    el = time.perf_counter() - t0
    value = w.nm * steps / el
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": args.gpus, "steps": steps, "warmup": min(args.warmup, 2),
        "ms_per_step": 1000.0 * el / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(w, "fp64", {"parallelism": "host OpenMP"}),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                         "sample": f"{steps} of the requested {args.steps} mdloop steps of the "
                                   f"{w.nm}-atom workload (bounded to {args.ref_seconds:.0f} s), "
                                   f"{nthreads} OpenMP threads; the Fortran reference cannot be "
                                   "compiled on this image, so the C restatement stands in"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# -------------------------------------------------------------------- ours --
def time_path(args, w, precision, local_rank, barrier, max_over_ranks, with_e2e):
    """One precision of the 2M-atom step: autotune (untimed), warm-up, K timed
    steps with the state in HBM, the launch-level profile, the roofline of the
    dominant kernel and, when asked, the end-to-end run through the C ABI."""
    import torch
    from moldy_b200 import MoldySystem
    world = dist_env()[2]
    sysm = MoldySystem.from_workload(w, precision=precision, device=local_rank)
    sysm.linkup()
    sysm.md_init()
    tune = sysm.autotune(nreps=5)
    stream = torch.cuda.ExternalStream(sysm.stream_handle(), device=local_rank)
    # untimed: the intermediate- and outer-list skins that give the shortest
    # steps here (outer rebuilds are rare, so each pair runs 100 steps)
    skin_ms = {}
    grid = [tuple(float(x) for x in args.skins.split("/"))] if args.skins else \
        [(mid, out) for mid in (0.1, 0.15, 0.2) for out in (0.6, 0.8, 1.0)]
    for mid, out in grid:
        sysm.set_mid_skin(mid)
        sysm.set_outer_skin(out)
        sysm.md_steps(10, thermo=False)
        t0 = time.perf_counter()
        sysm.md_steps(100, thermo=False)
        sysm.synchronize()
        skin_ms[f"{mid}/{out}"] = (time.perf_counter() - t0) * 1000.0 / 100
    best = min(skin_ms, key=skin_ms.get)
    best_mid, best_out = (float(x) for x in best.split("/"))
    sysm.set_mid_skin(best_mid)
    sysm.set_outer_skin(best_out)
    tune["list_skins_ms_per_step"] = skin_ms
    tune["chosen"]["mid_skin_A"] = best_mid
    tune["chosen"]["outer_skin_A"] = best_out
    sysm.md_steps(max(args.warmup, 3), thermo=False)
    sysm.synchronize()
    # the timed steps run without the per-launch events of the profiler
    # (launch counts are kept either way)
    sysm.reset_kernel_stats()
    builds0 = sysm.list_stats()["mid_builds"]
    obuilds0 = sysm.outer_builds()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        barrier()
        torch.cuda.synchronize()
        sysm.synchronize()
        e0.record(stream)
        sysm.md_steps(args.steps, thermo=False)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier()
    ms = e0.elapsed_time(e1)
    launches = int(sum(n for _, n in sysm.kernel_stats().values()))
    ms_max = max_over_ranks(ms)
    value = world * w.nm * args.steps / (ms_max / 1000.0)
    lst_timed = sysm.list_stats()
    out_builds_per_step = (sysm.outer_builds() - obuilds0) / args.steps
    # end to end through the C ABI, right after the timed steps: host state in,
    # the same K steps with their per-step thermo records, host state out.  An
    # untimed pass of the same call first sizes the pinned thermo staging.
    e2e = None
    if with_e2e:
        sysm.md_steps(args.steps, thermo=True)
        sysm.synchronize()
        st = sysm.get_state()
        pin = [torch.empty(w.nm, dtype=torch.float64, pin_memory=True).numpy() for _ in range(12)]
        for k, name in enumerate(("x0", "x1", "x2")):
            for c in range(3):
                pin[3 * k + c][:] = st[name][:, c]
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        sysm.set_state_soa(*pin[:9], b0=st["b0"], b1=st["b1"], b2=st["b2"])
        sysm.md_steps(args.steps, thermo=True)
        sysm.get_state_soa(pin[:9], forces=pin[9:12])
        e1.record(stream)
        e1.synchronize()
        barrier()
        ems = max_over_ranks(e0.elapsed_time(e1))
        h2d = 9 * 8 * w.nm + 3 * 72
        d2h = 12 * 8 * w.nm + args.steps * 104 + 4 * 72
        e2e = {"value": world * w.nm * args.steps / (ems / 1000.0), "unit": UNIT,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "ms": ems}

    # then a profiled stretch: per-kernel CUDA-event times on the library's stream
    prof_steps = min(args.steps, 300)
    sysm.reset_kernel_stats()
    sysm.set_profiling(True)
    e0.record(stream)
    sysm.md_steps(prof_steps, thermo=False)
    e1.record(stream)
    e1.synchronize()
    prof_ms = e0.elapsed_time(e1)
    sysm.set_profiling(False)
    stats = sysm.kernel_stats()
    _, numn = sysm.neighbour_list() if w.nm <= 4_000_000 else (None, None)
    n_half = float(np.mean(numn)) if numn is not None else 44.0
    lst = sysm.list_stats()
    n_full = lst["pairs"] / w.nm
    n_screen = lst["screened"] / w.nm
    mid_builds_per_step = (lst_timed["mid_builds"] - builds0) / args.steps
    dname, (dms, dlaunch) = max(stats.items(), key=lambda kv: kv[1][0])
    peak, peak_kind = load_peaks()
    bpa = kernel_bytes_per_atom(dname, n_half, n_full, n_screen, mixed=(precision == "mixed"))
    roofline = None
    if bpa is not None and dlaunch > 0:
        achieved = bpa * w.nm / (dms / 1000.0 / dlaunch) / 1e9
        traffic = None
        tr = (load_traffic() or {}).get(precision, {})
        if dname in tr.get("kernels", {}):
            traffic = float(tr["kernels"][dname]["dram_bytes_per_atom"]) * w.nm
        roofline = {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": peak,
                    "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": traffic, "algorithmic_bytes_per_launch": bpa * w.nm,
                    "avg_launch_ms": dms / dlaunch, "share_of_step": dms / prof_ms,
                    "profiled_steps": prof_steps}
    sysm.close()
    return {"value": value, "ms_per_step": ms_max / args.steps, "launches": launches, "stats": stats,
            "roofline": roofline, "e2e": e2e, "clocks": clk.summary(), "tune": tune,
            "n_half": n_half, "n_full": n_full, "n_screen": n_screen, "mid_builds_per_step": mid_builds_per_step,
            "out_builds_per_step": out_builds_per_step}


def _errors(f, pe, sig, f_ref, pe_ref, sig_ref, nm):
    df = f - f_ref
    return {"force_rms_err_eV_per_A": float(np.sqrt(np.mean(np.sum(df * df, axis=1)))),
            "force_max_err_eV_per_A": float(np.max(np.linalg.norm(df, axis=1))),
            "pe_err_eV_per_atom": abs(pe - pe_ref) / nm,
            "stress_max_err_GPa": float(np.max(np.abs(sig - sig_ref))) * 160.21766}


def accuracy(w, local_rank, nve_steps):
    """On the same 2M-atom state: the mixed path against the FP64 path, and both
    against the oracle (the C restatement of the reference, all host threads):
    real-force RMS and max errors, pe and stress differences, and whether the
    half list NLIST/NUMN is identical entry by entry.  Then the total-energy
    drift of an NVE run of the same lattice (te = ke + pe per atom,
    least-squares slope per ps) with the lookup tables in both precisions, and
    with the analytic pair functions (uselookup = 0, FP64)."""
    import oracle
    from moldy_b200 import MoldySystem
    from moldy_b200 import workloads as wl
    out = {}
    res = {}
    nl_gpu = None
    for prec in ("fp64", "mixed"):
        s = MoldySystem.from_workload(w, precision=prec, device=local_rank)
        s.linkup()
        fo = s.force()
        b0 = s.get_state()["b0"]
        res[prec] = (s.forces() @ b0.T, fo["pe"], -(fo["tp"] @ b0.T) / fo["vol"])
        if prec == "fp64":
            nl_gpu = s.neighbour_list()
        s.close()
    out.update(_errors(*res["mixed"], *res["fp64"], w.nm))
    # against the oracle on the same state
    oracle.build()
    nth = oracle.max_threads()
    o = oracle.from_workload(w, uselookup=True, threads=nth)
    t0 = time.perf_counter()
    o.force()
    t_o = time.perf_counter() - t0
    oo = o.force_out()
    ref = (o.forces() @ w.b0.T, oo["pe"], -(oo["tp"] @ w.b0.T) / oo["vol"])
    nlo, nno = o.nlist()
    o.close()
    mask = np.arange(w.nnbrs, dtype=np.int32)[None, :] < nno[:, None]
    nl_same = bool(np.array_equal(nno, nl_gpu[1]) and np.array_equal(np.where(mask, nlo, 0), nl_gpu[0]))
    del nlo, mask
    fr = np.linalg.norm(ref[0])
    out["vs_oracle"] = {
        "oracle": f"C restatement of the reference, FP64, {nth} OpenMP threads, {t_o:.2f} s for linkup, "
                  "half-list build and force",
        "neighbour_list_identical": nl_same,
        "half_list_entries": int(nno.sum()),
        "fp64": {**_errors(*res["fp64"], *ref, w.nm),
                 "force_rel_norm_err": float(np.linalg.norm(res["fp64"][0] - ref[0]) / fr)},
        "mixed": {**_errors(*res["mixed"], *ref, w.nm),
                  "force_rel_norm_err": float(np.linalg.norm(res["mixed"][0] - ref[0]) / fr)},
    }
    if nve_steps > 0:
        wn = wl.make_workload(w.meta["n"], sigma=0.05, temperature=300.0, ivol=1, nbrupdate=100, seed=5,
                              name="bcc_fe_nve_300K")
        dt_ps = wn.meta["dt_fs"] / 1000.0
        drift = {}
        for prec, lookup in (("fp64", True), ("mixed", True), ("fp64_exact", False)):
            s = MoldySystem.from_workload(wn, precision=prec.split("_")[0], uselookup=lookup,
                                          device=local_rank)
            s.linkup()
            s.md_init()
            th = s.md_steps(nve_steps, thermo=True)
            te = np.array([r["te"] for r in th]) / wn.nm
            t = np.arange(len(te)) * dt_ps
            slope = float(np.polyfit(t, te, 1)[0])
            drift[prec] = {"slope_eV_per_atom_per_ps": slope, "te_range_eV_per_atom": float(te.max() - te.min())}
            s.close()
        drift["fp64_exact"]["note"] = ("analytic pair functions (uselookup = 0): the tabulated dvee is not "
                                       "the derivative of the interpolated vee, which the lookup runs' "
                                       "drift reflects")
        out["nve_drift"] = {"workload": f"{wn.nm}-atom bcc Fe NVE, 300 K, {nve_steps} steps of 1 fs",
                            **drift,
                            "mixed_minus_fp64_eV_per_atom_per_ps": drift["mixed"]["slope_eV_per_atom_per_ps"] -
                            drift["fp64"]["slope_eV_per_atom_per_ps"]}
    return out


def run_ours(args):
    import torch
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    w = workload(args.n, seed=2 + rank)
    head = "mixed" if args.precision in ("both", "mixed") else "fp64"
    runs = {}
    # the headline (mixed) path first, its end-to-end run in a fresh process state
    order = ["mixed", "fp64"] if args.precision == "both" else [args.precision]
    for prec in order:
        runs[prec] = time_path(args, w, prec, local_rank, barrier, max_over_ranks,
                               with_e2e=(prec == head and not args.no_e2e))
    r = runs[head]
    acc = None
    if rank == 0 and args.precision == "both" and not args.no_accuracy:
        acc = accuracy(w, local_rank, args.nve_steps)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        torch.cuda.synchronize()
        cpu = cpu_baseline(w, args.cpu_seconds)
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0
    extra = {"neighbours_half_mean": r["n_half"], "screened_entries_per_atom": r["n_screen"],
             "interacting_pairs_per_atom": r["n_full"], "autotuned_variants": r["tune"]["chosen"],
             "intermediate_list_builds_per_step": r["mid_builds_per_step"],
             "outer_list_builds_per_step": r["out_builds_per_step"],
             "list_skins_ms_per_step": r["tune"].get("list_skins_ms_per_step")}
    line = {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": r["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if head == "fp64" else "f32+f64",
        "data": "synthetic (seeded bcc Fe lattice, Gaussian displacements, Maxwell-Boltzmann velocities)",
        "config": config_dict(w, head, extra),
        "e2e": r["e2e"], "roofline": r["roofline"], "cpu_baseline": cpu,
        "clocks": r["clocks"], "gpu_launches": r["launches"],
        "kernels": {k: {"ms": v[0], "launches": v[1]} for k, v in r["stats"].items() if v[1]},
        "kernels_note": "per-kernel CUDA-event totals over a separate profiled stretch of "
                        f"{min(args.steps, 300)} steps after the timed ones",
        "autotune_ms_per_launch": r["tune"]["ms"],
    }
    # the whole step against the fixed per-atom-step figure of the reference's
    # algorithm (x, v, a and F' read and written, two passes over the int32
    # half list: 160 + 8 n_half bytes), the same for both precisions
    peak, peak_kind = load_peaks()
    step_bytes = 160.0 + 8.0 * r["n_half"]
    line["step_roofline"] = {"bound": "hbm", "bytes_per_atom_step": step_bytes,
                             "achieved": step_bytes * r["value"] / 1e9, "peak": peak, "peak_kind": peak_kind,
                             "unit": "GB/s", "frac": step_bytes * r["value"] / 1e9 / peak}
    if "fp64" in runs and head != "fp64":
        f = runs["fp64"]
        line["fp64"] = {"value": f["value"], "ms_per_step": f["ms_per_step"], "roofline": f["roofline"],
                        "clocks": f["clocks"], "gpu_launches": f["launches"],
                        "kernels": {k: {"ms": v[0], "launches": v[1]} for k, v in f["stats"].items() if v[1]}}
        line["speedup_mixed_over_fp64"] = r["value"] / f["value"]
    if acc is not None:
        line["accuracy_mixed_vs_fp64"] = acc
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------- batch --
BATCH_METRIC = ("atom-evals/s, 1024 bcc Fe supercells of 128-8192 atoms: energy + forces + "
                "virial per system")


def batch_cpu_baseline(ws, seconds):
    """Oracle force + energy_calc over the supercells in order, on all host threads."""
    import oracle
    oracle.build()
    nthreads = oracle.max_threads()
    t0 = time.perf_counter()
    atoms = 0
    nsys = 0
    for w in ws:
        o = oracle.from_workload(w, uselookup=True, threads=nthreads)
        o.force()
        o.energy_calc()
        o.close()
        atoms += w.nm
        nsys += 1
        if time.perf_counter() - t0 >= seconds:
            break
    el = time.perf_counter() - t0
    return {"value": atoms / el, "unit": "atom-evals/s", "cores": nthreads, "kind": "port",
            "sample": f"{nsys} of the supercells ({atoms} atoms), each set up and evaluated once "
                      f"(list build + force + energy_calc), {nthreads} OpenMP threads, {el:.1f} s"}


def run_batch(args):
    import torch
    from moldy_b200 import MoldyBatch
    from moldy_b200 import workloads as wl
    from moldy_b200.adjoint import shard_configs
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    ws_all = wl.config_batch(nsys=args.nsys, seed=3)
    mine = shard_configs([w.nm for w in ws_all], world)[rank]
    ws = [ws_all[i] for i in mine]
    b = MoldyBatch.from_workloads(ws, device=local_rank)
    stream = torch.cuda.ExternalStream(b.stream_handle(), device=local_rank)

    def timed(fn, reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    boxes = [w.b0 for w in ws]
    raw = np.zeros(13 * len(ws))

    def force():
        # the C-ABI call with its preallocated result array (no Python post-processing)
        b.force_into(raw)

    def build_and_force():
        b.set_state(b0=boxes)          # new boxes: every list is built at the next evaluation
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        b.force()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    # untimed: the library's tuner picks the tile lanes (on list-building
    # evaluations) and the gather width (lists current), per precision; the
    # timed evaluations form the force routine's energy, forces and virial,
    # energy_calc's exact energies (the quench's) are timed separately
    prec = "fp64" if args.precision == "fp64" else "mixed"
    b.set_energy_calc(False)
    tunes = {}
    for p in ("fp64", "mixed"):
        b.set_precision(p)
        tunes[p] = b.autotune(nreps=3)
    b.set_precision(prec)
    b.set_tiles(tunes[prec]["chosen"]["lanes"], 256)
    b.set_gather(tunes[prec]["chosen"]["gather"])
    best_gather = {p: tunes[p]["chosen"]["gather"] for p in tunes}
    for _ in range(max(args.warmup, 3)):
        b.force()
    # evaluations with every list current (the positions do not move between
    # them; in a quench or MD run lists are kept until an atom moved half the skin)
    steps = max(1, min(args.steps, 200))
    l0 = b.launches()
    with ClockSampler(local_rank) as clk:
        if world > 1:
            torch.distributed.barrier()
        ms = timed(force, steps)
        if world > 1:
            torch.distributed.barrier()
    ms_max = max_over_ranks(ms)
    launches = b.launches() - l0
    ntot_all = sum(w.nm for w in ws_all)
    value = ntot_all / (ms_max / 1000.0)
    build_ms = max_over_ranks(float(np.median([build_and_force() for _ in range(5)])))
    # per-kernel times of an evaluation with current lists, and the same
    # evaluation with energy_calc's energies
    kt = [b.kernel_times() for _ in range(5)]
    ktimes = {k: float(np.median([t[k] for t in kt])) for k in kt[0]}
    # the dominant pass against its algorithmic bytes per atom: the compact
    # row (4 n + 4), the atom's cell-order record (32) and, density: F' into
    # cell order plus rho, F, F' (32); forces: its F' (8), F read (8), the
    # force (24), the force-routine energy (8) and the six virial moments (48)
    n_row = b.row_entries() / b.ntot
    peak, peak_kind = load_peaks()
    persistent = b.persistent_applies()
    eval_ms = None
    if persistent:
        # the timed evaluations are one persistent launch each: its bytes per
        # atom are the compact row and count read by both passes (2 (4 n + 4)),
        # the positions and cell order read into the records (24 + 4), the cell
        # order again per pass (8), rho, F, F' out (24), F read back (8), the
        # force (24) and the force-routine energy (8) out
        et = [b.eval_times() for _ in range(5)]
        eval_ms = {k: float(np.median([t[k] for t in et])) for k in ("current", "rebuilt")}
        bpa_p = 8 * n_row + 8 + 28 + 8 + 24 + 8 + 24 + 8
        achieved = bpa_p * b.ntot / (eval_ms["current"] / 1000.0) / 1e9
        roofline = {"bound": "hbm", "kernel": "batch_eval (persistent: list check, records in shared memory, "
                                              "density, forces, per-system sums)",
                    "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": None, "algorithmic_bytes_per_launch": bpa_p * b.ntot,
                    "avg_launch_ms": eval_ms["current"]}
        # the DRAM bytes of one launch on this workload, from an ncu capture
        # (profiles/batch_kernels_1024_supercells.md)
        tb = ((load_traffic() or {}).get("batch") or {}).get("kernels", {}).get("batch_eval")
        if tb and tb.get("atoms") == b.ntot:
            roofline["traffic"] = float(tb["dram_bytes_per_launch"])
    else:
        bpa = {"density": 4 * n_row + 4 + 32 + 32, "forces": 4 * n_row + 4 + 32 + 8 + 8 + 24 + 8 + 48}
        dom = max(("density", "forces"), key=lambda k: ktimes[k])
        achieved = bpa[dom] * b.ntot / (ktimes[dom] / 1000.0) / 1e9
        roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                    "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                    "algorithmic_bytes_per_launch": bpa[dom] * b.ntot, "avg_launch_ms": ktimes[dom]}
    b.set_energy_calc(True)
    b.force()
    ecalc_ms = max_over_ranks(timed(force, min(steps, 50)))
    b.set_energy_calc(False)
    b.force()

    # the other precision on the same lists, and the mixed path's errors
    # against the FP64 path (real forces, energy_calc energy per atom, stress)
    def snapshot():
        out = b.force()
        return b.split(b.forces()), out
    other = "fp64" if prec == "mixed" else "mixed"
    b.set_precision(other)
    b.set_gather(best_gather[other])
    b.force()
    other_ms = max_over_ranks(timed(force, min(steps, 50)))
    # the timed path (energy_calc off: the persistent launch in mixed
    # precision where it applies) against the FP64 path, then the per-pass
    # path with energy_calc's energies
    def errors(res_):
        (f64, o64), (fmx, omx) = res_["fp64"], res_["mixed"]
        d = np.concatenate([(x - y) @ w.b0.T for w, x, y in zip(ws, fmx, f64)])
        return {
            "force_rms_eV_per_A": float(np.sqrt(np.mean(np.sum(d * d, axis=1)))),
            "force_max_eV_per_A": float(np.max(np.linalg.norm(d, axis=1))),
            "pe_calc_max_abs_eV_per_atom": float(np.max(np.abs(omx["pe_calc"] - o64["pe_calc"]) / b.natoms)),
            "pe_max_abs_eV_per_atom": float(np.max(np.abs(omx["pe"] - o64["pe"]) / b.natoms)),
            "stress_max_abs_GPa": float(np.max(np.abs(omx["tp"] - o64["tp"]) / o64["vol"][:, None, None])
                                        * 160.2176),
        }
    res = {p_: None for p_ in ("fp64", "mixed")}
    res[other] = snapshot()
    b.set_precision(prec)
    b.set_gather(best_gather[prec])
    res[prec] = snapshot()
    accuracy = {"vs": "FP64 GPU path (bit-matched to the oracle at 1e-10)",
                "timed_path": {"persistent": b.persistent_applies(), **errors(res)}}
    b.set_energy_calc(True)
    res = {p_: None for p_ in ("fp64", "mixed")}
    b.set_precision(other)
    b.set_gather(best_gather[other])
    res[other] = snapshot()
    b.set_precision(prec)
    b.set_gather(best_gather[prec])
    res[prec] = snapshot()
    accuracy["per_pass_with_energy_calc"] = errors(res)
    b.set_energy_calc(False)

    # end to end: positions from pinned host memory, one evaluation, forces and
    # per-system results back, every step
    x = torch.empty((b.ntot, 3), dtype=torch.float64, pin_memory=True).numpy()
    x[:] = b.get_state()

    fxyz = torch.empty((b.ntot, 3), dtype=torch.float64, pin_memory=True).numpy()

    def e2e_step():
        b.set_positions(x)
        force()
        b.forces_xyz_into(fxyz)

    e2e = None
    if not args.no_e2e:
        e2e_ms = max_over_ranks(timed(e2e_step, min(steps, 20)))
        e2e = {"value": ntot_all / (e2e_ms / 1000.0), "unit": "atom-evals/s", "h2d_bytes_per_step": 24 * b.ntot,
               "d2h_bytes_per_step": 24 * b.ntot + 104 * len(ws), "ms": e2e_ms}

    # the quench of every supercell to max |F| <= 1e-4 eV/A (criterion of the
    # benchmark) from the starting positions; untimed sweep of the list skin,
    # then a fresh timed quench with the best
    def run_quench(skin):
        b.set_skin(skin)
        b.set_state(x, boxes)
        st0 = b.list_stats()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        q = b.quench(maxfn=2000, criterion=1, fmax=1e-4)
        e1.record(stream)
        e1.synchronize()
        st1 = b.list_stats()
        return q, max_over_ranks(e0.elapsed_time(e1)), st1["builds"] - st0["builds"], \
            st1["evaluations"] - st0["evaluations"]

    quench = None
    if not args.no_quench:
        skin_ms = {}
        b.set_gather(best_gather["fp64"])
        for sk in (0.0, 0.3, 0.6):
            skin_ms[sk] = run_quench(sk)[1]
        best_skin = min(skin_ms, key=skin_ms.get)
        # the quench evaluates in FP64 (its line search compares energies below
        # FP32 resolution) with the FP64 passes' best gather
        q, qms, qbuilds, qevals = run_quench(best_skin)
        b.set_gather(best_gather[prec])
        # every rank's systems, at their global indices (one all-gather)
        from moldy_b200.batch import gather_system_results
        shards = shard_configs([w.nm for w in ws_all], world)
        q = gather_system_results({k: q[k] for k in ("iflag", "fmax", "nfev", "f")}, shards, len(ws_all))
        natoms_all = np.array([w.nm for w in ws_all])
        rounds = int(q["nfev"].max())
        quench = {"seconds": qms / 1000.0, "systems": int(len(ws_all)), "converged": int((q["iflag"] == 0).sum()),
                  "cg_error_returns": int((q["iflag"] == 2).sum()), "max_function_values": rounds,
                  "median_function_values": float(np.median(q["nfev"])),
                  "systems_per_s": len(ws_all) / (qms / 1000.0),
                  "atom_evals_per_s": float((q["nfev"] * natoms_all).sum()) / (qms / 1000.0),
                  "max_force_eV_per_A": float(q["fmax"].max()), "skin_A": best_skin, "skin_sweep_ms": skin_ms,
                  "list_builds_per_system_evaluation": qbuilds / max(qevals, 1),
                  "precision": "fp64 (line search needs it; force() runs " + prec + ")"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = batch_cpu_baseline(ws_all, args.cpu_seconds)
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": BATCH_METRIC, "value": value, "unit": "atom-evals/s", "n_gpus": world, "steps": steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms_max, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "f32 arithmetic / f64 accumulate" if prec == "mixed" else "f64",
        "data": "synthetic (seeded strained bcc Fe supercells, Gaussian displacements 0.1 A)",
        "config": {"workload": f"{len(ws_all)} bcc Fe supercells, n ~ U{{4..16}}, strain +/-2%",
                   "atoms": ntot_all, "tile_lanes_per_atom": tunes[prec]["chosen"]["lanes"],
                   "gather": best_gather[prec], "autotune": tunes,
                   "timed_step": "one evaluation of every system with its list current: the force "
                                 "routine's energy, forces and virial (energy_calc off)",
                   "precision": prec, f"{other}_ms_per_step": other_ms,
                   "with_energy_calc_ms_per_step": ecalc_ms,
                   "evaluation_with_every_list_built_ms": build_ms,
                   "persistent_evaluation": persistent, "atom_lanes": tunes[prec]["chosen"].get("atom_lanes"),
                   "persistent_eval_ms": eval_ms,
                   "per_pass_kernel_ms": ktimes, "row_entries_per_atom": n_row,
                   "parallelism": f"supercells sharded over {world} rank(s) by atom count",
                   "l2": "per-evaluation working set (positions, cell order, forces, energies, virial) "
                         "> 126 MB L2"},
        "e2e": e2e,
        "quench": quench, "accuracy": accuracy, "cpu_baseline": cpu, "clocks": clk.summary(), "gpu_launches": launches,
        "roofline": roofline,
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------- adjoint --
ADJ_METRIC = "configs/s, force-matching loss and its knot gradient over 256 bcc Fe configurations of 1024 atoms"


def run_adjoint(args):
    import torch
    from moldy_b200 import FE_FE, MoldySystem
    from moldy_b200 import adjoint as adj
    from moldy_b200 import workloads as wl
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    ws_all = wl.config_adjoint(nconf=args.nconf)
    mine = adj.shard_configs([w.nm for w in ws_all], world)[rank]
    ws = [ws_all[i] for i in mine]
    s = MoldySystem.from_workload(ws[0], device=local_rank)
    stream = torch.cuda.ExternalStream(s.stream_handle(), device=local_rank)
    refs = []
    for w in ws:                                  # untimed: F, sigma at theta0
        s.set_state(x0=w.x0, b0=w.b0)
        _, f0, s0, _ = adj._evaluate(s)
        refs.append((f0, s0))
    rng = np.random.default_rng(7)
    theta = {k: torch.tensor(np.asarray(getattr(FE_FE, k)) * (1 + 1e-3 * rng.normal(size=len(getattr(FE_FE, k)))),
                             requires_grad=True) for k in adj.KNOT_NAMES}

    from moldy_b200 import MoldyBatch
    # the headline path: every configuration of this rank in one MoldyBatch,
    # positions, boxes and references on the device once (untimed); a pass is
    # the tables from the knots (host), one FP64 evaluation of all systems, the
    # loss and the table adjoint on the device, the knot contraction (host)
    # and the all-reduce of the knot gradient
    b = MoldyBatch.from_workloads(ws, device=local_rank)
    b.set_references([f for f, _ in refs], [sg for _, sg in refs])
    bstream = torch.cuda.ExternalStream(b.stream_handle(), device=local_rank)

    def one_pass():
        for t in theta.values():
            t.grad = None
        loss = adj.batch_force_matching_knots(b, theta)
        loss.backward()
        grads = [theta[k].grad for k in adj.KNOT_NAMES]
        adj.allreduce_gradients(grads)
        return loss.detach()

    for _ in range(max(args.warmup, 3)):
        one_pass()
    reps = max(1, min(args.steps, 50))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        e0.record(bstream)
        for _ in range(reps):
            loss_b = one_pass()
        e1.record(bstream)
        e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    g_batch = {k: theta[k].grad.numpy().copy() for k in adj.KNOT_NAMES}

    # beside it: the per-configuration engines (one MoldySystem per host
    # thread, each configuration uploaded, evaluated and differentiated alone)
    configs = [(w.x0, w.b0) for w in ws]
    systems = [s] + [MoldySystem.from_workload(ws[0], device=local_rank) for _ in range(args.adj_engines - 1)]

    def engine_pass():
        for t in theta.values():
            t.grad = None
        loss = adj.force_matching_knots(systems, configs, refs, theta)
        loss.backward()
        grads = [theta[k].grad for k in adj.KNOT_NAMES]
        adj.allreduce_gradients(grads)
        return loss.detach()

    engine_pass()
    e0.record(stream)
    loss_e = engine_pass()
    e1.record(stream)
    e1.synchronize()
    ms_engines = e0.elapsed_time(e1)
    g_eng = {k: theta[k].grad.numpy() for k in adj.KNOT_NAMES}
    agree = max(float(np.max(np.abs(g_batch[k] - g_eng[k])) / max(np.linalg.norm(g_eng[k]), 1e-300))
                for k in adj.KNOT_NAMES)
    if world > 1:
        t = torch.tensor([ms_engines], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_engines = float(t.item())
    value = len(ws_all) / (ms / 1000.0)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        oracle.build()
        nthreads = oracle.max_threads()
        t0 = time.perf_counter()
        nev = 0
        o = oracle.from_workload(ws_all[0], uselookup=True, threads=nthreads)
        while time.perf_counter() - t0 < min(args.cpu_seconds, 10.0):
            o.set_fetm(FE_FE.av, FE_FE.rv, FE_FE.ap, FE_FE.rp)
            o.set_lookup(True, 5000)
            o.ntc = 0
            o.force()
            nev += 1
        el = time.perf_counter() - t0
        cpu = {"value": nev / el / 33.0, "unit": "configs/s", "cores": nthreads, "kind": "port",
               "sample": f"{nev} oracle force evaluations (tables rebuilt, list rebuilt) of one 1024-atom "
                         f"configuration in {el:.1f} s; a knot gradient by central differences needs 33 "
                         "evaluations per configuration (the reference has no adjoint)"}
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0
    n = len(ws_all)
    line = {
        "metric": ADJ_METRIC, "value": value, "unit": "configs/s", "n_gpus": world, "steps": reps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded bcc Fe, T ~ U(300,1800) K displacements, strains +/-3%)",
        "config": {"workload": f"{n} bcc Fe configurations of 1024 atoms (8^3 cells)",
                   "path": "one MoldyBatch of all configurations (moldy_gpu_batch_force_matching)",
                   "parameters": "16 Fe-Fe knots (av, rv, ap, rp)", "loss": "sum |F - F0|^2 + |sigma - sigma0|^2",
                   "precision": "fp64"},
        "e2e": {"value": value, "unit": "configs/s", "h2d_bytes_per_step": 6 * 5001 * 12,
                "d2h_bytes_per_step": n * 8 + 6 * 5001 * 8,
                "note": "the timed pass is the user-facing call: tables built on the host and uploaded, loss and "
                        "table gradients copied back, knot contraction on the host; positions and references "
                        "stay on the device between passes"},
        "per_configuration_engines": {"value": len(ws_all) / (ms_engines / 1000.0), "unit": "configs/s",
                                      "engines_per_rank": args.adj_engines,
                                      "knot_gradient_max_rel_diff_vs_batch": agree},
        "cpu_baseline": cpu, "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------- small --
SMALL_METRIC = "atom-steps/s, 2000-atom bcc Fe NVE at 300 K, 100 steps (the reference's CPU-runnable case)"


def run_small(args):
    """The reference's own CPU-sized case (10^3 bcc cells, NVE, 100 steps): the
    oracle on all host threads, then each GPU path from the same start, timed
    (after a warm-up on a second copy) and compared with the oracle's final
    positions and total energy.  One GPU; other ranks exit."""
    import oracle
    import torch
    from moldy_b200 import MoldySystem
    from moldy_b200 import workloads as wl
    rank, local_rank, world = dist_env()
    if rank != 0:
        return 0
    torch.cuda.set_device(local_rank)
    w = wl.config_small_nve()
    nsteps = 100
    oracle.build()
    nth = oracle.max_threads()
    o = oracle.from_workload(w, uselookup=True, threads=nth)
    o.md_init()
    t0 = time.perf_counter()
    th_o = [o.md_step() for _ in range(nsteps)]
    el_o = time.perf_counter() - t0
    xo = o.get_state()["x0"]
    o.close()
    dt_ps = w.meta["dt_fs"] / 1000.0
    t = np.arange(nsteps) * dt_ps

    def drift(te):
        return float(np.polyfit(t, np.asarray(te) / w.nm, 1)[0])

    paths = {}
    clk_summary = None
    for prec in ("fp64", "mixed"):
        s = MoldySystem.from_workload(w, precision=prec, device=local_rank)
        s.linkup()
        s.md_init()
        th = s.md_steps(nsteps, thermo=True)
        xg = s.get_state()["x0"]
        s.close()
        d = (xg - xo) - np.round(xg - xo)
        pos_err = float(np.max(np.linalg.norm(d @ w.b0.T, axis=1)))
        te_err = float(max(abs(a["te"] - b["te"]) for a, b in zip(th, th_o)) / w.nm)
        s = MoldySystem.from_workload(w, precision=prec, device=local_rank)
        s.linkup()
        s.md_init()
        s.md_steps(max(args.warmup, 3), thermo=False)
        stream = torch.cuda.ExternalStream(s.stream_handle(), device=local_rank)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local_rank) as clk:
            torch.cuda.synchronize()
            e0.record(stream)
            s.md_steps(nsteps, thermo=False)
            e1.record(stream)
            e1.synchronize()
        ms = e0.elapsed_time(e1)
        launches = int(sum(n for _, n in s.kernel_stats().values()))
        s.close()
        paths[prec] = {"value": w.nm * nsteps / (ms / 1000.0), "ms_per_step": ms / nsteps,
                       "max_position_err_A_after_100_steps": pos_err, "max_te_err_eV_per_atom": te_err,
                       "nve_drift_eV_per_atom_per_ps": drift([a["te"] for a in th]), "clocks": clk.summary()}
        clk_summary = clk.summary()
    m = paths["mixed"]
    line = {
        "metric": SMALL_METRIC, "value": m["value"], "unit": UNIT, "n_gpus": 1, "steps": nsteps,
        "warmup": max(args.warmup, 3), "ms_per_step": m["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded bcc Fe lattice, Gaussian displacements 0.05 A, Maxwell-Boltzmann velocities)",
        "config": {"workload": w.name, "atoms": w.nm, "ensemble": "NVE", "dt_fs": w.meta["dt_fs"],
                   "nbrupdate": w.ntcm, "precision": "mixed", "paths": paths,
                   "note": "2000 atoms fill a few SMs: the step time is launch latency, not bandwidth"},
        "e2e": None,
        "cpu_baseline": {"value": w.nm * nsteps / el_o, "unit": UNIT, "cores": nth, "kind": "port",
                         "sample": f"the same {nsteps} steps by the oracle, {nth} OpenMP threads, {el_o:.2f} s",
                         "nve_drift_eV_per_atom_per_ps": drift([a["te"] for a in th_o])},
        "clocks": clk_summary, "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ liquid --
LIQ_METRIC = "atom-steps/s, 1.024M-atom bcc Fe heated 300 -> 2500 K (NPT, scalev every fs, nbrupdate 20)"


def run_liquid(args):
    import torch
    from moldy_b200 import MoldySystem
    from moldy_b200 import workloads as wl
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    w = wl.config_liquid(n=80, seed=5 + rank, temperature=300.0)
    prec = "mixed" if args.precision in ("both", "mixed") else "fp64"
    sysm = MoldySystem.from_workload(w, precision=prec, device=local_rank)
    sysm.linkup()
    sysm.md_init()
    sysm.autotune(nreps=3)
    stream = torch.cuda.ExternalStream(sysm.stream_handle(), device=local_rank)
    loops, nose = 22, 10.0
    per_loop = max(1, args.steps // loops) if args.steps != 1000 else 909
    sysm.md_steps(max(args.warmup, 3), thermo=False)
    sysm.reset_kernel_stats()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        recs, t_end = sysm.strainloops(loops, per_loop, temprq=300.0, tempsp=100.0, nose=nose, thermo=True)
        e1.record(stream)
        e1.synchronize()
        if world > 1:
            torch.distributed.barrier()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    nsteps = loops * per_loop
    value = world * w.nm * nsteps / (ms / 1000.0)
    launches = int(sum(n for _, n in sysm.kernel_stats().values()))
    temps = [r["temp"] for r in recs]
    # final segment without the thermostat: drift of the conserved quantity
    # th = ke + pe + P V + box KE (per atom per ps), both precisions from the same state
    drift = {}
    if rank == 0 and not args.no_accuracy:
        st = sysm.get_state()
        for p2 in ("fp64", "mixed"):
            s2 = MoldySystem.from_workload(w, precision=p2, device=local_rank)
            s2.set_state(st["x0"], st["x1"], st["x2"], st["b0"], st["b1"], st["b2"], tgid=st["tgid"])
            s2.linkup()
            s2.md_init()
            th = np.array([r["th"] for r in s2.md_steps(args.nve_steps)]) / w.nm
            t = np.arange(len(th)) * (w.meta["dt_fs"] / 1000.0)
            drift[p2] = {"slope_eV_per_atom_per_ps": float(np.polyfit(t, th, 1)[0]),
                         "range_eV_per_atom": float(th.max() - th.min())}
            s2.close()
    sysm.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": LIQ_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": nsteps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms / nsteps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if prec == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": w.name, "atoms": w.nm, "loops": loops, "steps_per_loop": per_loop,
                   "temprq_K": [300.0 + 100.0, t_end], "nose": nose, "nbrupdate": w.ntcm,
                   "precision": prec, "ensemble": "NPT Parrinello-Rahman, P=0 GPa"},
        "temperature_K": {"first_100_mean": float(np.mean(temps[:100])), "last_100_mean": float(np.mean(temps[-100:]))},
        "final_segment_drift": drift, "clocks": clk.summary(), "gpu_launches": launches,
        "e2e": None, "roofline": None, "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------- rdf --
RDF_METRIC = "atoms/s, rdf(500, 50) + Ackland-Jones of the 2M-atom bcc Fe cell"


def rdf_cpu_baseline(seconds):
    """The oracle's rdf (half list) + fourth-neighbour radius + Ackland-Jones
    on a bounded sample: 40^3-cell bcc Fe (128,000 atoms), all host threads."""
    import oracle
    from moldy_b200 import workloads as wl
    oracle.build()
    nthreads = oracle.max_threads()
    w = wl.make_workload(40, sigma=0.05, temperature=1200.0, ivol=0, seed=1)
    o = oracle.from_workload(w, uselookup=True, threads=nthreads)
    o.linkup()
    o.update_neighbourlist()
    t0 = time.perf_counter()
    reps = 0
    while True:
        h = o.rdf(500, 50, mode=0)
        rn = oracle.Oracle.rneighbour(h["hist"], h["natoms"], 50)
        o.ackland_jones(rn, mode=0)
        reps += 1
        if time.perf_counter() - t0 >= min(seconds, 10.0) or reps >= 20:
            break
    el = time.perf_counter() - t0
    return {"value": reps * w.nm / el, "unit": "atoms/s", "cores": nthreads, "kind": "port",
            "sample": f"{reps} analyses of a 40^3-cell bcc Fe box ({w.nm} atoms, list already built), "
                      f"{nthreads} OpenMP threads, {el:.1f} s"}


def run_rdf(args):
    """analysis_m::rdf(500, 50) on the 2M-atom cell after its list build: the
    half-list histogram, the fourth-neighbour radius and the Ackland-Jones
    class of every atom, each step through the public API with the results
    copied to the host; the all-pairs form (r < 10.02 A) is timed beside it."""
    import torch
    from moldy_b200 import MoldySystem, analysis
    from moldy_b200 import workloads as wl
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    w = wl.make_workload(args.n, sigma=0.05, temperature=1200.0, ivol=0, seed=1 + rank)
    s = MoldySystem.from_workload(w, device=local_rank)
    s.linkup()
    s.update_neighbourlist()
    stream = torch.cuda.ExternalStream(s.stream_handle(), device=local_rank)

    def step():
        h = analysis.rdf(s, 500, 50, "list")
        rn = analysis.rneighbour(h["hist"], h["natoms"], 50)
        return analysis.ackland_jones(s, rn, "list", with_chi=False)

    def timed(fn, reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    for _ in range(max(args.warmup, 3)):
        out = step()
    steps = max(1, min(args.steps, 50))
    s.reset_kernel_stats()
    with ClockSampler(local_rank) as clk:
        barrier()
        ms = max_over_ranks(timed(step, steps))
        barrier()
    stats = s.kernel_stats()
    launches = int(sum(n for _, n in stats.values()))
    hist_ms = max_over_ranks(timed(lambda: analysis.rdf(s, 500, 50, "list"), steps))
    all_ms = max_over_ranks(timed(lambda: analysis.rdf(s, 500, 50, "all"), min(steps, 5)))
    _, numn = s.neighbour_list()
    n_half = float(np.mean(numn))
    # algorithmic DRAM bytes of one histogram pass: the half-list row and its
    # count, the own position and atomic number (neighbour positions stay in L2)
    bpa = 4.0 * n_half + 4 + 32 + 4
    peak, peak_kind = load_peaks()
    achieved = bpa * w.nm / (hist_ms / 1000.0) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = rdf_cpu_baseline(args.cpu_seconds)
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0
    value = world * w.nm / (ms / 1000.0)
    line = {
        "metric": RDF_METRIC, "value": value, "unit": "atoms/s", "n_gpus": world, "steps": steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 distances, integer counts",
        "data": "synthetic (seeded bcc Fe lattice, Gaussian displacements 0.05 A)",
        "config": {"workload": f"bcc_fe_{w.nm}_rdf_500_50", "atoms": w.nm, "rnear_A": w.rnear,
                   "neighbours_half_mean": n_half, "parallelism": "replicas",
                   "timed_step": "histogram over the half list + fourth-neighbour radius + Ackland-Jones, "
                                 "results copied to the host",
                   "histogram_ms": hist_ms, "all_pairs_histogram_ms": all_ms,
                   "bcc_fraction": float(np.mean(out["aj"] == 1)),
                   "l2": "inputs larger than L2 (half list 4 n_half B/atom > 126 MB)"},
        "e2e": {"value": value, "unit": "atoms/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 501 * 8 + 8 + 8 + 8 * w.nm,
                "note": "each step is the public analysis call with its results copied back"},
        "roofline": {"bound": "hbm", "kernel": "k_rdf_list", "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                     "algorithmic_bytes_per_launch": bpa * w.nm, "avg_launch_ms": hist_ms},
        "cpu_baseline": cpu, "clocks": clk.summary(), "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)
    s.close()
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "liquid":
        return run_liquid(args)
    if args.workload == "rdf":
        return run_rdf(args)
    if args.workload == "small":
        return run_small(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
