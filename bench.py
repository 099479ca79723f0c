#!/usr/bin/env python3
"""Benchmark of the grid-integration Fock build (XC build of (H2O)_n, PBE).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl nkx|reference]
                    [--waters 64] [--precision auto|fp64|mixed]

A step is one Fock build (one SCF iteration's XC work: collocation, density,
functional, V_xc = Phi Z^T) over the whole synthetic (H2O)_n grid
(Treutler-Ahlrichs 75 radial x Lebedev 302 per atom, Becke, 256-point
batches, screening 1e-10), with the orbital coefficients already resident in
HBM.  `e2e` is the same build through the public API with page-locked host
buffers (C and occ copied in, V and E copied out inside the timed region).  One JSON line is
printed by rank 0.  With N > 1 the grid is split into Morton-contiguous,
cost-balanced batch ranges (one process per GPU, shard.balanced_split) and
the partial V_xc and E_xc are summed with an NCCL all-reduce inside the
timed region (strong scaling; with --aux the J fit vector is all-reduced
between the two phases of the build).

Beside the headline, `xc_plus_j` reports the mixed vs FP64 XC + fused DF-J
build of (H2O)_32 with the aux basis zeta_k = 0.3*1.8^k up to l = 3
(--j-waters; 0 skips it).

--impl reference times the CPU restatement of the reference's dense
algorithm (the oracle) on a bounded, seeded sample of the same grid on all
host cores, on the same metric.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Fock-build ms/SCF-iter and grid pts/s: mixed vs FP64 on B200 at dE_xc<=1e-6 Eh"
UNIT = "grid_pts/s"
FUNCS = ("GGA_X_PBE", "GGA_C_PBE")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="nkx", choices=["nkx", "reference"])
    ap.add_argument("--waters", type=int, default=64)
    ap.add_argument("--precision", default="auto", choices=["auto", "fp64", "mixed"])
    ap.add_argument("--cpu-sample", type=int, default=8192, help="points in the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--aux", action="store_true",
                    help="add the grid density-fitted J (aux zeta_k = 0.3*1.8^k up to l = 3) fused into V")
    ap.add_argument("--j-waters", type=int, default=32,
                    help="size of the XC + DF-J comparison reported beside the headline (0: skip)")
    ap.add_argument("--grad-waters", type=int, default=16,
                    help="size of the XC nuclear-gradient measurement reported beside the headline (0: skip)")
    ap.add_argument("--aggregate", type=int, default=0,
                    help="instead of water clusters: the C/H/N/O aggregate of this many atoms (1500: ~12000 "
                         "functions, ~3e7 points), closed shell with nocc = electrons / 2")
    ap.add_argument("--no-fp64", action="store_true",
                    help="skip the same-GPU FP64 comparison build (for very large workloads)")
    ap.add_argument("--no-scf", action="store_true",
                    help="skip the water SCF (Slater + VWN5, SCF to 1e-8 Eh) reported beside the headline")
    ap.add_argument("--no-autotune", action="store_true", help="keep the plan's default kernel choices")
    ap.add_argument("--tuning", default=None,
                    help="fixed kernel choices instead of the autotuner, as FockBuilder.set_tuning keywords, "
                         "e.g. v_pair=1,v_warps=8 (the V contraction on CTA pairs)")
    ap.add_argument("--tune-cache", default=None,
                    help="autotuner cache file: choices found there for this device and problem shape are "
                         "applied without timing, new ones are appended (a profiled run then replays the "
                         "choices of a plain run)")
    ap.add_argument("--aggregate-gate", type=int, default=1500,
                    help="also time and gate the mixed vs FP64 build of the C/H/N/O aggregate of this many atoms "
                         "beside the headline (0: skip)")
    ap.add_argument("--workspace-mb", type=int, default=0,
                    help="cap on the per-chunk collocation workspace in MiB (0: automatic); more chunks, same work")
    return ap.parse_args()


def workload(n, aggregate=0):
    from nukexc_b200 import molecules as M
    if aggregate:
        c, Z = M.aggregate(aggregate, seed=0)
        funcs = M.aggregate_basis(c, Z)
        C = M.random_orbitals(len(funcs), sum(Z) // 2, seed=0)
        return c, Z, funcs, C
    c, Z = M.water_cluster(n, seed=0)
    funcs = M.sto_basis(c, Z)
    C = M.random_orbitals(len(funcs), 5 * n, seed=0)
    return c, Z, funcs, C


def config(args, extra=None):
    agg = getattr(args, "aggregate", 0)
    if agg:
        cfg = {"workload": f"C/H/N/O aggregate, {agg} atoms (3:5:1:1, random packing, d_min 1.0 A) PBE XC Fock build",
               "atoms": agg,
               "basis": "even-tempered STO, heavy 3s2p1d zeta_k=1.4*2.4^k, H 2s zeta_k=1.2*2.4^k",
               "grid": "Treutler-Ahlrichs M4 75 x Lebedev 302 per atom, Becke (Laqua clamp), w>1e-15",
               "batch_points": 256, "screen_tol": 1e-10, "nocc": "electrons / 2", "occ": 1.0,
               "l2": "inputs larger than L2 (per-chunk workspace of several GB streamed each step)"}
    else:
        name = f"(H2O)_{args.waters} PBE XC" + (" + DF-J" if getattr(args, "aux", False) else "") + " Fock build"
        cfg = {"workload": name, "waters": args.waters,
               "basis": "even-tempered STO zeta_k=0.5*2.2^k, O 6s4p2d, H 4s2p",
               "grid": "Treutler-Ahlrichs M4 75 x Lebedev 302 per atom, Becke (Laqua clamp), w>1e-15",
               "batch_points": 256, "screen_tol": 1e-10, "nocc": 5 * args.waters, "occ": 1.0,
               "l2": "inputs larger than L2 (per-chunk workspace of several GB streamed each step)"}
    if extra:
        cfg.update(extra)
    return cfg


# ------------------------------------------------------- CPU baseline ----
def cpu_sample(c, Z, funcs, C, npts):
    """Seeded sample of the workload's grid: unpartitioned atom grids from
    the oracle, every k-th point, Becke-partitioned by the oracle."""
    from oracle import oracle as O
    nr = np.full(len(Z), 75, np.int32)
    Rs = np.array([O.radial_scale(z, "ta") for z in Z])
    L = O._lib()
    tot = L.orc_atom_grids(len(Z), np.ascontiguousarray(c).reshape(-1), nr, Rs, 1, 0.6, 29, None, None, None)
    pts = np.zeros((tot, 3))
    w = np.zeros(tot)
    own = np.zeros(tot, np.int32)
    L.orc_atom_grids(len(Z), np.ascontiguousarray(c).reshape(-1), nr, Rs, 1, 0.6, 29,
                     O._ptr(pts), O._ptr(w), O._ptr(own))
    idx = np.random.default_rng(0).choice(tot, size=min(npts, tot), replace=False)
    idx.sort()
    wp = O.becke(c, pts[idx], own[idx], w[idx])
    keep = wp > 1e-15
    return pts[idx][keep], wp[keep], tot, tot * float(keep.mean())


def cpu_baseline(c, Z, funcs, C, npts, reps=1):
    from oracle import oracle as O
    pts, w, tot, est = cpu_sample(c, Z, funcs, C, npts)
    ob = O.make_manual_basis(funcs)
    occ = np.ones(C.shape[1])
    O.xc_build(ob, pts[:256], w[:256], [101, 130], [C], [occ])  # warm-up
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        O.xc_build(ob, pts, w, [101, 130], [C], [occ])
        times.append(time.perf_counter() - t0)
    t = min(times)
    cores = os.cpu_count()
    return {"value": len(pts) / t, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{len(pts)} of {tot} grid points (seeded uniform sample, Becke-partitioned), "
                      f"full dense XC build on them, {t:.2f} s, OMP threads={cores}",
            "sample_seconds": t, "full_grid_points_estimate": est}


# ------------------------------------------------------------- clocks ----
class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def fp64_gemm_peak(torch):
    """cuBLAS DGEMM throughput (TFLOP/s), the FP64 denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e30
    for _ in range(3):
        e0.record()
        a @ b
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2 * n ** 3 / (best * 1e-3) / 1e12


def int8_gemm_peak(torch):
    """cuBLAS int8 GEMM throughput (TOP/s) measured in this run: the int8
    tensor-core denominator (the peaks file holds bf16 only).  None if the
    library call is unavailable."""
    try:
        n = 8192
        a = torch.randint(-128, 128, (n, n), dtype=torch.int8, device="cuda")
        b = torch.randint(-128, 128, (n, n), dtype=torch.int8, device="cuda").t().contiguous().t()
        for _ in range(5):
            torch._int_mm(a, b)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = 1e30
        for _ in range(12):
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
        return 2 * n ** 3 / (best * 1e-3) / 1e12
    except Exception:
        return None


def measured_traffic(workload, pairs_per_launch=None):
    """DRAM bytes per launch of the dominant kernel from the committed ncu capture
    of this workload (profiles/roofline_traffic.json), scaled by the pairs a
    launch covers in this run when the chunking differs from the capture's
    (the traffic of a V launch grows in proportion to its chunk), or None."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    if d.get("workload") != workload:
        return None
    t = d["dram_bytes_per_launch"]
    if pairs_per_launch and d.get("pairs_per_launch"):
        t *= pairs_per_launch / d["pairs_per_launch"]
    return t


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


# ---------------------------------------------------------- reference ----
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    c, Z, funcs, C = workload(args.waters, args.aggregate)
    npts = max(256, args.cpu_sample)
    for _ in range(args.warmup):
        cpu_baseline(c, Z, funcs, C, 512)
    runs = [cpu_baseline(c, Z, funcs, C, npts) for _ in range(args.steps)]
    v = float(np.median([r["value"] for r in runs]))
    cb = dict(runs[-1])
    cb["value"] = v
    # a step is the bounded sample (its own measured time); the time of one
    # whole-grid build at the sampled rate is reported beside it, flagged as
    # an extrapolation
    ms = 1e3 * float(np.median([r["sample_seconds"] for r in runs]))
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
            "step": "one dense XC build over a bounded seeded sample of the workload's grid points",
            "full_grid_ms_per_build": {"value": cb["full_grid_points_estimate"] / v * 1e3, "extrapolated": True,
                                       "how": "whole-grid point count / sampled points per second"},
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": config(args, {"precision": "fp64 (CPU oracle port of the reference dense algorithm)"}),
            "cpu_baseline": cb, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def xc_plus_j(n, steps, warmup, stream):
    """Mixed vs FP64 XC + fused DF-J Fock build on (H2O)_n with the aux basis
    zeta_k = 0.3*1.8^k up to l = 3 (CUDA events, device-resident C)."""
    import torch
    from nukexc_b200 import api as A
    from nukexc_b200 import molecules as M
    c, Z, funcs, Cm = workload(n)
    g = A.make_flat_grid(c, Z, 75, 29, weight_threshold=1e-15, radial="ta")
    t0 = time.perf_counter()
    fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs), (g.quad_points, g.weights),
                       aux=A.make_manual_basis(M.aux_basis(c, Z)), func_ids=FUNCS)
    setup = time.perf_counter() - t0
    Cd = torch.as_tensor(Cm, device="cuda")
    od = torch.ones(Cm.shape[1], dtype=torch.float64, device="cuda")
    out = {"workload": f"(H2O)_{n} PBE XC + DF-J Fock build", "npoints": int(len(g.weights)),
           "nbf": len(funcs), "naux": fb.naux, "plan_setup_s": setup}
    for prec in ("mixed", "fp64"):
        for _ in range(warmup):
            fb.build([Cd], [od], precision=prec, fuse_j=True, stream=stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            fb.build([Cd], [od], precision=prec, fuse_j=True, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        out[prec + "_ms_per_step"] = e0.elapsed_time(e1) / steps
        out[prec + "_coulomb_ms"] = fb.timing()["coulomb_ms"]
    out["mixed_speedup"] = out["fp64_ms_per_step"] / out["mixed_ms_per_step"]
    Em, Vm, Jm = fb.build([Cd], [od], precision="mixed", want_J=True, stream=stream.cuda_stream)
    Ed, Vd, Jd = fb.build([Cd], [od], precision="fp64", want_J=True, stream=stream.cuda_stream)
    out["accuracy"] = {"dE_xc": abs(Em - Ed), "max_abs_dV_xc": float((Vm[0] - Vd[0]).abs().max()),
                       "rel_dJ": float((Jm - Jd).abs().max() / Jd.abs().max())}
    fb.close()
    return out


def xc_gradient_check(n, stream, ngeom=10, ncomp=1, h=1e-4):
    """XC nuclear gradient of (H2O)_n PBE at seeded perturbed geometries (each
    atom + N(0, 0.05 bohr)): FP64 time per gradient and its largest deviation
    from Richardson-extrapolated central differences of the FP64 E_xc of the
    GPU build on a few seeded components (grid rebuilt at each displaced
    geometry, no weight-threshold compaction); the mixed-precision gradient's
    time and its largest deviation from the FP64 gradient."""
    import torch
    from nukexc_b200 import api as A
    from nukexc_b200 import molecules as M
    c0, Z = M.water_cluster(n, seed=0)
    funcs0 = M.sto_basis(c0, Z)
    Cm = M.random_orbitals(len(funcs0), 5 * n, seed=0)
    occ = np.ones(5 * n)
    rng = np.random.default_rng(11)

    def builder(c):
        g = A.make_flat_grid(c, Z, 75, 29, weight_threshold=-1.0, radial="ta")
        return A.FockBuilder(c, Z, A.make_manual_basis(M.sto_basis(c, Z)), g, func_ids=FUNCS)

    def energy(c):
        fb = builder(c)
        E, _, _ = fb.build([Cm], [occ], precision="fp64")
        fb.close()
        return E

    times, times_m, worst, worst_m, comps = [], [], 0.0, 0.0, []
    for k in range(ngeom):
        c = np.asarray(c0, float) + rng.normal(0.0, 0.05, size=np.shape(c0))
        fb = builder(c)
        fb.xc_gradient([Cm], [occ])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        G = fb.xc_gradient([Cm], [occ])
        times.append((time.perf_counter() - t0) * 1e3)
        fb.xc_gradient([Cm], [occ], precision="mixed")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Gm = fb.xc_gradient([Cm], [occ], precision="mixed")
        times_m.append((time.perf_counter() - t0) * 1e3)
        worst_m = max(worst_m, float(np.abs(Gm - G).max()))
        fb.close()
        for _ in range(ncomp):
            a, j = int(rng.integers(len(Z))), int(rng.integers(3))

            def central(hh):
                cp, cm = c.copy(), c.copy()
                cp[a, j] += hh
                cm[a, j] -= hh
                return (energy(cp) - energy(cm)) / (2 * hh)
            fd = (4.0 * central(h / 2) - central(h)) / 3.0
            worst = max(worst, abs(G[a, j] - fd))
            comps.append([k, a, j])
    return {"workload": f"(H2O)_{n} PBE XC nuclear gradient", "geometries": ngeom,
            "ms_per_gradient": float(np.median(times)), "fd_components": comps,
            "max_abs_error_vs_fd": worst, "gate": "<= 1e-5 Eh/bohr",
            "fd": "Richardson-extrapolated central differences, h = 1e-4 and 5e-5 bohr, FP64 GPU E_xc",
            "mixed": {"ms_per_gradient": float(np.median(times_m)), "max_abs_diff_vs_fp64_gradient": worst_m,
                      "note": "orbital values, density and X = C (occ T) from the int8-digit tensor-core "
                              "contractions; pair terms, STO Hessians (e^x to 1e-14) and Becke term in FP64"}}


def aggregate_gate(natoms, stream, int8_peak=None):
    """The 1500-atom workload: the seeded C/H/N/O aggregate (3:5:1:1, random
    packing in a sphere, d_min 1.0 A, ~12000 STO functions, ~3e7 points),
    PBE, nocc = electrons / 2: one warm-up and one timed mixed build, one
    timed FP64 build of the same plan, and the accuracy gate of the mixed
    build against it (|dE_xc| <= 1e-6 Eh, max|dV| <= 1e-7), all on the device
    (CUDA events on the launching stream)."""
    import torch
    from nukexc_b200 import api as A
    c, Z, funcs, Cm = workload(0, natoms)
    t0 = time.perf_counter()
    g = A.make_flat_grid(c, Z, 75, 29, weight_threshold=1e-15, radial="ta")
    fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs), g, func_ids=FUNCS)
    setup = time.perf_counter() - t0
    info = fb.info()
    Cd = torch.as_tensor(Cm, device="cuda")
    od = torch.ones(Cm.shape[1], dtype=torch.float64, device="cuda")
    out = {"workload": f"C/H/N/O aggregate, {natoms} atoms, PBE XC Fock build", "npoints": int(info["npoints"]),
           "nbf": len(funcs), "nocc": int(Cm.shape[1]), "npairs": int(info["npairs"]), "setup_s": setup}

    def timed(prec):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        E, V, _ = fb.build([Cd], [od], precision=prec, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        return E, V[0], e0.elapsed_time(e1), fb.timing()

    fb.build([Cd], [od], precision="mixed", stream=stream.cuda_stream)  # warm-up
    Em, Vm, ms_m, tm = timed("mixed")
    Vm = Vm.clone()
    Ed, Vd, ms_d, td = timed("fp64")
    out.update({"mixed_ms_per_build": ms_m, "mixed_points_per_s": info["npoints"] / (ms_m * 1e-3),
                "mixed_stage_ms": {k: v for k, v in tm.items() if k.endswith("_ms")},
                "v_roofline": v_roofline(fb, tm["vgemm_ms"], int8_peak),
                "launches_per_mixed_build": tm["launches"], "nchunks": int(fb.info()["nchunks"]),
                "fp64_ms_per_build": ms_d, "fp64_stage_ms": {k: v for k, v in td.items() if k.endswith("_ms")},
                "mixed_speedup": ms_d / ms_m,
                "accuracy": {"dE_xc": abs(Em - Ed), "max_abs_dV": float((Vm - Vd).abs().max()), "E_xc_fp64": Ed,
                             "gate": "dE<=1e-6 Eh, max|dV|<=1e-7"}})
    fb.close()
    del Vm, Vd
    torch.cuda.empty_cache()
    return out


def scf_water():
    """Water, Slater + VWN5, TA-M4 75 x Lebedev 302, closed-shell SCF to 1e-8
    Eh with the stand-in driver: on the GPU in FP64 and mixed precision, and
    the same SCF with the CPU oracle (the reference's dense algorithm, all
    host threads)."""
    from nukexc_b200 import api as A
    from nukexc_b200 import molecules as M
    from nukexc_b200 import scf
    from oracle import oracle as O
    xc = ("LDA_X", "LDA_C_VWN")
    c, Z = M.water()
    funcs = M.sto_basis(c, Z)
    aux = M.sto_basis(c, Z, {8: [(0, 6), (1, 5), (2, 4), (3, 2)], 1: [(0, 4), (1, 3), (2, 1)]}, alpha=0.8,
                      beta=2.5)
    enuc = scf.nuclear_repulsion(c, Z)
    out = {"workload": "H2O Slater+VWN5 SCF to 1e-8 Eh, TA-M4 75 x Lebedev 302, grid DF-J (91 aux)",
           "nbf": len(funcs)}
    g = A.make_flat_grid(c, Z, 75, 29, weight_threshold=1e-15, radial="ta")
    b = A.make_manual_basis(funcs)
    fb = A.FockBuilder(c, Z, b, g, aux=A.make_manual_basis(aux), func_ids=xc)
    S, T, V, H = A.compute_core_hamiltonian(b, c, Z, g.quad_points, g.weights)
    for prec in ("fp64", "mixed"):
        r = scf.rks(S.cpu().numpy(), H.cpu().numpy(), scf.gpu_fock(fb, prec), 5, enuc)
        out[prec] = {"energy": r["energy"], "iterations": r["iterations"], "converged": r["converged"],
                     "ms_per_iteration": 1e3 * float(np.median(r["seconds_per_iteration"]))}
    # the same SCF with everything on the device (scf.rks_device), and with
    # the Fock builds replayed from a CUDA graph (nkx_plan_set_graph)
    for prec in ("fp64", "mixed"):
        for graph in (False, True):
            fb.set_graph(graph)
            r = scf.rks_device(S, H, fb, 5, enuc, precision=prec)
            key = f"device_{prec}" + ("_graph" if graph else "")
            out[key] = {"energy": r["energy"], "iterations": r["iterations"], "converged": r["converged"],
                        "ms_per_iteration": 1e3 * float(np.median(r["seconds_per_iteration"]))}
    out["graph_replays"] = fb.info()["graph_replays"]
    fb.set_graph(False)
    fb.close()
    pts, w, _ = O.make_flat_grid(c, Z, 75, 29, weight_threshold=1e-15, scheme="ta")
    ob, oa = O.make_manual_basis(funcs), O.make_manual_basis(aux)
    So, To, Vo = O.core_hamiltonian(ob, c, Z, pts, w)
    Sa = O.aux_metric(oa, pts, w)

    def cpu_fock(Cocc):
        occ = 2.0 * np.ones(Cocc.shape[1])
        E, Vx = O.xc_build(ob, pts, w, [1, 7], [Cocc], [occ])
        J, _ = O.coulomb(ob, oa, pts, w, Cocc, occ, S=Sa)
        return E, Vx[0], J
    r = scf.rks(So, To + Vo, cpu_fock, 5, enuc)
    out["cpu_port"] = {"energy": r["energy"], "iterations": r["iterations"], "converged": r["converged"],
                       "ms_per_iteration": 1e3 * float(np.median(r["seconds_per_iteration"])),
                       "cores": os.cpu_count()}
    out["dE_gpu_fp64_vs_cpu"] = abs(out["fp64"]["energy"] - out["cpu_port"]["energy"])
    out["dE_mixed_vs_fp64"] = abs(out["mixed"]["energy"] - out["fp64"]["energy"])
    return out


# ---------------------------------------------------------------- nkx ----
def v_roofline(fb, vgemm_ms, peak):
    """The V contraction of one mixed build against the int8 peak: ten int8
    MMAs per FP64-equivalent product of sum_b 2 n_b^2 256."""
    ach = 10.0 * vgemm_flops(fb.batch_blocks()) / (vgemm_ms * 1e-3) / 1e12
    return {"achieved": ach, "unit": "TOP/s (int8)", "peak": peak, "frac": (ach / peak) if peak else None}


def vgemm_flops(info_pairs_per_batch, nz=1):
    """Algorithmic FLOPs of the V = Phi Z^T contraction: sum_b 2 n_b^2 256."""
    nb = np.asarray(info_pairs_per_batch, dtype=np.float64) * 128.0
    return float(nz * (2.0 * nb * nb * 256.0).sum())


def run_nkx(args):
    import torch
    from nukexc_b200 import api as A
    from nukexc_b200 import molecules as M  # noqa: F401
    from nukexc_b200 import shard as S

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    c, Z, funcs, Cm = workload(args.waters, args.aggregate)
    g = A.make_flat_grid(c, Z, 75, 29, weight_threshold=1e-15, radial="ta")
    b = A.make_manual_basis(funcs)
    # strong scaling: rank r integrates a Morton-contiguous, cost-balanced
    # range of the grid's 256-point batches
    if world > 1:
        sel = S.balanced_split(g.quad_points, b.center, A.cutoff_radii(b), Cm.shape[1], world)[rank]
    else:
        sel = np.arange(len(g.weights))
    pts, w = g.quad_points[sel], g.weights[sel]
    t0 = time.perf_counter()
    aux = A.make_manual_basis(M.aux_basis(c, Z)) if args.aux else None
    fb = A.FockBuilder(c, Z, b, (pts, w), aux=aux, func_ids=FUNCS, workspace_bytes=args.workspace_mb << 20)
    fuse = bool(args.aux)
    if aux is not None and dist is not None:
        S.shard_metric(fb, dist)  # the whole grid's (A|B), once per geometry
    setup_s = time.perf_counter() - t0
    info = fb.info()
    nbf = len(funcs)
    occ = np.ones(Cm.shape[1])
    Cd = torch.as_tensor(Cm, device="cuda")
    od = torch.as_tensor(occ, device="cuda")
    stream = torch.cuda.current_stream()
    prec = args.precision
    if prec == "auto":
        try:
            fb.build([Cd], [od], precision="mixed", fuse_j=fuse, stream=stream.cuda_stream)
            prec = "mixed"
        except Exception:
            prec = "fp64"
    tuning = None
    if prec == "mixed" and args.tuning:
        kw = {k: int(v) for k, v in (item.split("=") for item in args.tuning.split(","))}
        fb.set_tuning(**kw)
        tuning = dict(fb.tuning(), fixed=True)
    elif prec == "mixed" and not args.no_autotune:
        # the plan's autotuner picks the MMA widths, the Y path and the chunk
        # size by timing whole builds (untimed setup)
        t0 = time.perf_counter()
        tuning = fb.autotune([Cd], [od], cache_path=args.tune_cache, stream=stream.cuda_stream)
        tuning["seconds"] = time.perf_counter() - t0
        info = fb.info()

    # page-locked host buffers of the end-to-end step: C (column-major, as the
    # C-ABI takes it) and occ copied in, V copied out, every step
    pinned = {}

    def host_buffers():
        if not pinned:
            Cp = torch.empty((Cm.shape[1], nbf), dtype=torch.float64, pin_memory=True)
            Cp.copy_(torch.from_numpy(np.ascontiguousarray(Cm.T)))
            op = torch.empty(occ.shape[0], dtype=torch.float64, pin_memory=True)
            op.copy_(torch.from_numpy(occ))
            pinned.update(C=Cp.t(), occ=op, V=torch.empty(nbf * nbf, dtype=torch.float64, pin_memory=True))
        return pinned

    def step(host=False):
        if fuse and dist is not None:
            # J on a sharded grid: density, all-reduce of the fit vector y,
            # then the rest of the build; E and V all-reduced inside
            Cs, os_ = ([Cm], [occ]) if host else ([Cd], [od])
            E, _, _ = S.sharded_build(fb, Cs, os_, dist, precision=prec, want_J=False, fuse_j=True,
                                      stream=stream.cuda_stream)
            return E
        if host:
            hb = host_buffers()
            E, V, _ = fb.build([hb["C"]], [hb["occ"]], precision=prec, fuse_j=fuse, stream=stream.cuda_stream,
                               out_V=hb["V"])
            # the all-reduce of several ranks needs V back on the device
            V = torch.as_tensor(V[0], device="cuda") if dist is not None else V[0]
        else:
            E, V, _ = fb.build([Cd], [od], precision=prec, fuse_j=fuse, stream=stream.cuda_stream)
            V = V[0]
        if dist is not None:
            E, _ = S.allreduce_fock(E, [V], dist)
        return E

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    stage = {}
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
            t = fb.timing()
            launches += t["launches"]
            for k, v in t.items():
                stage[k] = stage.get(k, 0.0) + v
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    if dist is not None:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = tt.item()
        dist.barrier()
    total_pts = len(g.weights)
    value = total_pts / (ms * 1e-3)
    stage_ref = dict(stage)

    # the same-GPU FP64 kernels on the same build, and the accuracy gate
    fp64 = None
    if prec == "mixed" and not args.no_fp64:
        E_m, V_m, _ = fb.build([Cd], [od], precision="mixed", fuse_j=fuse, stream=stream.cuda_stream)
        V_m = V_m[0].clone()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        E_d, V_d, _ = fb.build([Cd], [od], precision="fp64", fuse_j=fuse, stream=stream.cuda_stream)
        f1.record(stream)
        torch.cuda.synchronize()
        fms, nf = f0.elapsed_time(f1), 1
        if args.steps > 1:
            # further FP64 builds timed back to back (the first one above also
            # gives the accuracy reference)
            nf = min(args.steps, 2)
            f0.record(stream)
            for _ in range(nf):
                fb.build([Cd], [od], precision="fp64", fuse_j=fuse, stream=stream.cuda_stream)
            f1.record(stream)
            torch.cuda.synchronize()
            fms = f0.elapsed_time(f1) / nf
        fp64_stage = {k: v for k, v in fb.timing().items() if k.endswith("_ms")}
        if dist is not None:
            tt = torch.tensor([fms], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            fms = tt.item()
        acc = {"dE_xc": abs(E_m - E_d), "max_abs_dV": float((V_m - V_d[0]).abs().max()),
               "E_xc_fp64": E_d, "gate": "dE<=1e-6 Eh, max|dV|<=1e-7"}
        if fuse:
            # V above holds V_xc + J; split them with separate-J builds (untimed)
            E_m2, Vx_m, J_m = fb.build([Cd], [od], precision="mixed", want_J=True, stream=stream.cuda_stream)
            E_d2, Vx_d, J_d = fb.build([Cd], [od], precision="fp64", want_J=True, stream=stream.cuda_stream)
            acc["max_abs_dV"] = float((Vx_m[0] - Vx_d[0]).abs().max())
            acc["max_abs_dV_fused_xc_plus_j"] = float((V_m - V_d[0]).abs().max())
            acc["max_abs_dJ"] = float((J_m - J_d).abs().max())
            acc["max_abs_J"] = float(J_d.abs().max())
            acc["rel_dJ"] = acc["max_abs_dJ"] / max(acc["max_abs_J"], 1e-300)
            acc["note"] = ("the mixed build's J reads the FP32 radial-factor table and the mixed density; "
                           "the FP64 build evaluates the potentials in FP64")
        fp64 = {"ms_per_step": fms, "value": total_pts / (fms * 1e-3), "steps": nf,
                "mixed_speedup": fms / ms, "accuracy": acc, "stage_ms": fp64_stage}

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        for _ in range(2):
            step(host=True)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step(host=True)
        torch.cuda.synchronize()
        em = (time.perf_counter() - t0) * 1e3 / args.steps
        if dist is not None:
            tt = torch.tensor([em], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            em = tt.item()
        e2e = {"value": total_pts / (em * 1e-3), "unit": UNIT, "ms_per_step": em,
               "h2d_bytes_per_step": int(Cm.nbytes + occ.nbytes), "d2h_bytes_per_step": int(nbf * nbf * 8 + 8)}

    if rank == 0:
        flops = vgemm_flops(fb.batch_blocks())
        vg_ms = stage_ref["vgemm_ms"] / args.steps
        peaks, src = measured_peaks()
        if prec == "fp64":
            peak = fp64_gemm_peak(torch)
            peak_note = f"cuBLAS DGEMM 8192^3 measured in this run ({src} peaks file has no FP64 figure)"
        else:
            # the int8 digit contraction executes 10 int8 MMAs per FP64-equivalent
            # product; denominator: cuBLAS int8 GEMM measured in this run, else
            # 2x the bf16 dense rate of the peaks file
            p8 = int8_gemm_peak(torch)
            if p8 is not None and p8 > 2.0 * peaks["bf16_tflops_sustained"]:
                peak = p8
                peak_note = "cuBLAS int8 GEMM 8192^3 measured in this run (torch._int_mm)"
            else:
                peak = 2.0 * peaks["bf16_tflops_sustained"]
                peak_note = f"int8 dense = 2 x bf16 dense sustained ({src} bf16 {peaks['bf16_tflops_sustained']})"
                if p8 is not None:
                    peak_note += f"; cuBLAS int8 GEMM measured {p8:.0f} TOP/s (lower, not used)"
        if prec == "fp64":
            ach, unit = flops / (vg_ms * 1e-3) / 1e12, "TFLOP/s"
        else:
            ach, unit = 10.0 * flops / (vg_ms * 1e-3) / 1e12, "TOP/s (int8)"
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "f64" if prec == "fp64" else "int8 digits (31-bit rows), int32 acc, f64 combine",
            "data": "synthetic",
            "config": config(args, {"precision": prec, "npoints": total_pts, "nbf": nbf,
                                    "nbatches": info["nbatches"], "npairs": info["npairs"],
                                    "nchunks": info["nchunks"], "plan_setup_s": setup_s, "autotune": tuning,
                                    "parallelism": (f"grid split into {world} Morton-contiguous, cost-balanced batch "
                                                    f"ranges, one GPU each; all-reduce of E, V"
                                                    + (" and of the J fit vector y" if fuse else "")
                                                    if world > 1 else "one GPU")}),
            "stage_ms_per_step": {k: v / args.steps for k, v in stage.items() if k.endswith("_ms")},
            "roofline": {"bound": "tensor", "kernel": "vgemm (V = Phi Z^T)", "achieved": ach, "peak": peak,
                         "unit": unit, "frac": ach / peak,
                         "traffic": (measured_traffic(config(args)["workload"], info["npairs"] / max(1, info["nchunks"]))
                                     if prec == "mixed" else None),
                         "traffic_unit": "DRAM bytes per V launch (ncu, profiles/roofline_traffic.json, scaled to "
                                         "this run's pairs per chunk)",
                         "peak_source": peak_note,
                         "algorithmic_flops_per_step": flops,
                         "fp64_equivalent_tflops": flops / (vg_ms * 1e-3) / 1e12},
            "fp64_same_gpu": fp64,
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "e2e": e2e,
        }
        if os.environ.get("NKX_BENCH_NO_CPU") is None and world == 1:
            line["cpu_baseline"] = cpu_baseline(c, Z, funcs, Cm, args.cpu_sample)
        if fp64 is not None:
            # the same-GPU FP64 comparator against its own roofline: its V
            # contraction (same algorithmic flops) against a cuBLAS DGEMM
            # measured in this run
            pd = fp64_gemm_peak(torch)
            v64 = flops / (fp64["stage_ms"]["vgemm_ms"] * 1e-3) / 1e12
            fp64["roofline"] = {"kernel": "vgemm_fp64_kernel (V = Phi Z^T, FP64 CUDA cores)", "achieved": v64,
                                "peak": pd, "unit": "TFLOP/s", "frac": v64 / pd,
                                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (torch.matmul f64)"}
        # the measurements below build plans of their own: the headline plan's
        # device memory (its chunk workspace can hold ~100 GB) is freed first
        fb.close()
        fb = None
        torch.cuda.empty_cache()
        if world == 1 and args.j_waters > 0 and not args.aux:
            line["xc_plus_j"] = xc_plus_j(args.j_waters, max(1, min(args.steps, 3)), args.warmup, stream)
        if world == 1 and args.grad_waters > 0:
            line["xc_gradient"] = xc_gradient_check(args.grad_waters, stream)
        if world == 1 and not args.no_scf:
            line["scf_water"] = scf_water()
        if world == 1 and args.aggregate_gate > 0 and not args.aggregate:
            line["aggregate_gate"] = aggregate_gate(args.aggregate_gate, stream, peak if prec == "mixed" else None)
        print(json.dumps(line), flush=True)
    if fb is not None:
        fb.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_nkx(args)


if __name__ == "__main__":
    main()
