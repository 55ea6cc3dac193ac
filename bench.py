"""Benchmark: Brownian-dynamics steps/s of BD_BOX's Ermak-McCammon step.

Workload (one GPU): a linear bead-spring chain of N=4096 beads (3N=12288),
the chain force field (harmonic bonds, LJ + Debye-Hueckel, cutoff 12 A),
free-space RPY hydrodynamics with Cholesky noise, D and its factor rebuilt
every 10 steps, mixed precision (FP32 tensor and stored D/L, FP16-split
Cholesky updates with FP64 diagonal tiles and FP64 sums). Inputs are
synthetic (seeded self-avoiding walk, seeded charges).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line on rank 0. ``value`` is steps/s of the whole job with
all state resident in HBM (K steps bracketed by a barrier and device
synchronisation, CUDA events on the engine's stream, max over ranks).
``e2e`` drives the same steps through the C ABI with host buffers: each
step copies its 3N Gaussians from pinned host memory and reads the 4N
coordinates back. With N > 1 every rank advances its own independent chain
(replicas; no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_BEADS = 4096
REFRESH = 10
REFRESH_TIMED = 10   # refreshes timed by themselves for the roofline
SEED = 2
METRIC = "BD steps/s at N=4096, mixed vs FP64 GPU at stated error; Cholesky TFLOP/s"


def make_deck(tmp: str, beads: int = N_BEADS):
    from bd_box_b200 import decks
    p = decks.write_chain_deck(tmp, f"chain{beads}", beads, seed=SEED, hydro="cholesky", steps=1000)
    return p, decks.read_deck(p)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
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
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[4 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------- CPU baseline
def reference_cpu(prm_path: str, deck, steps: int, single_thread: bool = True):
    """The reference's own CPU build (oracle/_ref/ref_harness: BD_BOX sources,
    -O3, OpenMP, LAPACK via OpenBLAS) on this host's cores, `steps` steps
    with D and its Cholesky factor rebuilt every REFRESH steps. Falls back to
    the C restatement of the oracle if the reference build is absent."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    cores = os.cpu_count() or 1
    n3 = 3 * deck.n
    d = os.path.dirname(prm_path)
    g = np.random.default_rng(7).standard_normal(n3 * (steps + 1))
    gpath = os.path.join(d, "gauss.bin")
    g.tofile(gpath)
    env = dict(os.environ, BDB_GAUSS_FILE=gpath, OMP_NUM_THREADS=str(cores),
               OPENBLAS_NUM_THREADS=str(cores))
    if os.path.exists(harness):
        def run(mode, threads, *extra):
            e = dict(env, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS=str(threads))
            t0 = time.perf_counter()
            subprocess.run([harness, os.path.basename(prm_path), mode, "out.bin", *extra], cwd=d, env=e, check=True,
                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            return time.perf_counter() - t0

        def rate(threads, reps):
            # start-up (reading the deck, first forces) is timed in its own
            # run of the same process and removed
            out = []
            for _ in range(reps):
                t = run("steps", threads, str(steps), str(REFRESH))
                t_init = run("forces", threads)
                out.append(steps / max(t - t_init, 1e-9))
            return out

        runs = rate(cores, 3)
        single = rate(1, 1)[0] if single_thread else None
        return {"value": float(np.median(runs)), "unit": "steps/s", "cores": cores, "kind": "reference",
                "runs": runs, "statistic": "median of 3 runs", "single_thread_value": single,
                "sample": f"{steps} steps of the N={deck.n} chain with one D build + LAPACK dpotrf per {REFRESH} "
                          f"steps (BD_BOX CPU sources, OpenMP + OpenBLAS, {cores} threads; start-up removed)"}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    o = pyoracle.Oracle(deck)
    t0 = time.perf_counter()
    o.run_steps(steps, g, refresh=REFRESH)
    t = time.perf_counter() - t0
    return {"value": steps / t, "unit": "steps/s", "cores": cores, "kind": "port",
            "sample": f"{steps} steps, oracle restatement (OpenMP {cores} threads)"}


# ------------------------------------------------------------------- GPU
def time_steps(torch, sysm, K, per_call=None):
    """K steps on the engine's stream, `per_call` steps per bdb_step call
    (all K in one call by default: the status word is read once, so the
    host never stalls the stream between steps)."""
    stream = torch.cuda.ExternalStream(sysm.lib.bdb_stream(sysm.h))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    per_call = per_call or K
    torch.cuda.synchronize()
    e0.record(stream)
    done = 0
    while done < K:
        k = min(per_call, K - done)
        sysm.step(k)
        done += k
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def time_refresh(torch, sysm, K):
    """K refreshes of the stored tensor and its factor (bdb_refresh: the
    refresh graph that the timed steps replay every REFRESH steps), CUDA
    events on the engine's stream; ms per refresh."""
    stream = torch.cuda.ExternalStream(sysm.lib.bdb_stream(sysm.h))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    sysm.refresh(K)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / K


def phase(sysm, name):
    import ctypes as C
    tot = C.c_double()
    calls = C.c_longlong()
    sysm._check(sysm.lib.bdb_phase_stats(sysm.h, name.encode(), C.byref(tot), C.byref(calls)))
    return tot.value, calls.value


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), d.get("bf16_tflops_sustained", 1400.0), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


def profile_value(name: str, key: str):
    """A figure recorded in a committed ncu summary (profiles/<name>.md,
    line '<key>: X'), or None."""
    p = os.path.join(ROOT, "profiles", name + ".md")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for ln in f:
            if ln.startswith(key + ":"):
                try:
                    return float(ln.split(":", 1)[1])
                except ValueError:
                    return None
    return None


def profile_traffic(name: str):
    """dram bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/<name>.md, line 'traffic_bytes_per_launch: X')."""
    p = os.path.join(ROOT, "profiles", name + ".md")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for ln in f:
            if ln.startswith("traffic_bytes_per_launch:"):
                try:
                    return float(ln.split(":", 1)[1])
                except ValueError:
                    return None
    return None


def run_ours(args):
    import ctypes as C

    import torch
    from bd_box_b200 import engine

    from bd_box_b200 import ranks

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist, rank, world, local = ranks.init("nccl")
    tmp = tempfile.mkdtemp(prefix="bdb_bench_")
    try:
        prm, deck = make_deck(tmp, args.beads)
        n3 = 3 * deck.n
        sysm = engine.System(deck, precision=engine.PREC_MIXED, refresh=REFRESH,
                             noise=engine.NOISE_PHILOX, seed=ranks.replica_seed(SEED, rank))
        sysm.autotune(True)
        # W warm-up steps, and at least two refreshes plus two steps: the
        # step graph is captured at the second step and the refresh graph
        # at the second refresh, so the timed steps replay both
        warm = max(args.warmup, 2 * REFRESH + 2)
        for _ in range(warm):
            sysm.step(1)
        sysm.lib.bdb_reset_stats(sysm.h)
        ranks.barrier(dist)
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            ms = time_steps(torch, sysm, args.steps)
        launches = C.c_longlong()
        sysm.lib.bdb_launches(sysm.h, C.byref(launches))
        # the refresh (tensor build + factorisation) alone, replayed from the
        # same graph as inside the timed steps: the roofline's launch
        refresh_ms = time_refresh(torch, sysm, REFRESH_TIMED)
        # the same steps as K one-step calls (a host round trip per step)
        ms_single = time_steps(torch, sysm, args.steps, per_call=1)
        # phase breakdown: a separate profiled pass of the same length (CUDA
        # events around every phase; eager launches, no graph replay)
        sysm.lib.bdb_reset_stats(sysm.h)
        sysm.lib.bdb_profile(sysm.h, 1)
        ms_prof = time_steps(torch, sysm, args.steps)
        sysm.lib.bdb_profile(sysm.h, 0)
        ms = ranks.max_over_ranks(dist, ms, "cuda")
        ranks.barrier(dist)
        value = world * args.steps / (ms / 1e3)
        fac_ms, fac_calls = phase(sysm, "factor")
        mv_ms, mv_calls = phase(sysm, "matvec")
        ref_ms, _ = phase(sysm, "refresh")
        bld_ms, bld_calls = phase(sysm, "build")
        frc_ms, frc_calls = phase(sysm, "forces")

        # e2e through the C ABI with host buffers (pinned)
        gh = torch.randn(args.steps * n3, dtype=torch.float64).pin_memory()
        ch = torch.empty(4 * deck.n, dtype=torch.float64).pin_memory()
        hsys = engine.System(deck, precision=engine.PREC_MIXED, refresh=REFRESH,
                             noise=engine.NOISE_HOST, seed=ranks.replica_seed(SEED, rank))
        hsys.autotune(True)   # the same configuration as the device-resident arm
        gp = C.cast(gh.data_ptr(), C.POINTER(C.c_double))
        cp = C.cast(ch.data_ptr(), C.POINTER(C.c_double))
        for k in range(warm):
            hsys.lib.bdb_step(hsys.h, 1, gp)
        ranks.barrier(dist)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(args.steps):
            rc = hsys.lib.bdb_step(hsys.h, 1, C.cast(gh.data_ptr() + 8 * k * n3, C.POINTER(C.c_double)))
            hsys._check(rc)
            hsys._check(hsys.lib.bdb_get_coord(hsys.h, cp))
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        e2e_s = ranks.max_over_ranks(dist, e2e_s, "cuda")
        e2e = {"value": world * args.steps / e2e_s, "unit": "steps/s",
               "h2d_bytes_per_step": 8 * n3, "d2h_bytes_per_step": 8 * 4 * deck.n}
        hsys.close()

        # plain FP64 GPU path (full Cholesky every step, the reference schedule)
        fp64 = None
        if rank == 0 and world == 1 and not args.skip_fp64:
            fp64 = fp64_case(torch, engine, deck, value)

        errors = None
        if rank == 0 and world == 1 and not args.skip_errors:
            errors = accuracy(torch, engine, deck)

        hbm, bf16, bf16s, src = peaks()
        # dominant phase: the refresh (tensor build + Cholesky factorisation,
        # one graph launch every REFRESH steps), timed by itself above
        n = 3 * deck.n
        flops = n ** 3 / 3.0
        fac_avg = fac_ms / max(fac_calls, 1)
        mv_avg = mv_ms / max(mv_calls, 1)
        refreshes_timed = -(-args.steps // REFRESH)
        ach = flops / (refresh_ms / 1e3) / 1e12
        split3 = bf16s / 3.0   # three FP16 MMAs per split product; FP16 runs at the BF16 rate
        roof = {"kernel": "refresh graph: k_build (tensor) + Cholesky factorisation (k_potrf128, k_trsm128, "
                          "k_syrk_tc, k_syrk_tc2); one launch = one refresh of the 12288^2 stored tensor and its "
                          "factor",
                "bound": "tensor", "achieved": ach, "peak": bf16s, "unit": "TFLOP/s", "frac": ach / bf16s,
                "frac_of_split_ceiling": ach / split3,
                "ceiling_split": {"value": split3, "note": "measured bf16 sustained / 3 (three FP16 MMAs per "
                                                           "product of FP16 hi/lo panels; FP16 at the BF16 rate)"},
                "algorithmic_flops_per_launch": flops,
                # one refresh is ~700 launches on three streams: its DRAM bytes
                # are not captured as a whole (a multi-metric capture of that
                # many launches); the per-kernel captures give the parts
                "traffic": None,
                "traffic_parts": {
                    "k_syrk_tc2_bytes_per_launch": profile_traffic("k_syrk_tc2_n12288"),
                    "k_syrk_tc2_tiles_in_that_launch": 1378,
                    "k_build_bytes_per_launch": profile_traffic("k_build_n12288"),
                    "source": "profiles/k_syrk_tc2_n12288.md, profiles/k_build_n12288.md (one kernel, 1-2 "
                              "launches each)"},
                "peak_source": f"{src} bf16 sustained", "ms_per_launch": refresh_ms,
                "launches_in_timed_region": refreshes_timed,
                "timed_region_consistency": {"refresh_ms_x_refreshes": refresh_ms * refreshes_timed,
                                             "timed_ms": ms,
                                             "ok": refresh_ms * refreshes_timed <= ms},
                "share_of_step_time": refresh_ms * refreshes_timed / ms,
                "autotuned_chain_sms": sysm.factor_tuning(),
                # tensor-pipe utilisation of the bulk update (ncu, not live)
                "tensor_pipe": {"kernel": "k_syrk_tc2",
                                "active_pct_of_active_cycles": profile_value("k_syrk_tc2_n12288",
                                                                             "tensor_pipe_active_pct"),
                                "active_pct_of_elapsed": profile_value("k_syrk_tc2_n12288",
                                                                       "tensor_pipe_elapsed_pct"),
                                "source": "profiles/k_syrk_tc2_n12288.md (one ncu capture)"}}
        # diagnostic split from the profiled pass (events around every phase
        # and kernel, eager launches): not the timed configuration
        roof["profiled_pass"] = {
            "phases_ms_per_call": {"factor": fac_avg, "build": bld_ms / max(bld_calls, 1),
                                   "matvec": mv_avg, "forces": frc_ms / max(frc_calls, 1)},
            "factor_kernels_us_per_launch": {
                k: 1e3 * t / max(c, 1) for k, (t, c) in
                ((k, phase(sysm, k)) for k in ("potrf", "trsm", "syrk_col", "syrk_rest"))}}
        roof["matvec"] = {"kernel": "k_strip_mv_tma (D.F + L.X, one pass over the stored matrix)", "bound": "hbm",
                          "achieved": 4.0 * n * n / (mv_avg / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                          "frac": 4.0 * n * n / (mv_avg / 1e3) / 1e9 / hbm, "ms_per_launch": mv_avg,
                          "traffic": profile_traffic("k_strip_mv_tma_n12288"), "peak_source": f"{src} hbm"}
        reps = None
        if not args.skip_replicas:
            # every rank takes part: with N processes the 256 chains are
            # sharded over them (bdb_shard_replicas)
            reps = replicas(torch, engine, max(3, args.steps // 5), 3, dist, rank, world)
        adj = None
        if rank == 0 and world == 1 and not args.skip_adjoint:
            adj = adjoint_case(torch, engine)
        ew = ews = None
        if rank == 0 and world == 1 and not args.skip_ewald:
            ew = ewald_case(torch, engine)
            ews = ewald_case(torch, engine, steps=2, method="smith")
        igt = None
        if rank == 0 and world == 1 and not args.skip_igt:
            igt = igt_case(torch, engine, deck)
        cpu = None
        if rank == 0 and world == 1 and not args.skip_cpu:
            cpu = reference_cpu(prm, deck, args.cpu_steps)
        out = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded self-avoiding chain, seeded charges; Philox noise)",
            "config": {"workload": f"chain N={deck.n} (3N={n}), free-space RPY + Cholesky noise, D and L rebuilt "
                                   f"every {REFRESH} steps, mixed precision",
                       "warmup_steps_run": warm,
                       "beads": deck.n, "refresh": REFRESH, "precision": "mixed (FP32 D/L, FP16-split updates, "
                                                                         "FP64 diagonal tiles and sums)",
                       "l2": "inputs larger than L2 (stored D/L 604 MB read every step)",
                       "parallelism": "replicas" if world > 1 else "single"},
            "single_step_calls": {"value": args.steps / (ms_single / 1e3), "unit": "steps/s",
                                  "ms_per_step": ms_single / args.steps,
                                  "note": "the same K steps as K bdb_step(1) calls, each ending in a host read of the status word"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches.value),
            "clocks": clk.summary(), "fp64_gpu": fp64, "errors": errors, "replicas": reps, "adjoint": adj, "ewald_suspension": ew,
            "smith_suspension": ews,
            "igt": igt,
        }
        if rank == 0:
            print(json.dumps(out), flush=True)
        sysm.close()
        ranks.finish(dist)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def fp64_case(torch, engine, deck, mixed_value):
    """This library's plain FP64 path: FP64 tensor, FP64 Cholesky (DMMA
    panels and trailing updates), FP64 products. Steps/s with D and its
    factor rebuilt every step (BD_BOX's schedule) and every REFRESH steps
    (the mixed path's schedule, so that mixed/FP64 at the same schedule is
    the gain of the precision alone); Cholesky TFLOP/s of the FP64 refresh."""
    out = {}
    s64 = engine.System(deck, precision=engine.PREC_FP64, refresh=1, noise=engine.NOISE_PHILOX, seed=5)
    s64.step(2)
    k64 = 3
    ms = time_steps(torch, s64, k64)
    out["refresh_1"] = {"value": k64 / (ms / 1e3), "unit": "steps/s"}
    rms = time_refresh(torch, s64, 3)
    n = 3 * deck.n
    out["refresh_ms"] = rms
    out["cholesky_tflops"] = n ** 3 / 3.0 / (rms / 1e3) / 1e12
    s64.close()
    s10 = engine.System(deck, precision=engine.PREC_FP64, refresh=REFRESH, noise=engine.NOISE_PHILOX, seed=5)
    s10.step(REFRESH + 2)
    k10 = 2 * REFRESH
    ms = time_steps(torch, s10, k10)
    out[f"refresh_{REFRESH}"] = {"value": k10 / (ms / 1e3), "unit": "steps/s"}
    s10.close()
    out["value"] = out["refresh_1"]["value"]
    out["unit"] = "steps/s"
    out["mixed_over_fp64"] = {"same_schedule": mixed_value / out[f"refresh_{REFRESH}"]["value"],
                              "fp64_every_step": mixed_value / out["refresh_1"]["value"]}
    out["note"] = "FP64 everywhere; value = D and Cholesky rebuilt every step (BD_BOX's schedule)"
    return out


def accuracy(torch, engine, deck):
    """Relative errors of the mixed path against the FP64 GPU path (itself
    checked against the oracle in the parity tests): ||B B^T - D||/||D||,
    D.F and one step's displacement from the same state and noise."""
    n3 = 3 * deck.n
    g = np.random.default_rng(11).standard_normal(n3)
    sm = engine.System(deck, precision=engine.PREC_MIXED, refresh=REFRESH, noise=engine.NOISE_HOST)
    s64 = engine.System(deck, precision=engine.PREC_FP64, refresh=REFRESH, noise=engine.NOISE_HOST)
    out = {}
    try:
        out["factor_rel"] = sm.factor_error()
    except Exception as e:  # noqa: BLE001
        out["factor_rel"] = f"unavailable: {e}"
    rf_m, rf_d = sm.compute_Rf(), s64.compute_Rf()
    out["df_rel"] = float(np.linalg.norm(rf_m - rf_d) / np.linalg.norm(rf_d))
    x0 = s64.get_coord()
    sm.step(1, g)
    s64.step(1, g)
    dm = sm.get_coord()[:, :3] - x0[:, :3]
    dd = s64.get_coord()[:, :3] - x0[:, :3]
    out["displacement_rel"] = float(np.linalg.norm(dm - dd) / np.linalg.norm(dd))
    sm.close()
    s64.close()
    return out


def replicas(torch, engine, steps, warmup, dist=None, rank=0, world=1):
    """Batched-replica workload: 256 independent chains, bead counts uniform
    in [64, 1024] (seeded), chain force field, free-space RPY with TEA noise,
    FP32 tensor with FP64 TEA sums, all in one batch (bdb_create_batch).
    Aggregate bead-steps/s over `steps` device-noise steps. With several
    processes each runs its shard of the chains (bdb_shard_replicas, no
    collective on the data path) and the time is the slowest rank's
    (strong scaling: the total work is fixed). On one process, also the
    per-replica displacement error of one step against the FP64 batch with
    the same Gaussians."""
    from bd_box_b200 import decks, ranks
    sizes = decks.replica_sizes()
    shard = engine.shard_replicas(sizes, world)
    mine = np.flatnonzero(shard == rank)
    with tempfile.TemporaryDirectory() as d:
        ds = [decks.read_deck(decks.write_chain_deck(d, f"r{k}", int(sizes[k]), seed=1000 + int(k), hydro="geyer"))
              for k in mine]
    total = int(sizes.sum())
    ms, launches, tea_tile = 0.0, 0, None
    if ds:
        b = engine.System(ds, precision=engine.PREC_MIXED, noise=engine.NOISE_PHILOX,
                          seed=ranks.replica_seed(SEED, rank))
        b.autotune(True)
        for _ in range(warmup):
            b.step(1)
        ranks.barrier(dist)
        ms = time_steps(torch, b, steps)
        launches = b.launches()
        tea_tile = b.tuning()[0]
        b.close()
    else:
        ranks.barrier(dist)
    ms = ranks.max_over_ranks(dist, ms, "cuda")
    out = {"workload": f"{len(sizes)} chains, beads uniform in [64,1024] (seeded), sum N={total}, "
                       f"sum N^2={int((sizes.astype(np.int64) ** 2).sum())}, TEA noise, mixed precision, "
                       + ("one batch" if world == 1 else f"sharded over {world} processes, one batch each"),
           "metric": "bead-steps/s", "value": total * steps / (ms / 1e3), "steps": steps,
           "ms_per_step": ms / steps, "gpu_launches": launches, "autotuned_tea_tile": tea_tile,
           "scaling": "strong", "displacement_rel_vs_fp64": None}
    if world == 1:
        g = np.random.default_rng(13).standard_normal(3 * total)
        bm = engine.System(ds, precision=engine.PREC_MIXED, noise=engine.NOISE_HOST)
        b64 = engine.System(ds, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
        x0 = b64.get_coord()
        bm.step(1, g)
        b64.step(1, g)
        xm, x64 = bm.get_coord(), b64.get_coord()
        bm.close()
        b64.close()
        errs = []
        for k in range(len(ds)):
            lo, hi = b64.begins[k], b64.begins[k] + ds[k].n
            dd = x64[lo:hi, :3] - x0[lo:hi, :3]
            dm = xm[lo:hi, :3] - x0[lo:hi, :3]
            errs.append(float(np.linalg.norm(dm - dd) / np.linalg.norm(dd)))
        out["displacement_rel_vs_fp64"] = {"max": max(errs), "median": float(np.median(errs))}
    return out


def adjoint_case(torch, engine):
    """Adjoint workload: an N=1024 chain with the chain force field, free-space
    RPY with Cholesky noise at a fixed Philox sequence, 200 steps, checkpoint
    every 20; loss = mean squared deviation of 128 seeded bead-pair distances
    from seeded targets in [10, 60] A. The electrostatic and LJ cutoffs lie
    beyond the chain's extent, so no pair crosses a cutoff under the finite
    differences. The mixed-precision adjoint (FP32 forward and triangular
    solves, FP64 sums) and the FP64 one are timed; both are checked against
    central differences (h = 1e-4) of the FP64 forward along a random
    direction of the initial positions and for the four scale factors (LJ
    epsilon, LJ sigma, bond H, Debye length)."""
    import copy
    from bd_box_b200 import decks
    with tempfile.TemporaryDirectory() as d:
        deck = decks.read_deck(decks.write_chain_deck(d, "adj1024", 1024, seed=21, hydro="cholesky",
                                                      extra={"cutoff_c": 1000, "cutoff_lj": 1000}))
    rng = np.random.default_rng(4)
    pairs = np.array([rng.choice(deck.n, 2, replace=False) for _ in range(128)], dtype=np.int32)
    targets = rng.uniform(10, 60, size=len(pairs))
    K, ck, h = 200, 20, 1e-4

    def scaled(x0=None, sc=(1.0, 1.0, 1.0, 1.0)):
        dk = copy.deepcopy(deck)
        if x0 is not None:
            dk.coord = dk.coord.copy()
            dk.coord[:, :3] = x0
        dk.LJ = dk.LJ.copy()
        dk.LJ[:, 1] *= sc[0]
        dk.LJ[:, 0] *= sc[1]
        dk.bond_parms = dk.bond_parms.copy()
        dk.bond_parms[:, 2] *= sc[2]
        dk.prm = dict(dk.prm)
        dk.prm["kappa_c"] = dk.prm["kappa_c"] / sc[3]
        return dk

    def loss_at(dk):
        s = engine.System(dk, precision=engine.PREC_FP64, refresh=1, noise=engine.NOISE_PHILOX, seed=99)
        s.step(K)
        x = s.get_coord()[:, :3]
        s.close()
        r = np.linalg.norm(x[pairs[:, 1]] - x[pairs[:, 0]], axis=1)
        return float(np.mean((r - targets) ** 2))

    out = {"workload": "chain N=1024, Cholesky noise (fixed Philox sequence), 200 steps, checkpoint 20, 128 "
                       "pair-distance loss; cutoffs beyond the chain's extent"}
    grads = {}
    for name, prec in (("mixed", engine.PREC_MIXED), ("fp64", engine.PREC_FP64)):
        s = engine.System(deck, precision=prec, refresh=1, noise=engine.NOISE_PHILOX, seed=99)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        loss, gx, gp = s.adjoint(K, ck, pairs, targets)
        torch.cuda.synchronize()
        t_grad = time.perf_counter() - t0
        s.close()
        s = engine.System(deck, precision=prec, refresh=1, noise=engine.NOISE_PHILOX, seed=99)
        t0 = time.perf_counter()
        s.step(K)
        torch.cuda.synchronize()
        t_fwd = time.perf_counter() - t0
        s.close()
        grads[name] = (gx, gp)
        out[name] = {"loss": loss, "seconds_per_gradient": t_grad, "seconds_forward_only": t_fwd,
                     "gradient_over_forward": t_grad / t_fwd}
    v = rng.standard_normal((deck.n, 3))
    v /= np.linalg.norm(v)
    c0 = deck.coord[:, :3]
    fd_x = (loss_at(scaled(c0 + h * v)) - loss_at(scaled(c0 - h * v))) / (2 * h)
    fd_p = []
    for k in range(4):
        sp, sm = [1.0] * 4, [1.0] * 4
        sp[k] += h
        sm[k] -= h
        fd_p.append((loss_at(scaled(sc=sp)) - loss_at(scaled(sc=sm))) / (2 * h))
    for name in ("mixed", "fp64"):
        gx, gp = grads[name]
        an = float(np.sum(gx * v))
        out[name]["fd_check"] = {
            "h": h, "position_direction": {"fd": fd_x, "adjoint": an, "rel_err": abs(fd_x - an) / abs(fd_x)},
            "scale_factors": {nm: {"fd": fd_p[k], "adjoint": float(gp[k]), "rel_err": abs(fd_p[k] - gp[k]) / abs(fd_p[k])}
                              for k, nm in enumerate(("lj_epsilon", "lj_sigma", "bond_H", "debye_length"))}}
    gxm, gpm = grads["mixed"]
    gxd, gpd = grads["fp64"]
    out["mixed_vs_fp64_gradient_rel"] = {"positions": float(np.linalg.norm(gxm - gxd) / np.linalg.norm(gxd)),
                                         "scale_factors": [float(abs(a - b) / abs(b)) for a, b in zip(gpm, gpd)]}
    return out


EWALD_R = 4   # lattice radius of the Ewald sums: D.F within 1e-6 of R = 5 (R = 3: 7e-6)


def ewald_case(torch, engine, steps=3, method="beenakker"):
    """Periodic suspension: N=4096 spheres of radius 1 A at volume fraction
    0.10, Ewald-summed RPY (Beenakker or Smith) over the lattice sphere of
    radius EWALD_R, with TEA noise computed on the fly, WCA repulsion via
    cell lists; steps/s of the mixed path and one step's displacement error
    against the FP64 path with the same noise."""
    from bd_box_b200 import decks
    with tempfile.TemporaryDirectory() as d:
        deck = decks.read_deck(decks.write_suspension_deck(d, "susp4096", 4096, seed=8, ewald_r=EWALD_R,
                                                           extra={"ewald_method": method}))
    s = engine.System(deck, precision=engine.PREC_MIXED, noise=engine.NOISE_PHILOX, seed=SEED)
    s.autotune(True)
    s.step(1)
    ms = time_steps(torch, s, steps)
    tea_tile = s.tuning()[0]
    s.close()
    g = np.random.default_rng(6).standard_normal(3 * deck.n)
    sm = engine.System(deck, precision=engine.PREC_MIXED, noise=engine.NOISE_HOST)
    s64 = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    x0 = s64.get_coord()
    t0 = time.perf_counter()
    s64.step(1, g)
    torch.cuda.synchronize()
    t64 = time.perf_counter() - t0
    sm.step(1, g)
    dd = s64.get_coord()[:, :3] - x0[:, :3]
    dm = sm.get_coord()[:, :3] - x0[:, :3]
    box = deck.box[0]
    dd -= box * np.round(dd / box)
    dm -= box * np.round(dm / box)
    sm.close()
    s64.close()
    return {"workload": f"periodic suspension N=4096, phi=0.10, {method.capitalize()} Ewald R={EWALD_R}, TEA on the fly, "
                        "mixed precision",
            "metric": "steps/s", "value": steps / (ms / 1e3), "ms_per_step": ms / steps,
            "fp64_steps_per_s": 1.0 / t64, "autotuned_tea_tile": tea_tile,
            "displacement_rel_vs_fp64": float(np.linalg.norm(dm - dd) / np.linalg.norm(dd))}


def igt_case(torch, engine, deck, steps=5):
    """IGT predictor-corrector (igt_const) on the bench chain: two tensor
    builds and two Cholesky factorisations per step (D at r, then the
    average of D(r) and D(r')); steps/s of the mixed and FP64 paths and one
    step's displacement error of mixed against FP64 with the same noise."""
    s = engine.System(deck, precision=engine.PREC_MIXED, noise=engine.NOISE_PHILOX, seed=SEED)
    s.step_igt(1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.step_igt(steps)
    torch.cuda.synchronize()
    t_mixed = (time.perf_counter() - t0) / steps
    s.close()
    n3 = 3 * deck.n
    g = np.random.default_rng(7).standard_normal(2 * n3)
    sm = engine.System(deck, precision=engine.PREC_MIXED, noise=engine.NOISE_HOST)
    s64 = engine.System(deck, precision=engine.PREC_FP64, noise=engine.NOISE_HOST)
    x0 = s64.get_coord()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s64.step_igt(1, g)
    torch.cuda.synchronize()
    t64 = time.perf_counter() - t0
    sm.step_igt(1, g)
    dd = s64.get_coord()[:, :3] - x0[:, :3]
    dm = sm.get_coord()[:, :3] - x0[:, :3]
    sm.close()
    s64.close()
    return {"workload": f"chain N={deck.n}, free-space RPY + Cholesky noise, IGT predictor-corrector (igt_const)",
            "metric": "steps/s", "value": 1.0 / t_mixed, "ms_per_step": 1e3 * t_mixed,
            "fp64_steps_per_s": 1.0 / t64,
            "displacement_rel_vs_fp64": float(np.linalg.norm(dm - dd) / np.linalg.norm(dd))}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    tmp = tempfile.mkdtemp(prefix="bdb_ref_")
    try:
        prm, deck = make_deck(tmp)
        steps = max(1, min(args.steps, args.cpu_steps))
        cpu = reference_cpu(prm, deck, steps, single_thread=False)
        out = {"metric": METRIC, "value": cpu["value"], "unit": "steps/s", "n_gpus": world, "steps": steps,
               "warmup": 0, "ms_per_step": 1e3 / cpu["value"], "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded self-avoiding chain)",
               "config": {"workload": f"chain N={deck.n}, free-space RPY + Cholesky noise, D and L rebuilt every "
                                      f"{REFRESH} steps", "beads": deck.n, "refresh": REFRESH},
               "impl": "reference", "cpu_baseline": cpu,
               "e2e": {"value": cpu["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out), flush=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def relaunch_as_ranks(n: int):
    """--gpus N > 1 outside a torchrun launch: run this script again as N
    ranks on this node (one process per GPU) under torch.distributed.run, so
    that --gpus N always means N processes."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
    sys.stdout.flush()
    os.execv(sys.executable, cmd)


def run_stub(args):
    """The launcher and the timing protocol without a GPU (gloo ranks on
    CPU): each rank sleeps a rank-dependent time per step in place of the
    step, the time is bracketed by barriers and reduced as the max over
    ranks, and rank 0 prints the JSON line. For tests of the multi-process
    path only."""
    from bd_box_b200 import ranks
    dist, rank, world, _ = ranks.init("gloo", timeout_s=60)
    for _ in range(args.warmup):
        time.sleep(0.001)
    ranks.barrier(dist)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        time.sleep(0.01 * (1 + rank))
    ranks.barrier(dist)
    ms = 1e3 * (time.perf_counter() - t0)
    ms = ranks.max_over_ranks(dist, ms, "cpu")
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": world * args.steps / (ms / 1e3), "unit": "steps/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": ms / args.steps, "scaling": "weak", "stub": True}), flush=True)
    ranks.finish(dist)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-errors", action="store_true")
    ap.add_argument("--skip-replicas", action="store_true")
    ap.add_argument("--skip-adjoint", action="store_true")
    ap.add_argument("--skip-ewald", action="store_true")
    ap.add_argument("--skip-igt", action="store_true")
    ap.add_argument("--stub", action="store_true", help="CPU-only stand-in step (tests of the launcher)")
    ap.add_argument("--beads", type=int, default=N_BEADS,
                    help="chain length of the main workload (smaller sizes for profiler captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        relaunch_as_ranks(args.gpus)
    if args.stub:
        run_stub(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
