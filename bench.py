#!/usr/bin/env python
"""Headline benchmark: converged NR solves/s of the Monte-Carlo DC + transient job.

Workload (one "step"): 4096 seeded Monte-Carlo instances of a 256-stage CMOS
inverter chain with 64 diode clamps (IS 1e-14 A, N 1, RS 10 ohm) and 1 fF node
caps (n = 322 unknowns); per-device VTO ~ N(card, 30 mV), KP ~ N(card, 5 %).
Every instance solves its DC operating point, then a 200-step backward-Euler
transient (1 ps) of a 0 -> 1.8 V input ramp. A "solve" is one converged
nonlinear solve of one instance at one time point (DC point or transient step),
so a fully converged step is 4096 * 201 solves. Synthetic inputs, fixed seeds.

value  : mixed precision (FP32 Jacobian + FP32 LU, FP64 residual/refinement),
         inputs resident in HBM, device time from CUDA events around each job,
         L2 flushed (512 MiB write) between timed steps.
e2e    : the same job through the C ABI with host buffers (karam_run_mc: H2D of
         the per-instance parameters, D2H of voltages + stats), wall clock.
fp64   : the plain FP64 GPU Newton path on the same job, for the comparison
         the headline metric names.
--impl reference : the reference CPU implementation of the path (compiled from
         the reference sources: generic device kernels, stampSoABlock, CSR
         assembly, solveSparse_LU) on all host threads, a bounded sample of
         instances per step.

Multi-GPU (torchrun): every rank solves its own batch of instances (weak
scaling, no collective on the data path); timings are reduced with MAX.
"""
from __future__ import annotations

import argparse
import contextlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STAGES, CLAMPS = 256, 64
TRAN_STEPS, DT = 200, 1e-12
POLISH = dict(polish_max=8, polish_rel=1e-11, polish_abs=1e-14)
SEEDER_FIRST = 1_000_000  # training instances: MC ids from here on
SEEDER_BATCHES = 4
SEEDER_EPOCHS = 30
MAX_HALVINGS = 6
METRIC = "solves/sec at <=1e-9 rel err: seeded mixed-precision vs plain FP64 NR, 1xB200"
FALLBACK_HBM_GBS = 6650.0
FALLBACK_BF16_TFLOPS = 1590.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="karam", choices=["karam", "reference"])
    ap.add_argument("--instances", type=int, default=4096)
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="instances in the CPU-baseline sample (0 = sized to ~15 s)")
    ap.add_argument("--seeder-batches", type=int, default=SEEDER_BATCHES,
                    help="batches of plain-NR DC solutions the learned seeder trains on (untimed)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the config-1 latency, config-3 uneven-batch and config-5 seeder "
                         "measurements")
    ap.add_argument("--config3-steps", type=int, default=500,
                    help="trapezoidal steps of the config-3 uneven batch")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--max-rounds", type=int, default=0,
                    help="stop every job after this many NR rounds (profiling captures of a "
                         "bounded part of the workload; the result line is marked partial)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
class Dist:
    def __init__(self, want_gpus):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        if self.world > 1 and want_gpus not in (1, self.world):
            raise SystemExit(f"--gpus {want_gpus} under a launcher of {self.world} ranks")
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as td
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            td.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.td = td
            self.torch = torch
            self.pg = True

    def barrier(self):
        if self.pg:
            self.td.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64,
                              device="cuda" if self.torch.cuda.is_available() else "cpu")
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64,
                              device="cuda" if self.torch.cuda.is_available() else "cpu")
        self.td.all_reduce(t, op=self.td.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.td.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "samples": len(sm),
                "reasons": sorted(reasons)}


def measured_peaks(kind="hbm"):
    """(peak, "measured" | "fallback"): the HBM copy bandwidth in GB/s, or with
    kind="bf16" the burst cuBLAS BF16 GEMM rate in TFLOP/s."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["bf16_tflops" if kind == "bf16" else "hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return (FALLBACK_BF16_TFLOPS if kind == "bf16" else FALLBACK_HBM_GBS), "fallback"


def profiled_traffic(kernel):
    """DRAM bytes (read + write) of one launch of `kernel` at the full
    4096-instance batch, from the committed ncu summaries: lines of the form
    `traffic_bytes_per_full_launch <kernel>: <bytes>` under profiles/."""
    key = f"traffic_bytes_per_full_launch {kernel}:"
    pdir = os.path.join(ROOT, "profiles")
    try:
        for name in sorted(os.listdir(pdir)):
            if name.endswith(".md"):
                for line in open(os.path.join(pdir, name)):
                    if line.startswith(key):
                        return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def workload(n_inst, first):
    from karam_b200 import circuits
    nl = circuits.config2()
    inst = circuits.mc_instances(nl, n_inst, first_instance=first)
    return nl, inst


@contextlib.contextmanager
def native_stdout_to_stderr():
    """The reference library prints start-up notes on the C stdout; send them to
    stderr so stdout carries only the bench line."""
    sys.stdout.flush()
    saved = os.dup(1)
    try:
        os.dup2(2, 1)
        yield
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(saved)


def cpu_sample_run(nl, inst, count, threads):
    """Reference CPU implementation (oracle/_ref when built, else the restatement)
    on `count` instances with `threads` host threads; returns (seconds, solves, kind)."""
    from oracle import pyoracle
    kind = "reference" if pyoracle.available("ref") else "port"
    if kind == "port":
        pyoracle.build("port")
    with native_stdout_to_stderr():
        orc = pyoracle.Oracle("ref" if kind == "reference" else "port")
        t0 = time.perf_counter()
        _, st = orc.run_batch(nl, inst, 0, count, dt=DT, n_steps=TRAN_STEPS, n_threads=threads,
                              linear_solver=pyoracle.LS_SPARSE, max_halvings=MAX_HALVINGS, **POLISH)
        el = time.perf_counter() - t0
    solves = sum(TRAN_STEPS + 1 for s in st if s["converged"])
    return el, solves, kind


def run_reference(args, dist):
    if dist.rank != 0:
        return
    threads = os.cpu_count() or 1
    nl, inst = workload(max(threads * 4, 32), 0)
    count = args.cpu_sample or threads * 2
    for _ in range(args.warmup):
        cpu_sample_run(nl, inst, min(count, threads), threads)
    total_t = total_s = 0.0
    kind = "reference"
    for _ in range(args.steps):
        el, solves, kind = cpu_sample_run(nl, inst, count, threads)
        total_t += el
        total_s += solves
    value = total_s / total_t
    sample = f"{count} instances x (DC + {TRAN_STEPS} BE steps) per step, {threads} threads"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_t / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "MC inverter chain 256 stages + 64 diode clamps, n=322, "
                               "DC + 200 BE steps of 1 ps", "instances_per_step": count,
                   "solver": "oracle/_ref: reference sources, solveSparse_LU"
                   if kind == "reference" else "oracle port (restatement)"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def eval_stamp_bytes(info, mixed, tran=False):
    """Algorithmic HBM bytes of one evaluation + stamping of one instance
    (k_es): KP/VTO read (FP32), the trial point x and the accepted point v read
    (FP64; v for the convergence test), the Jacobian value slots written (FP32
    or FP64), the KCL residual written (FP64), and in transient the capacitor
    history v_prev read. Device values live in shared memory only."""
    n, nm, nv, nc = info["n"], info["n_mos"], info["n_slots"], info["n_cap"]
    b = 8 * nm + 8 * n + 8 * n + (4 if mixed else 8) * nv + 8 * n
    return b + (8 * nc if tran else 0)


def lu_bytes(info, mixed):
    """Algorithmic HBM bytes of one control-flow + factor/solve pass of one
    instance (k_lu): the Jacobian value slots and the KCL residual read, x and
    v read and written back, the state record read and written."""
    n, nv = info["n"], info["n_slots"]
    return (4 if mixed else 8) * nv + 8 * n + 4 * 8 * n + 2 * 104


def run_karam(args, dist):
    import karam_b200 as K
    from karam_b200 import _abi as A

    ni = args.instances
    nl, inst = workload(ni, dist.rank * ni)
    ctx = K.Context(dist.local)
    prob = K.Problem(ctx, nl, max_instances=ni)
    prob.set_instances(inst)
    info = prob.info

    flush = None
    try:
        import torch
        if torch.cuda.is_available():
            flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32,
                                device=f"cuda:{dist.local}")
    except Exception:
        flush = None

    def l2_flush():
        if flush is not None:
            flush.zero_()
            import torch
            torch.cuda.synchronize()

    def job(opts):
        prob.run_mc_device(DT, TRAN_STEPS, A.TRAN_BE, opts)
        t = prob.timing()
        _, st = prob.read_results()
        conv = sum(1 for s in st if s["status"] == A.ST_CONVERGED)
        return t, conv, st

    # the learned seeder, trained before timing on plain-NR DC solutions of
    # SEEDER_BATCHES x ni other instances (ids from SEEDER_FIRST on, disjoint
    # from the benchmark's)
    from karam_b200 import circuits
    t_s0 = time.perf_counter()
    seeder = K.Seeder(prob, width=512, hidden_layers=3, init_seed=1)
    plain_dc = K.options(precision=A.PREC_MIXED, **POLISH)
    n_train = 0
    for b in range(args.seeder_batches):
        prob.set_instances(circuits.mc_instances(
            nl, ni, first_instance=SEEDER_FIRST + (dist.rank * args.seeder_batches + b) * ni))
        prob.solve_dc(plain_dc)
        n_train += seeder.add_dc(prob)
    t_s1 = time.perf_counter()
    seeder_loss = seeder.train(epochs=SEEDER_EPOCHS, batch=256, lr=1e-3, shuffle_seed=1)
    t_s2 = time.perf_counter()
    prob.set_instances(inst)
    v_plain_dc, st_plain_dc = prob.solve_dc(plain_dc)
    guess = seeder.predict(prob)
    ok_dc = [i for i, s in enumerate(st_plain_dc) if s["status"] == A.ST_CONVERGED]
    seed_err = np.abs(guess[ok_dc] - v_plain_dc[ok_dc])
    prob.set_seeder(seeder)

    # the headline arm: mixed precision seeded by the learned seeder; beside
    # it the statistical seeder (plain DC of the first 8 instances inside the
    # job, their EMA seeds the rest) and unseeded mixed precision; the
    # comparison arm: plain FP64 NR from the reference seed
    mixed = K.options(precision=A.PREC_MIXED, max_halvings=MAX_HALVINGS,
                      max_rounds=args.max_rounds, seeded=A.SEED_MLP, **POLISH)
    mixed_ema = K.options(precision=A.PREC_MIXED, max_halvings=MAX_HALVINGS,
                          max_rounds=args.max_rounds, seeded=A.SEED_EMA, **POLISH)
    mixed_plain = K.options(precision=A.PREC_MIXED, max_halvings=MAX_HALVINGS,
                            max_rounds=args.max_rounds, **POLISH)
    fp64 = K.options(precision=A.PREC_FP64, max_halvings=MAX_HALVINGS,
                     max_rounds=args.max_rounds, **POLISH)

    for _ in range(args.warmup):
        l2_flush()
        job(mixed)

    clocks = Clocks(dist.local)
    dist.barrier()
    clocks.start()
    tot_ms = 0.0
    solves = 0
    launches = 0
    rescues = 0
    rounds = 0
    conv_min = ni
    for _ in range(args.steps):
        l2_flush()
        t, conv, st = job(mixed)
        tot_ms += t["job_ms"]
        solves += conv * (TRAN_STEPS + 1)
        rounds += t["rounds"]
        rescues += t["rescues"]
        launches += (t["eval_launches"] + t["lu_launches"] + t["rescue_launches"]
                     + t["other_launches"])
        lanes = t["lanes"]
        lu_name = ["k_lu<float>", "k_lu_nd<float>", "k_lu_big<float, smem>",
                   "k_lu_big<float, global>", "k_lu_big<float, packed>",
                   "k_persist<float>", "k_lu_big<float, global, global y>"][t["level_schedule"]]
        conv_min = min(conv_min, conv)
    clk = clocks.stop()
    dist.barrier()
    v_mixed, st_mixed = prob.read_results()

    # the kernel split: one more job of the headline arm with CUDA events
    # around every kernel of every round (the events slow the graph down, so
    # the timed jobs above run without them)
    l2_flush()
    tk, _, _ = job(K.options(precision=A.PREC_MIXED, max_halvings=MAX_HALVINGS,
                             max_rounds=args.max_rounds, seeded=A.SEED_MLP,
                             kernel_timing=1, **POLISH))
    eval_ms, lu_ms, rescue_ms = tk["eval_ms"], tk["lu_ms"], tk["rescue_ms"]
    evals_dc, evals_tran, rounds_k = tk["evals_dc"], tk["evals_tran"], tk["rounds"]
    seed_fallbacks = sum(1 for s in st_mixed[A.SEED_HISTORY:] if not s["seeded_ok"])
    t_max = dist.max(tot_ms)
    all_solves = dist.sum(solves)
    value = all_solves / (t_max / 1e3)

    # plain FP64 GPU Newton path, same job and timing rules
    fp_ms = 0.0
    fp_solves = 0
    for _ in range(max(1, args.warmup // 3)):
        job(fp64)
    for _ in range(args.steps):
        l2_flush()
        t, conv, _ = job(fp64)
        fp_ms += t["job_ms"]
        fp_solves += conv * (TRAN_STEPS + 1)
    v_fp64, st_fp64 = prob.read_results()
    fp_value = dist.sum(fp_solves) / (dist.max(fp_ms) / 1e3)

    # mixed precision with the statistical seeder and without a seeder
    def arm(opts):
        ms = 0.0
        solves = 0
        job(opts)
        for _ in range(args.steps):
            l2_flush()
            t, conv, _ = job(opts)
            ms += t["job_ms"]
            solves += conv * (TRAN_STEPS + 1)
        return dist.sum(solves) / (dist.max(ms) / 1e3)

    ema_value = arm(mixed_ema)
    mp_value = arm(mixed_plain)

    # end to end through the C ABI with host buffers
    h2d = inst.mos_kp.nbytes + inst.mos_vto.nbytes
    d2h = ni * info["n"] * 8 + ni * A.C.sizeof(A.KaramInstanceStats)
    e2e_t = 0.0
    e2e_solves = 0
    for _ in range(args.steps):
        l2_flush()
        dist.barrier()
        t0 = time.perf_counter()
        v, st = prob.run_mc(inst, DT, TRAN_STEPS, A.TRAN_BE, mixed)
        e2e_t += time.perf_counter() - t0
        e2e_solves += sum(TRAN_STEPS + 1 for s in st if s["status"] == A.ST_CONVERGED)
    e2e_value = dist.sum(e2e_solves) / dist.max(e2e_t)

    # rooflines: evaluation + stamping (k_es) and factor/solve (k_lu_nd or
    # k_lu), algorithmic bytes per live instance-round over their event time
    # in the instrumented job
    peak, peak_kind = measured_peaks()
    es_b = evals_dc * eval_stamp_bytes(info, True) + evals_tran * eval_stamp_bytes(info, True, True)
    lu_b = (evals_dc + evals_tran) * lu_bytes(info, True)
    es_gbs = es_b / (eval_ms / 1e3) / 1e9 if eval_ms else 0.0
    lu_gbs = lu_b / (lu_ms / 1e3) / 1e9 if lu_ms else 0.0
    tot_k = eval_ms + lu_ms + rescue_ms
    kernels = {
        "k_es<float>": {"ms_per_step": eval_ms, "share": eval_ms / tot_k,
                        "achieved_gbs": es_gbs, "frac": es_gbs / peak,
                        "bytes_per_instance_eval": eval_stamp_bytes(info, True, True)},
        lu_name: {"ms_per_step": lu_ms, "share": lu_ms / tot_k,
                  "achieved_gbs": lu_gbs, "frac": lu_gbs / peak,
                  "bytes_per_instance_round": lu_bytes(info, True), "lanes_per_cta": lanes},
        "k_rescue": {"ms_per_step": rescue_ms, "share": rescue_ms / tot_k},
    }
    dom = lu_name if lu_ms >= eval_ms else "k_es<float>"
    roofline = {
        "kernel": dom, "bound": "hbm", "achieved": kernels[dom]["achieved_gbs"], "peak": peak,
        "unit": "GB/s", "frac": kernels[dom]["frac"], "peak_source": peak_kind,
        "traffic": profiled_traffic(dom),
        "traffic_source": "ncu capture of one full-batch DC round (dram__bytes_read + write), "
                          "profiles/round_kernels_config2.md",
        "algorithmic_bytes_per_full_launch": ni * (lu_bytes(info, True) if dom == lu_name
                                                   else eval_stamp_bytes(info, True, True)),
        "algorithmic_bytes_model": "transient round (capacitor history read); achieved uses it",
        "algorithmic_bytes_per_full_launch_dc": ni * (lu_bytes(info, True) if dom == lu_name
                                                      else eval_stamp_bytes(info, True, False)),
        "avg_launch_us": 1e3 * (lu_ms if dom == lu_name else eval_ms) / rounds_k,
    }

    # evaluation + stamping alone at full batch (every instance live), CUDA events
    v_probe = np.repeat(v_mixed[:1], ni, axis=0)
    es_us = []
    for _ in range(5):
        l2_flush()
        prob.eval_stamp(v_probe, A.PREC_MIXED)
        es_us.append(1e3 * prob.timing()["eval_ms"])
    es_us = statistics.median(es_us[1:])
    es_bytes = ni * eval_stamp_bytes(info, mixed=True)
    eval_roofline = {"kernel": "k_es<float>, all instances live", "bound": "hbm",
                     "achieved": es_bytes / (es_us / 1e6) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": es_bytes / (es_us / 1e6) / 1e9 / peak, "launch_pair_us": es_us,
                     "algorithmic_bytes": es_bytes}

    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {
            "workload": "MC inverter chain 256 stages + 64 diode clamps, n=322, nnz=1219; "
                        "DC + 200 BE steps of 1 ps",
            "instances_per_gpu": ni, "solves_per_instance": TRAN_STEPS + 1,
            "precision": "mixed: FP32 Jacobian/LU, FP64 residual + Newton refinement",
            "seeder": {
                "kind": "learned: MLP 1026-512-512-512-322, GELU, BF16 weights, FP32 "
                        "accumulation, Adam/MSE on plain-NR DC solutions; seeds every instance "
                        "at the final GMIN step, fallback to full GMIN stepping after 10 "
                        "iterations",
                "train_instances": n_train, "train_data_s": t_s1 - t_s0,
                "train_s": t_s2 - t_s1, "epochs": SEEDER_EPOCHS, "final_loss": seeder_loss,
                "seed_err_max_v": float(seed_err.max()) if ok_dc else None,
                "seed_err_rms_v": float(np.sqrt(np.mean(seed_err ** 2))) if ok_dc else None,
                "timed": "training and its data are set up before timing; inference runs "
                         "inside every timed job"},
            "seed_fallbacks": seed_fallbacks,
            "polish": POLISH, "max_halvings": MAX_HALVINGS,
            "l2": "flushed (512 MiB write) between timed steps",
            "converged_fraction": conv_min / ni,
        },
        **({"partial": f"every job stopped after {args.max_rounds} NR rounds"}
           if args.max_rounds else {}),
        "fp64": {"value": fp_value, "unit": "solves/s",
                 "speedup_mixed_vs_fp64": value / fp_value if fp_value else None},
        "mixed_unseeded": {"value": mp_value, "unit": "solves/s"},
        "mixed_ema_seeded": {"value": ema_value, "unit": "solves/s",
                             "seeder": "NeuralSeeder::predictSeed restated: plain DC of the "
                                       "first 8 instances inside each job"},
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": roofline,
        "kernels": kernels,
        "kernels_from": {"job": "one more headline job with CUDA events around every kernel "
                                "of every round (the timed jobs run without them)",
                         "job_ms": tk["job_ms"]},
        "eval_stamp_full_batch": eval_roofline,
        "rounds_per_step": rounds / args.steps,
        "gpu_launches": launches,
        "rescues_per_step": rescues / args.steps,
        "clocks": clk,
    }

    if dist.rank == 0 and dist.world == 1 and not args.no_configs:
        line["config1"] = config1_latency(ctx)
        line["config5"] = config5_seeder(ctx)
        # the 32-stage family of the same method (130 features), a smaller training set
        line["config5_32stage"] = config5_seeder(ctx, n_train=40960, n_test=8192, stages=32)
        line["config3"] = config3_uneven(dist.local, steps=args.config3_steps)
        line["ac"] = ac_sweep_leg(ctx)
        line["config4_tile"] = config4_tile(ctx)
    if dist.rank == 0 and not args.no_accuracy:
        line["accuracy"] = accuracy_check(nl, inst, v_mixed, v_fp64, st_mixed, st_fp64)
        line["outcomes"] = outcome_check(nl, inst, st_mixed, st_fp64)
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        count = args.cpu_sample or threads * 2
        el, cs, kind = cpu_sample_run(nl, inst, count, threads)
        line["cpu_baseline"] = {
            "value": cs / el, "unit": "solves/s", "cores": threads, "kind": kind,
            "sample": f"{count} instances x (DC + {TRAN_STEPS} BE steps), {threads} threads, "
                      f"{el:.1f} s"}
    if dist.rank == 0:
        print(json.dumps(line), flush=True)
    prob.set_seeder(None)
    seeder.close()
    prob.close()
    ctx.close()


def config4_tile(ctx, N=64, steps=1000, dt=1e-12, n_check=32, check_steps=150, big_N=128, big_steps=100):
    """Tiles of the large single-instance workload (circuits.power_grid_mesh):
    one N x N mesh, DC then `steps` backward-Euler steps of `dt`, FP32 LU +
    FP64 refinement against plain FP64 on the GPU (the level-scheduled
    kernels; the 1024 x 1024 mesh itself needs the supernodal solver, which is
    not built). Accuracy and the CPU rate: an n_check x n_check tile, DC +
    check_steps steps, GPU mixed precision against the reference-built oracle
    (sparse LU), one thread. Then a big_N x big_N tile, DC + big_steps steps,
    with the oracle's KCL residual as its accuracy check."""
    import karam_b200 as K
    from karam_b200 import _abi as A
    from karam_b200 import circuits
    from oracle import pyoracle
    out = {"workload": f"{N} x {N} power-grid mesh tile (0.1-1 ohm segments, 10 fF caps, VDD pads every "
                       f"64 border nodes, pulsed NMOS loads at 1.9 % of nodes); DC + {steps} BE steps of "
                       f"{dt * 1e12:g} ps, one instance"}
    nl = circuits.power_grid_mesh(N)
    prob = K.Problem(ctx, nl, max_instances=1)
    prob.set_instances(None)
    out["n"] = nl.n_nodes
    for name, prec in (("mixed", A.PREC_MIXED), ("fp64", A.PREC_FP64)):
        opts = K.options(precision=prec, **POLISH)
        prob.run_mc_device(dt, 4, A.TRAN_BE, opts)  # warm-up
        t = time.perf_counter()
        prob.run_mc_device(dt, steps, A.TRAN_BE, opts)
        wall = time.perf_counter() - t
        tm = prob.timing()
        _, st = prob.read_results()
        out[name] = {"solves_per_s": (steps + 1) / wall if st[0]["status"] == A.ST_CONVERGED else 0.0,
                     "wall_s": wall, "device_ms": tm["job_ms"], "rounds": tm["rounds"],
                     "iterations": st[0]["iterations"], "converged": st[0]["status"] == A.ST_CONVERGED,
                     "schedule": lu_name_of(tm)}
    prob.close()
    out["speedup_mixed_vs_fp64"] = (out["mixed"]["solves_per_s"] / out["fp64"]["solves_per_s"]
                                    if out["fp64"]["solves_per_s"] else None)
    # accuracy and the CPU rate on a smaller tile
    nl = circuits.power_grid_mesh(n_check)
    prob = K.Problem(ctx, nl, max_instances=1)
    prob.set_instances(None)
    nodes = [3, 3 + n_check * n_check // 2 + n_check // 2, nl.n_nodes]
    opts = K.options(precision=A.PREC_MIXED, **POLISH)
    prob.solve_dc(opts)
    v, st, wave = prob.step_transient(dt, check_steps, A.TRAN_BE, opts, wave_nodes=nodes)
    prob.close()
    kind = "ref" if pyoracle.available("ref") else "port"
    if kind == "port":
        pyoracle.build("port")
    with native_stdout_to_stderr():
        orc = pyoracle.Oracle(kind)
        t = time.perf_counter()
        vd, sd = orc.solve_dc(nl, linear_solver=pyoracle.LS_SPARSE, **POLISH)
        vt, stt, w_ref = orc.transient(nl, vd, dt, check_steps, A.TRAN_BE, wave_nodes=nodes,
                                       linear_solver=pyoracle.LS_SPARSE, **POLISH)
        cpu_t = time.perf_counter() - t
    out["check"] = {"tile": f"{n_check} x {n_check} (n = {nl.n_nodes}), DC + {check_steps} steps, mixed",
                    "max_scaled_err_vs_oracle": float(np.max(np.abs(v[0] - vt) / (1e-9 * np.abs(vt) + 1e-12))),
                    "max_abs_wave_diff_v": float(np.max(np.abs(wave[0] - w_ref)))}
    out["cpu_baseline"] = {"value": (check_steps + 1) / cpu_t, "unit": "solves/s", "cores": 1,
                           "kind": "reference" if kind == "ref" else "port",
                           "sample": f"the {n_check} x {n_check} tile, DC + {check_steps} steps, sparse LU "
                                     f"(solveSparse_LU with the Min-Fill ordering), {cpu_t:.1f} s"}
    # a 128 x 128 tile: the largest the level-scheduled kernels take; its
    # accuracy is the oracle's KCL residual at the DC point and the last step
    # (the oracle's own solve is a dense LU at this size)
    nl = circuits.power_grid_mesh(big_N)
    t = time.perf_counter()
    prob = K.Problem(ctx, nl, max_instances=1)
    analysis_s = time.perf_counter() - t
    prob.set_instances(None)
    big = {"tile": f"{big_N} x {big_N} (n = {nl.n_nodes}), DC + {big_steps} BE steps of {dt * 1e12:g} ps",
           "host_analysis_s": analysis_s}
    for name, prec in (("mixed", A.PREC_MIXED), ("fp64", A.PREC_FP64)):
        opts = K.options(precision=prec, **POLISH)
        prob.run_mc_device(dt, 2, A.TRAN_BE, opts)  # warm-up
        t = time.perf_counter()
        prob.run_mc_device(dt, big_steps, A.TRAN_BE, opts)
        wall = time.perf_counter() - t
        tm = prob.timing()
        _, st = prob.read_results()
        big[name] = {"solves_per_s": (big_steps + 1) / wall if st[0]["status"] == A.ST_CONVERGED else 0.0,
                     "wall_s": wall, "device_ms": tm["job_ms"], "rounds": tm["rounds"],
                     "iterations": st[0]["iterations"], "converged": st[0]["status"] == A.ST_CONVERGED,
                     "schedule": lu_name_of(tm)}
    vdc, _ = prob.solve_dc(K.options(precision=A.PREC_MIXED, **POLISH))
    nodes = np.arange(1, nl.n_nodes + 1, dtype=np.int32)
    v, _, wave = prob.step_transient(dt, 2, A.TRAN_BE, K.options(precision=A.PREC_MIXED, **POLISH),
                                     wave_nodes=nodes)
    prob.close()
    with native_stdout_to_stderr():
        big["kcl_residual_dc"] = orc.kcl_residual(nl, vdc[0])
        big["kcl_residual_step2"] = orc.kcl_residual(nl, v[0], h=dt, v_prev=wave[0][0], t=2 * dt)
    out["tile128"] = big
    return out


def lu_name_of(tm):
    return ["pivot records", "warp per instance", "CTA per instance, shared memory",
            "CTA per instance, global memory", "CTA per instance, packed program",
            "persistent CTA per instance",
            "CTA per instance, global memory, solve vector in global memory"][tm["level_schedule"]]


def ac_sweep_leg(ctx, n_instances=4096, n_points=16, f_start=1e6, f_stop=1e12, input_node=2,
                 oracle_sample=4):
    """Small-signal AC sweep (karam_ac_sweep) of the config-2 Monte-Carlo batch
    at its DC points: each instance's Y(jw) = the FP64 NR Jacobian at its DC
    point + jwC, driven at the chain's input, over n_points log-spaced
    frequencies; one CTA per (instance, frequency) factors Y on the static
    pivots in complex FP64. Timed: the call (device time of the Jacobian
    evaluation + the sweep, and wall time with the copies back). Accuracy: the
    first instances against the oracle's sweep (dense complex LU with partial
    pivoting) at the same DC points, which also gives the CPU rate on that
    sample (the oracle's restatement of the reference's dense solve, one thread)."""
    import karam_b200 as K
    from karam_b200 import _abi as A
    from karam_b200 import circuits
    from oracle import pyoracle
    nl = circuits.config2()
    inst = circuits.mc_instances(nl, n_instances)
    prob = K.Problem(ctx, nl, max_instances=n_instances)
    prob.set_instances(inst)
    v, st = prob.solve_dc(K.options(precision=A.PREC_MIXED, **POLISH))
    conv = [i for i in range(n_instances) if st[i]["status"] == A.ST_CONVERGED]
    prob.ac_sweep(f_start, f_stop, n_points, input_node)  # warm-up
    t = time.perf_counter()
    f, x, status = prob.ac_sweep(f_start, f_stop, n_points, input_node)
    wall = time.perf_counter() - t
    dev_ms = prob.timing()["job_ms"]
    ok_points = int(np.sum(status == A.ST_CONVERGED))
    kind = "ref" if pyoracle.available("ref") else "port"
    if kind == "port":
        pyoracle.build("port")
    worst, cpu_t = 0.0, 0.0
    with native_stdout_to_stderr():
        orc = pyoracle.Oracle(kind)
        for i in conv[:oracle_sample]:
            t0 = time.perf_counter()
            x_ref, _ = orc.ac(nl, v[i], f_start, f_stop, n_points, input_node, inst=inst, idx=i)
            cpu_t += time.perf_counter() - t0
            worst = max(worst, float(np.max(np.abs(x[i] - x_ref) / (1e-9 * np.abs(x_ref) + 1e-12))))
    prob.close()
    n_done = min(oracle_sample, len(conv))
    return {
        "workload": f"config-2 MC batch ({n_instances} instances, n = {nl.n_nodes}) at its DC points, "
                    f"{n_points} log-spaced points {f_start:g}..{f_stop:g} Hz, input node {input_node}",
        "points_per_s": ok_points / wall, "points_per_s_device": ok_points / (dev_ms * 1e-3),
        "wall_ms": wall * 1e3, "device_ms": dev_ms, "points_ok": ok_points,
        "points": n_instances * n_points, "dc_converged": len(conv),
        "max_scaled_err_vs_oracle": worst,
        "scaled": "|dv| / (1e-9 |v| + 1e-12 V) on complex node voltages",
        "cpu_baseline": {"value": n_done * n_points / cpu_t if cpu_t else None, "unit": "points/s",
                         "cores": 1, "kind": "reference" if kind == "ref" else "port",
                         "sample": f"{n_done} instances x {n_points} points, dense complex LU "
                                   f"(solveComplexLU_Sparse), {cpu_t:.2f} s"},
    }


def config1_latency(ctx, reps=50):
    """Config 1: plain FP64 DC operating point of the 32-stage chain (VIN 0.9 V),
    single instance, no seed, no batching: latency per solve through the C ABI
    (host wall clock per call, and the device time of the job), NR iterations
    beside the reference-built oracle's."""
    import karam_b200 as K
    from karam_b200 import _abi as A
    from karam_b200 import circuits
    from oracle import pyoracle
    nl = circuits.config1()
    prob = K.Problem(ctx, nl, max_instances=1)
    prob.set_instances(None)

    def timed(schedule):
        opts = K.options(precision=A.PREC_FP64, schedule=schedule)
        for _ in range(3):
            prob.solve_dc(opts)
        wall, dev = [], []
        for _ in range(reps):
            t0 = time.perf_counter()
            v, st = prob.solve_dc(opts)
            wall.append(time.perf_counter() - t0)
            dev.append(prob.timing()["job_ms"])
        return v, st, 1e6 * statistics.median(wall), 1e3 * statistics.median(dev), prob.timing()

    # the default schedule (the persistent kernel: every round in one launch)
    # and the round-per-launch graph of the block-per-instance kernels
    v, st, wall, dev, t = timed(0)
    vg, stg, wall_g, dev_g, _ = timed(-3)
    kind = "ref" if pyoracle.available("ref") else "port"
    if kind == "port":
        pyoracle.build("port")
    with native_stdout_to_stderr():
        orc = pyoracle.Oracle(kind)
        v_ref, st_ref = orc.solve_dc(nl)
        cpu = []
        for _ in range(20):  # the reference CPU path, one host thread, same run
            t0 = time.perf_counter()
            orc.solve_dc(nl)
            cpu.append(time.perf_counter() - t0)
    prob.close()
    return {"workload": "32-stage inverter chain, VIN 0.9 V, n=34; plain FP64 DC, 1 instance",
            "us_per_solve_wall": wall, "us_per_solve_device": dev,
            "schedule": "persistent CTA (all NR rounds in one launch)" if t["level_schedule"] == 5
                        else f"level_schedule {t['level_schedule']}",
            "rounds": t["rounds"],
            "graph_rounds": {"us_per_solve_wall": wall_g, "us_per_solve_device": dev_g,
                             "schedule": "CUDA graph of per-round launches (CTA per instance, packed)",
                             "identical_result": bool(np.array_equal(v, vg))},
            "cpu_reference": {"us_per_solve": 1e6 * statistics.median(cpu), "cores": 1,
                              "kind": "reference" if kind == "ref" else "port",
                              "sample": "20 solves of the same DC, one host thread"},
            "iterations": st[0]["iterations"], "iterations_oracle": st_ref["iterations"],
            "converged": st[0]["status"] == A.ST_CONVERGED,
            "max_abs_diff_vs_oracle_v": float(np.max(np.abs(v[0] - v_ref)))}


CONFIG3_FIRST = 6_000_000  # Monte-Carlo ids of the uneven batch's load parameters


def config3_uneven(device, n_instances=2048, steps=500, dt=10e-12, oracle_sizes=(8, 9, 16)):
    """Uneven batch: n_instances N x N resistor grids with N ~ U{8..64}
    (circuits.config3_sizes), each a DC point then `steps` trapezoidal steps.

    One problem per grid size. Headline (mixed / fp64): every size in ONE
    launch of the multi-problem persistent kernel (karam_run_mc_multi, one
    CTA per instance, the largest grids first), wall clock of the call and the
    device time of the job. For comparison (per_size_streams): each size on
    its own context (stream) from host threads, each size's factor/solve
    schedule measured first by karam_tune_schedule; the two must give the
    same results (the schedules run the same elimination in the same order).
    FP32 LU + FP64 refinement against plain FP64. Every size shares one grid
    (seeded by N); instances vary in their loads' KP/VTO (ids from
    CONFIG3_FIRST). Accuracy: one instance of each sampled size against the
    reference-built oracle over the whole transient, which also gives the
    reference CPU rate on that sample."""
    import threading
    import karam_b200 as K
    from karam_b200 import _abi as A
    from karam_b200 import circuits
    sizes = circuits.config3_sizes(n_instances)
    groups = {}
    for i, N in enumerate(sizes):
        groups.setdefault(int(N), []).append(i)
    t0 = time.perf_counter()
    probs = []
    for N, ids in sorted(groups.items()):
        nl = circuits.grid_circuit(N)
        draws = [circuits.sample_mos_variation(nl, 1, first_instance=CONFIG3_FIRST + i) for i in ids]
        inst = circuits.Instances(len(ids), np.concatenate([d[0] for d in draws]),
                                  np.concatenate([d[1] for d in draws]))
        ctx = K.Context(device)
        prob = K.Problem(ctx, nl, max_instances=len(ids))
        prob.set_instances(inst)
        probs.append((N, ids, nl, inst, ctx, prob))
    t_build = time.perf_counter() - t0

    def run(prec, n_steps):
        opts = K.options(precision=prec, max_halvings=MAX_HALVINGS, **POLISH)
        errs = []

        def one(prob):
            try:
                prob.run_mc_device(dt, n_steps, A.TRAN_TRAP, opts)
                prob.sync()
            except Exception as e:  # re-raised below
                errs.append(e)
        threads = [threading.Thread(target=one, args=(g[5],)) for g in probs]
        t = time.perf_counter()
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        wall = time.perf_counter() - t
        if errs:
            raise errs[0]
        out = {}
        conv = 0
        kinds = {}
        for N, ids, nl, inst, ctx, prob in probs:
            v, st = prob.read_results()
            conv += sum(1 for s in st if s["status"] == A.ST_CONVERGED)
            k = ["pivot records", "warp per instance", "CTA per instance, shared memory",
                 "CTA per instance, global memory",
                 "CTA per instance, packed program",
                 "persistent CTA per instance",
                 "CTA per instance, global memory, solve vector in global memory"][
                     prob.timing()["level_schedule"]]
            kinds[k] = kinds.get(k, 0) + 1
            out[N] = (v, st)
        return wall, conv, kinds, out

    streams = {}
    for name, prec in (("mixed", A.PREC_MIXED), ("fp64", A.PREC_FP64)):
        # the measured schedule of every size (karam_tune_schedule: 16 DC
        # rounds per feasible schedule), before timing
        t = time.perf_counter()
        for g in probs:
            g[5].tune_schedule(K.options(precision=prec, max_halvings=MAX_HALVINGS, **POLISH), 16)
        t_tune = time.perf_counter() - t
        run(prec, 4)  # warm-up: plans, workspaces, graphs
        wall, conv, kinds, out = run(prec, steps)
        streams[name] = {"solves_per_s": conv * (steps + 1) / wall, "wall_s": wall,
                         "converged": conv, "schedules_by_size": kinds, "tune_s": t_tune,
                         "_out": out}
    # the same batch again as one launch, the per-size contexts freed first
    for g in probs:
        g[5].close()
        g[4].close()
    shared_ctx = K.Context(device)
    multi = []
    for N, ids, nl, inst, _, _ in probs:
        mp = K.Problem(shared_ctx, nl, max_instances=len(ids))
        mp.set_instances(inst)
        multi.append(mp)

    def run_one_launch(prec, n_steps):
        opts = K.options(precision=prec, max_halvings=MAX_HALVINGS, **POLISH)
        t = time.perf_counter()
        K.run_mc_multi(multi, dt, n_steps, A.TRAN_TRAP, opts)
        wall = time.perf_counter() - t
        out, conv = {}, 0
        for (N, *_), mp in zip(probs, multi):
            v, st = mp.read_results()
            conv += sum(1 for s in st if s["status"] == A.ST_CONVERGED)
            out[N] = (v, st)
        return wall, multi[0].timing(), conv, out

    res = {}
    for name, prec in (("mixed", A.PREC_MIXED), ("fp64", A.PREC_FP64)):
        run_one_launch(prec, 4)  # warm-up: plans, workspaces
        wall, tm, conv, out = run_one_launch(prec, steps)
        same = all(np.array_equal(out[N][0], streams[name]["_out"][N][0]) and
                   [s["status"] for s in out[N][1]] == [s["status"] for s in streams[name]["_out"][N][1]]
                   for N in out)
        res[name] = {"solves_per_s": conv * (steps + 1) / wall, "wall_s": wall,
                     "device_ms": tm["job_ms"],
                     "solves_per_s_device": conv * (steps + 1) / (tm["job_ms"] * 1e-3),
                     "rounds_max": tm["rounds"], "converged": conv, "launches": 1,
                     "equals_per_size_streams": bool(same), "_out": out}
        streams[name].pop("_out")
        res[name]["per_size_streams"] = streams[name]
    for mp in multi:
        mp.close()
    shared_ctx.close()
    both = []
    for N, ids, *_ in probs:
        vm, sm = res["mixed"]["_out"][N]
        vf, sf = res["fp64"]["_out"][N]
        for k in range(len(ids)):
            if sm[k]["status"] == A.ST_CONVERGED and sf[k]["status"] == A.ST_CONVERGED:
                both.append(float(np.max(np.abs(vm[k] - vf[k]) / (1e-9 * np.abs(vf[k]) + 1e-12))))
    # the smallest instances against the reference-built oracle
    from oracle import pyoracle
    kind = "ref" if pyoracle.available("ref") else "port"
    if kind == "port":
        pyoracle.build("port")
    worst, cpu_t, cpu_solves, sample = 0.0, 0.0, 0, []
    by_size = {}
    with native_stdout_to_stderr():
        orc = pyoracle.Oracle(kind)
        # one instance of each sampled size over the whole transient, the sizes
        # side by side on host threads (the oracle releases the interpreter)
        chosen = [g for g in probs if g[0] in oracle_sizes]
        outs = {}

        def one(g):
            N, ids, nl, inst, ctx, prob = g
            t = time.perf_counter()
            outs[N] = orc.run_batch(nl, inst, 0, 1, dt=dt, n_steps=steps, method=A.TRAN_TRAP,
                                    n_threads=1, linear_solver=pyoracle.LS_SPARSE,
                                    max_halvings=MAX_HALVINGS, polish_max=8) + (time.perf_counter() - t,)
        threads = [threading.Thread(target=one, args=(g,)) for g in chosen]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        for N, ids, nl, inst, ctx, prob in chosen:
            v_ref, st, secs = outs[N]
            vm, sm = res["mixed"]["_out"][N]
            cpu_t += secs
            if st[0]["converged"] and sm[0]["status"] == A.ST_CONVERGED:
                cpu_solves += steps + 1
                e = float(np.max(np.abs(vm[0] - v_ref[0]) / (1e-9 * np.abs(v_ref[0]) + 1e-12)))
                worst = max(worst, e)
                by_size[N] = e
            sample.append(f"N={N} (n={prob.n})")
    for r in res.values():
        r.pop("_out")
    return {
        "workload": f"{n_instances} N x N resistor grids, N ~ U{{8..64}} ({len(groups)} sizes, "
                    f"n = 66..4098), 1 pF caps, diode clamps at 10 % and pulsed NMOS loads at 5 % "
                    f"of nodes; DC + {steps} trapezoidal steps of {dt * 1e12:g} ps",
        "problems": len(groups), "build_s": t_build,
        "mixed": res["mixed"], "fp64": res["fp64"],
        "speedup_mixed_vs_fp64": res["mixed"]["solves_per_s"] / res["fp64"]["solves_per_s"],
        "max_scaled_diff_mixed_vs_fp64": max(both) if both else None,
        "max_scaled_err_vs_oracle": worst,
        "scaled_err_vs_oracle_by_size": by_size,
        "fixture_check": grid_fixture_check(device),
        "scaled": "|dv| / (1e-9 |v| + 1e-12 V)",
        "cpu_baseline": {"value": cpu_solves / cpu_t if cpu_t else None, "unit": "solves/s",
                         "cores": 1, "kind": "reference" if kind == "ref" else "port",
                         "sample": "one instance of each of the sizes " + ", ".join(sample)
                                   + f", full transient, {cpu_t:.1f} s of CPU time (one thread each)"},
    }


def grid_fixture_check(device):
    """The larger grids of the family (16 x 16, 32 x 32, 64 x 64) against the
    fixtures generated from the reference-built library (tests/golden/gridN.npz:
    DC of two Monte-Carlo instances, then 20 trapezoidal steps of 40 ps over
    the gate ramp for instance 0), mixed precision on the default schedule:
    max |dv| / (1e-9 |v| + 1e-12 V) of the DC points, the final point and the
    recorded waveform."""
    import karam_b200 as K
    from karam_b200 import _abi as A
    from karam_b200 import circuits
    out = {}
    ctx = K.Context(device)
    for N in (16, 32, 64):
        path = os.path.join(ROOT, "tests", "golden", f"grid{N}.npz")
        if not os.path.exists(path):
            continue
        g = np.load(path)
        nl = circuits.grid_circuit(N)
        prob = K.Problem(ctx, nl, max_instances=2)
        prob.set_instances(circuits.Instances(2, g["mc_kp"], g["mc_vto"]))
        opts = K.options(precision=A.PREC_MIXED, max_halvings=6, **POLISH)
        v, st = prob.solve_dc(opts)
        sc = lambda a, b: float(np.max(np.abs(a - b) / (1e-9 * np.abs(b) + 1e-12)))
        dc = max(sc(v[i], g["dc_v"][i]) for i in range(2))
        nodes = [int(x) for x in g["tran_wave_nodes"]]
        vt, stt, wave = prob.step_transient(40e-12, 20, A.TRAN_TRAP, opts, wave_nodes=nodes)
        out[f"N={N}"] = {"n": prob.n, "dc": dc, "final": sc(vt[0], g["tran_v"]),
                         "wave_max_abs_v": float(np.max(np.abs(wave[0] - g["tran_wave"]))),
                         "converged": bool(st[0]["status"] == A.ST_CONVERGED and
                                           stt[0]["status"] == A.ST_CONVERGED)}
        prob.close()
    ctx.close()
    return out


def config5_seeder(ctx, n_train=200704, n_test=16384, batch=4096, epochs=10, stages=256,
                   oracle_sample=16):
    """Config 5: the learned seeder on the inverter-chain family (`stages`
    stages, VIN 0.9 V) with VDD ~ U(1.2, 2.0) and the MC device variation:
    trained on plain-NR DC solutions of n_train instances, evaluated on n_test
    held-out instances against a plain start (reference seed + GMIN stepping):
    NR iterations, solves/s and the fallback rate; the inference's tcgen05
    GEMM throughput inside the timed jobs; and, on oracle_sample instances the
    plain GPU NR failed and as many it converged, whether the reference-built
    oracle (FP64, sparse LU) reaches the same outcome. VDD draws: numpy PCG64
    seeded by the batch's first instance id."""
    import karam_b200 as K
    from karam_b200 import _abi as A
    from karam_b200 import circuits
    from oracle import pyoracle
    nl = circuits.inverter_chain(stages=stages, vdd=1.8, vin=0.9)

    def instances(first, n):
        inst = circuits.mc_instances(nl, n, first_instance=first)
        vdd = np.random.default_rng(first).uniform(1.2, 2.0, n)
        inst.vs_dc = np.stack([vdd, np.full(n, 0.9)], axis=1)
        return inst

    prob = K.Problem(ctx, nl, max_instances=batch)
    plain = K.options(precision=A.PREC_MIXED, **POLISH)
    t0 = time.perf_counter()
    seeder = K.Seeder(prob, width=512, hidden_layers=3, init_seed=5)
    added = 0
    for b in range(n_train // batch):
        prob.set_instances(instances(2_000_000 + b * batch, batch))
        prob.solve_dc(plain)
        added += seeder.add_dc(prob)
    t1 = time.perf_counter()
    loss = seeder.train(epochs=epochs, batch=256, lr=1e-3, shuffle_seed=7)
    t2 = time.perf_counter()
    prob.set_seeder(seeder)
    seeded = K.options(precision=A.PREC_MIXED, seeded=A.SEED_MLP, **POLISH)
    res = {"plain": {"ms": 0.0, "it": [], "conv": 0}, "seeded": {"ms": 0.0, "it": [], "conv": 0}}
    fallbacks = 0
    err = []
    diff = 0.0
    seed_ms = 0.0
    failed, passed = [], []  # (batch first id, index) of plain-NR outcomes, for the oracle check
    for b in range(n_test // batch):
        first = 3_000_000 + b * batch
        prob.set_instances(instances(first, batch))
        v0, st0 = prob.solve_dc(plain)
        res["plain"]["ms"] += prob.timing()["job_ms"]
        failed += [(first, i) for i, s in enumerate(st0) if s["status"] != A.ST_CONVERGED]
        passed += [(first, i) for i, s in enumerate(st0) if s["status"] == A.ST_CONVERGED]
        guess = seeder.predict(prob)
        v1, st1 = prob.solve_dc(seeded)
        res["seeded"]["ms"] += prob.timing()["job_ms"]
        seed_ms += prob.timing()["seed_ms"]
        for k, st in (("plain", st0), ("seeded", st1)):
            res[k]["it"] += [s["iterations"] + s["polish_iters"] for s in st]
            res[k]["conv"] += sum(s["status"] == A.ST_CONVERGED for s in st)
        fallbacks += sum(1 for s in st1 if not s["seeded_ok"])
        ok = [i for i, (a, c) in enumerate(zip(st0, st1))
              if a["status"] == A.ST_CONVERGED and c["status"] == A.ST_CONVERGED]
        err += np.max(np.abs(guess[ok] - v0[ok]), axis=1).tolist()
        diff = max(diff, float(np.max(np.abs(v1[ok] - v0[ok]) / (1e-9 * np.abs(v0[ok]) + 1e-12))))
    prob.set_seeder(None)
    seeder.close()
    n_out = prob.n
    prob.close()
    dims = [2 * len(nl.mos) + len(nl.vsrc), 512, 512, 512, n_out]
    flops_per_row = 2.0 * sum(a * b for a, b in zip(dims[:-1], dims[1:]))
    peak = measured_peaks(kind="bf16")[0]
    jobs = n_test // batch
    inf_tflops = flops_per_row * batch / (seed_ms / jobs / 1e3) / 1e12 if seed_ms else None
    train_tflops = 3.0 * flops_per_row * added * epochs / (t2 - t1) / 1e12
    # the plain outcome against the reference-built oracle on a sample of the
    # failures and of the converged instances
    kind = "ref" if pyoracle.available("ref") else "port"
    if kind == "port":
        pyoracle.build("port")
    agree = {"gpu_failed": 0, "oracle_failed_too": 0, "gpu_converged": 0, "oracle_converged_too": 0}
    pick = np.random.default_rng(5)
    fail_sel = []
    with native_stdout_to_stderr():
        orc = pyoracle.Oracle(kind)
        for group, key, okey in ((failed, "gpu_failed", "oracle_failed_too"),
                                 (passed, "gpu_converged", "oracle_converged_too")):
            if not group:
                continue
            sel = [group[j] for j in pick.choice(len(group), min(oracle_sample, len(group)), replace=False)]
            for first, i in sel:
                inst1 = instances(first, batch).slice(i, i + 1)
                _, st = orc.run_batch(nl, inst1, 0, 1, n_threads=1, linear_solver=pyoracle.LS_SPARSE, **POLISH)
                agree[key] += 1
                agree[okey] += int(bool(st[0]["converged"]) == (key == "gpu_converged"))
                if key == "gpu_failed":
                    fail_sel.append((inst1, bool(st[0]["converged"])))
    # the same failures of the mixed-precision plain start, solved again on the
    # GPU in FP64: does the outcome follow the precision or the algorithm?
    if fail_sel:
        sub_inst = circuits.Instances(len(fail_sel), np.concatenate([x.mos_kp for x, _ in fail_sel]),
                                      np.concatenate([x.mos_vto for x, _ in fail_sel]),
                                      np.concatenate([x.vs_dc for x, _ in fail_sel]))
        p64 = K.Problem(ctx, nl, max_instances=len(fail_sel))
        p64.set_instances(sub_inst)
        _, st64 = p64.solve_dc(K.options(precision=A.PREC_FP64, **POLISH))
        p64.close()
        agree["fp64_gpu_converged"] = sum(s["status"] == A.ST_CONVERGED for s in st64)
        agree["fp64_gpu_agrees_with_oracle"] = sum((s["status"] == A.ST_CONVERGED) == oc
                                                   for s, (_, oc) in zip(st64, fail_sel))
    out = {"workload": f"{stages}-stage inverter chain, VIN 0.9 V, VDD ~ U(1.2, 2.0) + MC VTO/KP; DC",
           "network": f"MLP {dims[0]}-512-512-512-{n_out} (GELU), "
                      "BF16 weights, FP32 accumulation, Adam/MSE",
           "inference": {"ms_per_batch": seed_ms / jobs if jobs else None, "batch": batch,
                         "gflop_per_batch": flops_per_row * batch / 1e9,
                         "tflops": inf_tflops, "frac_of_bf16_peak": inf_tflops / peak if inf_tflops else None,
                         "peak_tflops": peak,
                         "timed": "features + four tcgen05 GEMM layers + activations, CUDA events in the job"},
           "training_tflops": train_tflops,
           "plain_outcome_vs_oracle": {**agree, "oracle": kind,
                                       "sample": f"{oracle_sample} plain-NR failures and {oracle_sample} "
                                                 "converged instances, FP64 sparse LU"},
           "train_solutions": added, "train_data_s": t1 - t0, "train_s": t2 - t1,
           "epochs": epochs, "final_loss": loss, "heldout": n_test,
           "fallback_rate": fallbacks / n_test,
           "seed_err_median_v": float(np.median(err)), "seed_err_max_v": float(np.max(err)),
           "max_scaled_diff_seeded_vs_plain": diff,
           "scaled": "|dv| / (1e-9 |v| + 1e-12 V) over instances converged both ways"}
    for k in ("plain", "seeded"):
        it = np.array(res[k]["it"])
        out[k] = {"solves_per_s": res[k]["conv"] / (res[k]["ms"] / 1e3),
                  "nr_iterations_mean": float(it.mean()), "nr_iterations_p99": float(np.percentile(it, 99)),
                  "converged": res[k]["conv"]}
    return out


def accuracy_check(nl, inst, v_mixed, v_fp64, st_mixed, st_fp64, sample=6):
    """Max relative error of the final transient voltages against the FP64
    oracle (fully polished) on a few instances, and mixed vs FP64 GPU paths on
    every instance."""
    from karam_b200 import _abi as A
    from oracle import pyoracle
    kind = "ref" if pyoracle.available("ref") else "port"
    if kind == "port":
        pyoracle.build("port")
    idx = [i for i, s in enumerate(st_mixed) if s["status"] == A.ST_CONVERGED][:sample]
    sub = inst.slice(min(idx), max(idx) + 1) if idx else None
    worst = 0.0
    worst_rel = 0.0
    if idx:
        with native_stdout_to_stderr():
            orc = pyoracle.Oracle(kind)
            v_ref, st = orc.run_batch(nl, sub, 0, sub.n, dt=DT, n_steps=TRAN_STEPS,
                                      n_threads=os.cpu_count() or 1,
                                      linear_solver=pyoracle.LS_SPARSE,
                                      max_halvings=MAX_HALVINGS, polish_max=8)
        for i in idx:
            r = v_ref[i - min(idx)]
            d = np.abs(v_mixed[i] - r)
            worst = max(worst, float(np.max(d / (1e-9 * np.abs(r) + 1e-12))))
            big = np.abs(r) > 1e-3
            if big.any():
                worst_rel = max(worst_rel, float(np.max(d[big] / np.abs(r[big]))))
    both = [i for i, (s, f) in enumerate(zip(st_mixed, st_fp64))
            if s["status"] == A.ST_CONVERGED and f["status"] == A.ST_CONVERGED]
    d = np.abs(v_mixed[both] - v_fp64[both])
    diff = float(np.max(d / (1e-9 * np.abs(v_fp64[both]) + 1e-12))) if both else None
    return {"max_scaled_err_vs_oracle": worst, "max_rel_err_vs_oracle_above_1mV": worst_rel,
            "oracle": kind, "instances_checked": len(idx),
            "max_scaled_diff_mixed_vs_fp64": diff, "instances_converged_both": len(both),
            "scaled": "|dv| / (1e-9 |v| + 1e-12 V); <= 1 meets the 1e-9 relative bar"}


def outcome_check(nl, inst, st_mixed, st_fp64, converged_sample=16):
    """Which instances fail, and whether the reference-built oracle (FP64,
    sparse LU, plain GMIN stepping) fails on the same ones: every instance the
    plain FP64 GPU arm did not converge, plus as many it converged (seeded
    draw), each run DC + the full BE transient on its own host thread."""
    import threading
    from karam_b200 import _abi as A
    from oracle import pyoracle
    kind = "ref" if pyoracle.available("ref") else "port"
    if kind == "port":
        pyoracle.build("port")
    fail64 = [i for i, s in enumerate(st_fp64) if s["status"] != A.ST_CONVERGED]
    failmx = [i for i, s in enumerate(st_mixed) if s["status"] != A.ST_CONVERGED]
    conv = [i for i, s in enumerate(st_fp64) if s["status"] == A.ST_CONVERGED]
    pick = np.random.default_rng(3)
    conv = sorted(pick.choice(conv, min(converged_sample, len(conv)), replace=False).tolist())
    res = {}
    with native_stdout_to_stderr():
        orc = pyoracle.Oracle(kind)

        def one(i):
            _, st = orc.run_batch(nl, inst.slice(i, i + 1), 0, 1, dt=DT, n_steps=TRAN_STEPS,
                                  n_threads=1, linear_solver=pyoracle.LS_SPARSE,
                                  max_halvings=MAX_HALVINGS, polish_max=8)
            res[i] = bool(st[0]["converged"])
        ids = sorted(set(fail64) | set(failmx) | set(conv))
        for k in range(0, len(ids), os.cpu_count() or 1):
            threads = [threading.Thread(target=one, args=(i,)) for i in ids[k:k + (os.cpu_count() or 1)]]
            for th in threads:
                th.start()
            for th in threads:
                th.join()
    return {"failed_fp64_arm": fail64, "failed_headline_arm": failmx,
            "oracle_failed": [i for i in ids if not res[i]],
            "fp64_arm_agrees_with_oracle": sum(res[i] == (st_fp64[i]["status"] == A.ST_CONVERGED)
                                               for i in ids),
            "checked": len(ids), "oracle": kind,
            "sample": f"every instance either GPU arm failed plus {len(conv)} the FP64 arm converged; "
                      "DC + full BE transient each"}


def spawn_ranks(n):
    """`--gpus n` outside a launcher: start n local ranks through
    torch.distributed.run (rendezvous on 127.0.0.1) and return their exit
    code. Refuses rather than measure fewer GPUs than asked for."""
    import socket
    import subprocess
    try:
        import torch
        visible = torch.cuda.device_count()
    except Exception:
        visible = 0
    if visible < n:
        print(json.dumps({"metric": METRIC, "error": f"--gpus {n} needs {n} visible GPUs, "
                          f"{visible} are visible"}), flush=True)
        return 2
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__),
           *sys.argv[1:]]
    return subprocess.run(cmd).returncode


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    dist = Dist(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, dist)
        else:
            run_karam(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
