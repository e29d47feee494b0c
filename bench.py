#!/usr/bin/env python
"""Benchmark of the Groth16/BN128 prover hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--no-cpu]

Prints ONE JSON line (rank 0).  Under torchrun (N > 1) every rank runs its own replica of
the workload (proofs are independent: no data-path collective); the timed region is
bracketed by barriers, device time is the max over ranks, and ``value`` is the total over
all ranks (weak scaling).  With N > 1 the line also carries ``sharded_g1_msm_2^20``: one
2^20-term G1 MSM split over the N GPUs (one-point NCCL all-gather of the partial sums), the
strong-scaling case of a single MSM.

Workload (the configuration the headline metric is quoted on): full Groth16 prove for a
synthetic R1CS of 2^20 constraints (nConstraints = 2^20 - 2, one public input, A and B rows
with 3 nonzeros with uniform random Fr coefficients over earlier wires -- every wire but the
last layer's is read in A and in B -- C row = one output wire set to (A.w)(B.w)); proving key
from seeded toxic waste, resident in HBM with its fixed-base MSM tables; fixed r, s.

``value``: the served engine -- one step = one proof from a device-resident witness, K proofs
overlapped across --slots contexts, device time (CUDA events on a marker stream) around all K.
``e2e``: the same through the public C ABI prove server (cs_server_*), witness in host
memory, proof back in host memory, K requests submitted at once, wall clock.
``latency_ms``: p50/p99 submit -> proof through the server under Poisson arrivals at 70% of
that saturated rate.  ``single_proof``: one proof per call (cs_prove_device), device time.
``plain_per_call``: the reference's flow through the drop-in entry points (mpoly_eval_server_h,
ntt_interpolandmul_server_h, ec_jacreduce_server_h per MSM with the key points copied per
call), wall clock; ``served_vs_plain`` = e2e / plain.  ``served_mix``: 8 circuits spanning
2^12..2^20 constraints (both ends and six seeded log-uniform sizes; the 2^20 one is the
headline circuit), requests uniform over them, saturation and Poisson 50% / 90% with p50/p99.  ``batched_msm``: 64 G1 + 8 G2 MSMs of 2^floor(U(10,20))
terms in one batch plan per group (autotuned windows, CUDA graph replay) vs one call per
instance.  Also one BN128 G1 MSM of 2^20 terms (``g1_msm_2^20_ms``: generic bases, scalars split
by GLV) and the fixed-base G1 MSM a proof runs four times over the same bases
(``g1_fixed_msm_2^20_ms``), whose bucket-accumulation kernel -- the dominant kernel of every
proof -- carries the roofline.

``proof_check``: every proof of the timed served run and of the e2e run equals the
one-proof-per-call proof byte for byte; on rank 0 at N = 1 that proof also equals the
reference's CPU proving sequence run in the reference's own library on the same key,
witness, r and s, and passes the Groth16 pairing check.

``cpu_baseline``: that CPU proof, timed -- one whole 2^20-constraint proof of the
benchmark circuit through the reference's own CPU implementation (oracle/_ref, built from
the reference sources; the C restatement when that library is absent) on all host cores,
stage by stage (QAP, H step, five multi-exponentiations).

``per_config`` (rank 0, N = 1): the single-op configurations against the reference library
on the same seeded inputs, results compared word for word -- one G1 MSM of 2^16 terms
(config 1), the 2^20 NTT, INTT and H step (config 2): GPU device ms beside CPU wall ms.

``--impl reference``: the same CPU prover alone, in a process that never loads this
library: the 2^20 circuit and key are built on the CPU (oracle/synth_cpu.py, word for word
the GPU builder's), untimed; each step is the next stage of the 2^20 proving sequence (7
stages make one proof), so the K steps are bounded samples of the workload, and ``value`` is
1 / (the sum of the stages' mean times).  ``proof_sha256`` in both lines names the proof
each arm made from the same inputs.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "Groth16 proofs/s + p50/p99 latency, 2^20 G1 MSM ms; served vs plain, 1 B200"
UNIT = "proofs/s (2^20 constraints)"
# 256-bit Montgomery product, 8x32-bit limbs: 64 a*b + 64 m*p wide (32x32->64) products + 8 m
PRODUCTS_PER_MONT = 136
MONT_PER_MADD = 11     # mixed addition, 7M + 4S (the canonical count of the MSM cost model)
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one k_accumulate launch of
# the 2^20-term fixed-base G1 MSM (window 20), from an ncu capture of that launch
ACC_TRAFFIC_BYTES = 1_747_153_664 + 68_581_376
# smsp__issue_active (fraction of cycles issuing) and the busiest pipes of the same capture:
# the counter view of the roofline fraction below, whose peak is a builder-measured rate
ACC_NCU = {"issue_active": 0.593, "pipe_alu": 0.535, "pipe_fp64": 0.485}
L2_BYTES = 126 * 1024 * 1024
LOG_M = 20
R_INT, S_INT = 0x1234567890abcdef, 0xfedcba0987654321
CIRCUIT_SEED, KEY_SEED = 100, 101


# ----------------------------------------------------------------- clocks sampler ---
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        threading.Thread(target=self._read, daemon=True).start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
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
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------- distributed ----
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    """Max of a per-rank device time over all ranks (NCCL on the GPUs; gloo on the host)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def pct(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = min(len(xs) - 1, max(0, int(round(q / 100.0 * (len(xs) - 1)))))
    return xs[k]


# ---------------------------------------------------------------- CPU reference ------
def cpu_reference_prove(pk_host: dict, w: np.ndarray):
    """One proof of the benchmark circuit by the reference's CPU proving sequence in the
    reference's own library (oracle/_ref; the restatement where it is absent), all host
    threads, timed stage by stage.  Returns (proof, seconds per stage, kind, threads)."""
    from oracle.oracle import Oracle, RefLib
    from oracle.prover import cpu_prove_stages
    o = Oracle()
    ref = RefLib.get() if RefLib.available() else None
    stages, st = cpu_prove_stages(o, pk_host, w, R_INT, S_INT, ref=ref)
    times = {}
    for name, fn in stages:
        t0 = time.perf_counter()
        fn()
        times[name] = time.perf_counter() - t0
    return st["proof"], times, ("reference" if ref else "port"), (os.cpu_count() or 1)


def proof_sha256(proof: np.ndarray) -> str:
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(proof, dtype=np.uint32).tobytes()).hexdigest()


# ----------------------------------------------------------------------- workloads ---
class ProveWorkload:
    def __init__(self, ctx, log_m: int, seed: int):
        import torch
        from cusnarks_b200.groth import SyntheticCircuit, setup_pk, Prover
        from cusnarks_b200.synth import to_limbs
        self.torch = torch
        self.ctx = ctx
        self.circ = SyntheticCircuit(ctx, log_m, seed=seed)
        self.pk = setup_pk(ctx, self.circ, seed=seed + 1)
        self.prover = Prover(ctx, self.pk)
        self.r, self.s = to_limbs(R_INT), to_limbs(S_INT)
        dev = torch.device("cuda", ctx.device)
        self.d_w = self.circ.d_w
        self.d_proof = torch.zeros(64, dtype=torch.int32, device=dev)
        self.h_w = torch.from_numpy(self.circ.w.view(np.int32)).pin_memory()
        self.h_proof = torch.zeros(64, dtype=torch.int32).pin_memory()
        self.flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()

    def l2_flush(self):
        self.flush.add_(1)
        self.torch.cuda.synchronize()

    def step(self) -> float:
        self.prover.prove_device(self.d_w.data_ptr(), self.r, self.s, self.d_proof.data_ptr())
        self.ctx.sync()
        return self.ctx.last_ms

    def e2e_step(self) -> float:
        from cusnarks_b200._lib import lib, check
        t0 = time.perf_counter()
        check(lib().cs_prove(self.ctx.handle, self.prover.handle, self.h_w.data_ptr(), self.r.ctypes.data,
                             self.s.ctypes.data, self.h_proof.data_ptr()), self.ctx.handle)
        return (time.perf_counter() - t0) * 1e3

    @property
    def h2d_bytes(self):
        return self.circ.n_vars * 32 + 64

    d2h_bytes = 256


class MsmWorkload:
    def __init__(self, ctx, log_n: int, seed: int):
        import torch
        from cusnarks_b200.synth import random_field, g1_generator
        self.torch = torch
        self.ctx = ctx
        self.n = 1 << log_n
        rng = np.random.Generator(np.random.PCG64(seed))
        dev = torch.device("cuda", ctx.device)
        self.d_k = torch.from_numpy(random_field(rng, self.n).view(np.int32)).to(dev)
        self.d_s = torch.from_numpy(random_field(rng, self.n).view(np.int32)).to(dev)
        g = torch.from_numpy(g1_generator().view(np.int32)).to(dev)
        self.d_p = torch.empty((self.n, 16), dtype=torch.int32, device=dev)
        self.d_out = torch.zeros(16, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        ctx.scmul_device(self.d_k.data_ptr(), g.data_ptr(), self.n, self.d_p.data_ptr(), point_stride_words=0)
        ctx.sync()
        self.keep = g

    def step(self):
        """The generic MSM (cs_msm_device): (ms, bucket-accumulation ms)."""
        self.ctx.msm_device(self.d_s.data_ptr(), self.d_p.data_ptr(), self.n, self.d_out.data_ptr())
        self.ctx.sync()
        return self.ctx.last_ms, self.ctx.last_phase_ms

    def build_fixed(self):
        """The fixed-base table of the proof's G1 MSMs over the same bases (window c: W = 254 / c
        + 1 windows, table T[j n + i] = 2^(c j) P_i), built untimed."""
        from cusnarks_b200 import Context
        self.c_fixed = Context.msm_fixed_window(self.n)
        pts = Context.msm_fixed_table_points(self.n, self.c_fixed)
        self.d_table = self.torch.empty((pts, 16), dtype=self.torch.int32, device=self.d_p.device)
        self.ctx.msm_fixed_table_device(self.d_p.data_ptr(), self.n, self.c_fixed, self.d_table.data_ptr())
        self.ctx.sync()

    def step_fixed(self):
        """The fixed-base MSM a proof runs four times (cs_msm_fixed_device): (ms, accumulation ms)."""
        self.ctx.msm_fixed_device(self.d_s.data_ptr(), self.d_table.data_ptr(), self.n, self.c_fixed,
                                  self.d_out.data_ptr())
        self.ctx.sync()
        return self.ctx.last_ms, self.ctx.last_phase_ms

    def fixed_units(self):
        """Bucket entries of one fixed-base accumulation launch: n terms x (254 / c + 1) windows."""
        from cusnarks_b200._lib import lib
        return self.n * lib().cs_msm_num_windows(self.c_fixed), self.c_fixed


def sharded_msm_leg(ctx, world, rank, reps: int, log_n: int = 20, seed: int = 7):
    """One 2^log_n G1 MSM split over all ranks (cusnarks_b200.sharded): each rank makes its own
    shard's bases and scalars on its GPU; per call, local MSM + one-point all-gather (NCCL) +
    point sum.  Device span per rank (events around the synchronising call), max over ranks."""
    import torch
    from cusnarks_b200.sharded import sharded_msm, shard_range
    from cusnarks_b200.synth import random_field, g1_generator
    n = 1 << log_n
    lo, hi = shard_range(n, rank, world)
    rng = np.random.Generator(np.random.PCG64(seed + 31 * rank))
    dev = torch.device("cuda", ctx.device)
    k = torch.from_numpy(random_field(rng, hi - lo).view(np.int32)).to(dev)
    sc = torch.from_numpy(random_field(rng, hi - lo).view(np.int32)).to(dev)
    g = torch.from_numpy(g1_generator().view(np.int32)).to(dev)
    pts = torch.empty((hi - lo, 16), dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    ctx.scmul_device(k.data_ptr(), g.data_ptr(), hi - lo, pts.data_ptr(), point_stride_words=0)
    ctx.sync()
    for _ in range(2):
        sharded_msm(ctx, sc, pts)
    spans = []
    for _ in range(reps):
        barrier(world)
        spans.append(device_span_ms(lambda: sharded_msm(ctx, sc, pts)))
    ms = max_over_ranks(statistics.median(spans), world)
    return {"ms": round(ms, 3), "terms": n, "terms_per_rank": hi - lo, "ranks": world,
            "basis": "one 2^20 G1 MSM split over the ranks (contiguous shards, one-point NCCL all-gather, "
                     "point sum); device span per call, median of reps, max over ranks (strong scaling)"}


class ServedDevice:
    """Proofs from a device-resident witness overlapped across `slots` contexts (each with
    its own streams and scratch): the served engine without the host copies."""

    def __init__(self, wl, slots: int, max_requests: int):
        import torch
        from cusnarks_b200 import Context
        self.wl = wl
        self.ctxs = [wl.ctx] + [Context(wl.ctx.device) for _ in range(slots - 1)]
        dev = torch.device("cuda", wl.ctx.device)
        # one output per request, so every proof of a run can be checked afterwards
        self.proofs = torch.zeros((max(max_requests, slots), 64), dtype=torch.int32, device=dev)

    def run(self, k: int):
        from cusnarks_b200._lib import lib, check
        wl = self.wl
        for i in range(k):
            c = self.ctxs[i % len(self.ctxs)]
            check(lib().cs_prove_device(c.handle, wl.prover.handle, _vp(wl.d_w.data_ptr()), wl.r.ctypes.data,
                                        wl.s.ctypes.data, _vp(self.proofs[i].data_ptr())), c.handle)
        for c in self.ctxs:
            c.sync()

    def close(self):
        for c in self.ctxs[1:]:
            c.close()


def _vp(x):
    import ctypes
    return ctypes.c_void_p(x)


def device_span_ms(fn):
    """Device time (CUDA events on a marker stream) around fn(), which synchronises."""
    import torch
    s = torch.cuda.Stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(s)
    fn()
    torch.cuda.synchronize()
    b.record(s)
    b.synchronize()
    return a.elapsed_time(b)


def served_run(srv, jobs, rate_hz=None, seed=0, proofs=None):
    """Submits jobs [(key, w, r, s)] all at once (rate_hz None) or as a Poisson stream;
    returns (wall seconds first submit -> last proof, latencies ms); appends the proofs to
    `proofs` when given."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t0 = time.perf_counter()
    tickets = []
    at = 0.0
    for key, w, r, s in jobs:
        if rate_hz:
            at += rng.exponential(1.0 / rate_hz)
            dt = t0 + at - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
        tickets.append(srv.submit(key, w, r, s))
    lat = []
    for t in tickets:
        pr, info = srv.wait(t)
        lat.append(info["latency_ms"])
        if proofs is not None:
            proofs.append(pr)
    return time.perf_counter() - t0, lat


def served_mix(ctx, slots: int, n_requests: int, seed: int = 5, big=None):
    """Config 5: 8 circuits spanning 2^12..2^20 constraints (the two ends plus six seeded
    log-uniform draws), keys resident, requests over them (uniform) at Poisson rates 50% /
    90% of the measured saturation.  big: (circuit, prover) of a 2^20 circuit to reuse."""
    from cusnarks_b200.groth import SyntheticCircuit, setup_pk, Prover
    from cusnarks_b200.server import ProveServer
    from cusnarks_b200.synth import to_limbs
    rng = np.random.Generator(np.random.PCG64(seed))
    logs = sorted([12, 20] + [int(x) for x in rng.integers(12, 21, 6)])
    circs, provers, owned = [], [], []
    for i, lm in enumerate(logs):
        if lm == 20 and big is not None and big[0] not in circs:
            circs.append(big[0])
            provers.append(big[1])
            continue
        c = SyntheticCircuit(ctx, lm, seed=300 + i)
        circs.append(c)
        provers.append(Prover(ctx, setup_pk(ctx, c, seed=400 + i)))
        owned.append(provers[-1])
    srv = ProveServer(ctx.device, slots=slots, reserve_bytes=1 << 30)
    keys = [srv.add_key(p) for p in provers]
    r, s = to_limbs(0x1234567890abcdef), to_limbs(0xfedcba0987654321)
    pick = rng.integers(0, 8, n_requests)
    jobs = [(keys[k], circs[k].w, r, s) for k in pick]
    served_run(srv, jobs)                         # warm every slot's scratch, twiddles and batch plans
    wall, lat = served_run(srv, jobs)
    sat = len(jobs) / wall
    out = {"circuits_log2": logs, "slots": slots, "requests": len(jobs),
           "saturation": {"proofs_per_s": round(sat, 2), "p50_ms": round(pct(lat, 50), 2),
                          "p99_ms": round(pct(lat, 99), 2), "arrivals": "all at once"}}
    for frac in (0.5, 0.9):
        wall, lat = served_run(srv, jobs, rate_hz=frac * sat, seed=seed + int(frac * 10))
        out[f"poisson_{int(frac * 100)}pct"] = {"rate_hz": round(frac * sat, 2),
                                                "proofs_per_s": round(len(jobs) / wall, 2),
                                                "p50_ms": round(pct(lat, 50), 2), "p99_ms": round(pct(lat, 99), 2)}
    out["max_concurrent"] = srv.stats()["max_concurrent"]
    srv.close()
    for p in owned:
        p.close()
    return out


def batched_msm(ctx, reps: int, seed: int = 4):
    """Config 4: 64 G1 + 8 G2 MSMs, N = 2^floor(U(10, 20)) (seeded), bases from seeded pools of
    k_i * G, scalars uniform in Fr; one batch plan per group (windows autotuned), replayed as
    CUDA graphs; compared with one cs_msm_device call per instance (default windows)."""
    import torch
    from cusnarks_b200.synth import random_field, g1_generator, g2_generator
    rng = np.random.Generator(np.random.PCG64(seed))
    dev = torch.device("cuda", ctx.device)
    out = {"instances": {"g1": 64, "g2": 8}}
    groups = []
    for ec2, count in ((False, 64), (True, 8)):
        pw = 32 if ec2 else 16
        logs = [int(x) for x in rng.integers(10, 21, count)]
        sizes = [1 << L for L in logs]
        pool_n = max(sizes)
        k = torch.from_numpy(random_field(rng, pool_n).view(np.int32)).to(dev)
        g = torch.from_numpy((g2_generator() if ec2 else g1_generator()).view(np.int32)).to(dev)
        pool = torch.empty((pool_n, pw), dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        ctx.scmul_device(k.data_ptr(), g.data_ptr(), pool_n, pool.data_ptr(), ec2=ec2, point_stride_words=0)
        ctx.sync()
        sc = torch.from_numpy(random_field(rng, sum(sizes)).view(np.int32)).to(dev)
        outs = torch.zeros((count, pw), dtype=torch.int32, device=dev)
        ref = torch.zeros((count, pw), dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        offs = np.concatenate([[0], np.cumsum(sizes)])
        jobs = []
        for q, n in enumerate(sizes):
            p0 = int(rng.integers(0, pool_n - n + 1))
            jobs.append((sc.data_ptr() + 32 * int(offs[q]), pool.data_ptr() + 4 * pw * p0, n,
                         outs.data_ptr() + 4 * pw * q))
        tuned = ctx.msm_autotune(10, 20, ec2=ec2)
        groups.append((ec2, logs, jobs, outs, ref, tuned, (k, g, pool, sc)))
    plans = [ctx.msm_batch(jobs, ec2=ec2) for ec2, _, jobs, _, _, _, _ in groups]

    def run_batch():
        for pl in plans:
            pl.run(graph=True)
        ctx.sync()

    def run_single():
        for ec2, _, jobs, _, ref, _, _ in groups:
            pw = 32 if ec2 else 16
            for q, (s_, p_, n, _) in enumerate(jobs):
                ctx.msm_device(s_, p_, n, ref.data_ptr() + 4 * pw * q, ec2=ec2)
        ctx.sync()

    for _ in range(2):
        run_batch()
        run_single()
    tb = min(device_span_ms(run_batch) for _ in range(reps))
    ts = min(device_span_ms(run_single) for _ in range(reps))
    equal = all(torch.equal(o, r) for _, _, _, o, r, _, _ in groups)
    out.update({"log2_sizes_g1": groups[0][1], "log2_sizes_g2": groups[1][1],
                "terms": {"g1": int(sum(1 << L for L in groups[0][1])), "g2": int(sum(1 << L for L in groups[1][1]))},
                "windows_tuned_g1": groups[0][5], "windows_tuned_g2": groups[1][5],
                "batch_ms": round(tb, 3), "per_call_ms": round(ts, 3), "speedup": round(ts / tb, 3),
                "graph": True, "equal_to_single": bool(equal),
                "basis": "device time (CUDA events) of the two graph replays (G1 batch, G2 batch) vs 72 "
                         "cs_msm_device calls; best of the timed repetitions"})
    for pl in plans:
        pl.close()
    return out


def run_ours(args, world, rank, local):
    import torch
    from cusnarks_b200 import Context
    from cusnarks_b200.context import kernel_launches
    ctx = Context(local)
    peak_wide = ctx.pipe_rate(3)
    wl = ProveWorkload(ctx, args.log_m, seed=CIRCUIT_SEED + rank)
    sd = ServedDevice(wl, args.slots, args.steps)
    # one proof per call (resident key): lone-proof device latency
    for _ in range(args.warmup):
        wl.step()
    single = []
    for _ in range(args.steps):
        wl.l2_flush()
        single.append(wl.step())
    ref_proof = wl.d_proof.cpu().numpy().view(np.uint32).copy()
    # served engine, device witness: `steps` proofs overlapped across the slots
    for _ in range(args.warmup):
        sd.run(args.slots)
    sampler = ClockSampler(local) if rank == 0 else None
    barrier(world)
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
    l0 = kernel_launches()
    span = device_span_ms(lambda: sd.run(args.steps))
    launches = kernel_launches() - l0
    barrier(world)
    clocks = sampler.stop() if sampler else None
    total_ms = max_over_ranks(span, world)
    ms_per_step = total_ms / args.steps
    value = world * 1e3 / ms_per_step
    served_proofs = sd.proofs[:args.steps].cpu().numpy().view(np.uint32)
    served_equal = bool((served_proofs == ref_proof[None, :]).all())
    sd.close()
    # end to end: the C-ABI server, host witness in, proof out to host
    from cusnarks_b200.server import ProveServer
    srv = ProveServer(local, slots=args.slots, reserve_bytes=1 << 30)
    key = srv.add_key(wl.prover)
    # at least 30 requests: with fewer, the pipeline's fill and drain dominate the wall clock
    jobs = [(key, wl.circ.w, wl.r, wl.s)] * max(30, args.steps)
    served_run(srv, jobs[:args.slots])
    e2e_proofs = []
    wall, lat_sat = served_run(srv, jobs, proofs=e2e_proofs)
    e2e_equal = all(np.array_equal(pr, ref_proof) for pr in e2e_proofs)
    e2e_ms = max_over_ranks(wall * 1e3 / len(jobs), world)
    # latency under a Poisson stream at 70% of the saturated rate
    wall_p, lat = served_run(srv, jobs[:1] * 120, rate_hz=0.7 * 1e3 / e2e_ms, seed=11)
    srv.close()
    # plain per-call path: the reference's flow through the drop-in entry points
    from cusnarks_b200.groth import pk_to_host
    from cusnarks_b200.plain import PlainProver
    plain = PlainProver(pk_to_host(wl.pk))
    rr, ss = int.from_bytes(wl.r.tobytes(), "little"), int.from_bytes(wl.s.tobytes(), "little")
    plain.prove(wl.circ.w, rr, ss)
    t0 = time.perf_counter()
    n_plain = 2
    for _ in range(n_plain):
        plain.prove(wl.circ.w, rr, ss)
    plain_ms = (time.perf_counter() - t0) * 1e3 / n_plain
    del plain
    # the 2^20 G1 MSM (generic, GLV split) and the proof's dominant kernel: the bucket
    # accumulation of its fixed-base G1 MSMs (same bases and scalars, fixed-base table)
    mw = MsmWorkload(ctx, 20, seed=7 + rank)
    for _ in range(3):
        mw.step()
    msm_ms = []
    for _ in range(max(3, args.steps)):
        msm_ms.append(mw.step()[0])
        wl.l2_flush()
    mw.build_fixed()
    for _ in range(3):
        mw.step_fixed()
    fixed_ms, acc_ms = [], []
    for _ in range(max(3, args.steps)):
        t, a = mw.step_fixed()
        fixed_ms.append(t)
        acc_ms.append(a)
        wl.l2_flush()
    units, window = mw.fixed_units()
    acc = statistics.mean(acc_ms)
    achieved = units * MONT_PER_MADD * PRODUCTS_PER_MONT / (acc * 1e-3)
    e2e_val = world * 1e3 / e2e_ms
    line = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32x8 (256-bit Montgomery integers)",
        "data": "synthetic: seeded R1CS (3 nonzeros per A/B row, every wire used), seeded toxic waste, "
                "GPU-generated key",
        "config": {"workload": "Groth16 prove, synthetic R1CS 2^20 constraints (domain 2^20), proving key "
                               "and fixed-base tables resident in HBM, fixed r,s",
                   "n_vars": wl.circ.n_vars, "domain": 1 << args.log_m,
                   "path": f"served engine: proofs overlapped over {args.slots} slots, device witness",
                   "l2": "inputs larger than L2 (proving key + tables ~6 GB)"},
        "latency_ms": {"p50": round(pct(lat, 50), 3), "p99": round(pct(lat, 99), 3),
                       "basis": "served (C-ABI server, host witness), Poisson arrivals at 70% of the "
                                "saturated rate, 2^20 circuit, submit -> proof in host memory"},
        "single_proof": {"proofs_per_s": round(1e3 / statistics.median(single), 3),
                         "p50_ms": round(pct(single, 50), 3), "p99_ms": round(pct(single, 99), 3),
                         "basis": "one proof per call (cs_prove_device), device time"},
        "served_vs_single": round(value / world * statistics.median(single) / 1e3, 3),
        "plain_per_call": {"proofs_per_s": round(1e3 / plain_ms, 3), "ms": round(plain_ms, 1),
                           "basis": "the reference's flow through the drop-in entry points: mpoly_eval, "
                                    "ntt_interpolandmul, 6 ec_jacreduce calls; the key's point arrays are "
                                    "built once per key on the host and copied to the GPU by every call, "
                                    "with the call's scalars; wall clock"},
        "served_vs_plain": round(e2e_val * plain_ms / 1e3, 2),
        "g1_msm_2^20_ms": round(statistics.median(msm_ms), 3),
        "g1_fixed_msm_2^20_ms": round(statistics.median(fixed_ms), 3),
        "roofline": {"bound": "int issue (ALU column sums + FP64 split products)",
                     "kernel": "k_accumulate+k_combine (bucket accumulation of the proof's fixed-base G1 MSMs)",
                     "achieved": round(achieved / 1e12, 4), "peak": round(peak_wide / 1e12, 4),
                     "unit": "T wide products/s", "frac": round(achieved / peak_wide, 4),
                     "traffic": ACC_TRAFFIC_BYTES, "ncu": ACC_NCU,
                     "kernel_ms": round(acc, 4), "units_per_launch": units,
                     "window": window,
                     "basis": "2^20-term fixed-base G1 MSM as in the proof: N*(254/c+1) bucket entries x 11 Montgomery products x 136 32x32->64 "
                              "products / kernel ms (CUDA events around the kernels); peak = live "
                              "mad.wide.u32 rate (cs_bench_pipe mode 3), the ceiling of a 32-bit CIOS "
                              "product (this kernel computes products in radix 2^52 on the FP64 pipe); "
                              "traffic = ncu DRAM bytes per launch"},
        "e2e": {"value": round(e2e_val, 3), "unit": UNIT, "ms": round(e2e_ms, 3),
                "h2d_bytes_per_step": wl.h2d_bytes, "d2h_bytes_per_step": wl.d2h_bytes,
                "basis": f"C-ABI prove server ({args.slots} slots), {len(jobs)} requests submitted at once, "
                         "host witness in, proof out; wall clock"},
        "gpu_launches": launches,
        "clocks": clocks,
        "proof_check": {"served_bytes_equal": served_equal, "served_proofs": int(served_proofs.shape[0]),
                        "e2e_bytes_equal": bool(e2e_equal), "e2e_proofs": len(e2e_proofs),
                        "proof_sha256": proof_sha256(ref_proof),
                        "basis": "every proof of the timed served run and of the e2e run equals the "
                                 "one-proof-per-call proof (cs_prove_device) byte for byte"},
    }
    if world > 1:  # every rank takes part (collective)
        line["sharded_g1_msm_2^20"] = sharded_msm_leg(ctx, world, rank, reps=max(3, args.steps))
    if rank == 0 and not args.no_batch:
        line["batched_msm"] = batched_msm(ctx, reps=3)
    if rank == 0 and not args.no_mix:
        line["served_mix"] = served_mix(ctx, args.slots, args.mix_requests, big=(wl.circ, wl.prover))
    if rank == 0 and world == 1 and not args.no_cpu:
        from cusnarks_b200.groth import pk_to_host
        from oracle.prover import verify
        host = pk_to_host(wl.pk)
        cpu_proof, stage_s, kind, threads = cpu_reference_prove(host, wl.circ.w)
        sec = sum(stage_s.values())
        line["cpu_baseline"] = {"value": round(1.0 / sec, 6), "unit": UNIT, "cores": threads, "kind": kind,
                                "sample": "one whole proof of the 2^20-constraint benchmark circuit (same key, "
                                          "witness, r, s as the GPU proofs): the reference's CPU proving "
                                          "sequence in its own library, all host threads",
                                "s_per_proof": round(sec, 2),
                                "stages_s": {k: round(v, 3) for k, v in stage_s.items()}}
        line["proof_check"]["cpu_reference_bytes_equal"] = bool(np.array_equal(cpu_proof, ref_proof))
        line["proof_check"]["pairing"] = bool(verify(host["vk"], ref_proof, wl.circ.public_inputs))
        line["proof_check"]["basis"] += ("; on rank 0 it also equals the reference library's CPU proof and "
                                         "passes the Groth16 pairing check")
        line["per_config"] = per_config_leg(ctx, reps=max(3, args.steps))
    if rank == 0:
        print(json.dumps(line), flush=True)
    wl.prover.close()
    ctx.close()


def per_config_leg(ctx, reps: int):
    """The single-op configurations, GPU against the reference's CPU library on the same seeded
    inputs (results compared word for word): config 1, one G1 MSM of 2^16 terms
    (ec_jacreduce_server_h); config 2, the 2^20 NTT and INTT (ntt_h / intt_h) and the 2^20 H
    step (ntt_interpolandmul_server_h; the coset variant has no reference counterpart).  GPU:
    device ms (CUDA events), median of reps; CPU: one call, wall clock, all host threads."""
    import torch
    from oracle.oracle import Oracle, RefLib, hstep_roots_table, random_field as fr_random
    from cusnarks_b200.synth import random_field, g1_generator
    if not RefLib.available():
        return {"unavailable": "oracle/_ref (the reference library) is not built"}
    ref, o = RefLib.get(), Oracle()
    dev = torch.device("cuda", ctx.device)
    out = {"cpu_threads": os.cpu_count() or 1}

    def gpu_ms(call):
        ts = []
        for _ in range(reps + 1):
            call()
            ctx.sync()
            ts.append(ctx.last_ms)
        return statistics.median(ts[1:])

    def cpu_s(call):
        t0 = time.perf_counter()
        r = call()
        return r, time.perf_counter() - t0

    def host(t):
        return t.cpu().numpy().view(np.uint32)

    # config 1
    n = 1 << 16
    rng = np.random.Generator(np.random.PCG64(16))
    dk = torch.from_numpy(random_field(rng, n).view(np.int32)).to(dev)
    s = random_field(rng, n)
    ds = torch.from_numpy(s.view(np.int32)).to(dev)
    g = torch.from_numpy(g1_generator().view(np.int32)).to(dev)
    dp = torch.empty((n, 16), dtype=torch.int32, device=dev)
    dout = torch.zeros(16, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    ctx.scmul_device(dk.data_ptr(), g.data_ptr(), n, dp.data_ptr(), point_stride_words=0)
    ctx.sync()
    ms = gpu_ms(lambda: ctx.msm_device(ds.data_ptr(), dp.data_ptr(), n, dout.data_ptr()))
    want, sec = cpu_s(lambda: ref.msm(s, host(dp), 0, 6))
    out["config1_g1_msm_2^16"] = {"gpu_ms": round(ms, 3), "cpu_ms": round(sec * 1e3, 1),
                                  "equal": bool(np.array_equal(host(dout), want))}
    # config 2
    L = 20
    rng = np.random.Generator(np.random.PCG64(220))
    A = o.to_mont(fr_random(rng, 1 << L, 1), 1)  # Fr elements (pidx 1), as the config-2 tests draw them
    B = o.to_mont(fr_random(rng, 1 << L, 1), 1)
    dA, dB = torch.from_numpy(A.view(np.int32)).to(dev), torch.from_numpy(B.view(np.int32)).to(dev)
    dF, dI = torch.empty_like(dA), torch.empty_like(dA)
    dM = torch.zeros((2 << L, 8), dtype=torch.int32, device=dev)
    dH = torch.zeros((1 << L, 8), dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    roots = o.find_roots(L)
    f_ms = gpu_ms(lambda: ctx.ntt_device(dA.data_ptr(), dF.data_ptr(), L, 1))
    i_ms = gpu_ms(lambda: ctx.ntt_device(dA.data_ptr(), dI.data_ptr(), L, -1, fmat=1))
    F, f_s = cpu_s(lambda: ref.ntt(A, roots, L))
    Iv, i_s = cpu_s(lambda: ref.intt(A, roots, L, 1, 1))
    out["config2_ntt_2^20"] = {"gpu_ms": round(f_ms, 3), "cpu_ms": round(f_s * 1e3, 1),
                               "equal": bool(np.array_equal(host(dF), F))}
    out["config2_intt_2^20"] = {"gpu_ms": round(i_ms, 3), "cpu_ms": round(i_s * 1e3, 1),
                                "equal": bool(np.array_equal(host(dI), Iv))}
    h_ms = gpu_ms(lambda: ctx.hstep_device(0, dA.data_ptr(), dB.data_ptr(), 0, L, dM.data_ptr()))
    M, h_s = cpu_s(lambda: ref.interpolandmul(A, B, hstep_roots_table(o, L), L, 2, os.cpu_count() or 1))
    out["config2_hstep_2^20"] = {"gpu_ms": round(h_ms, 3), "cpu_ms": round(h_s * 1e3, 1),
                                 "equal": bool(np.array_equal(host(dM), M))}
    c_ms = gpu_ms(lambda: ctx.hstep_device(1, dA.data_ptr(), dB.data_ptr(), dB.data_ptr(), L, dH.data_ptr()))
    out["config2_hstep_coset_2^20"] = {"gpu_ms": round(c_ms, 3)}
    return out


def run_reference(args, world, rank):
    """The reference's own CPU prover on the 2^20 workload, in a process that never loads this
    library: the circuit and key are built on the CPU (untimed); step i runs stage i mod 7 of
    the proving sequence (QAP, H step, five multi-exponentiations), all host threads."""
    if rank != 0:
        return
    from oracle.oracle import Oracle, RefLib
    from oracle.prover import cpu_prove_stages, verify
    from oracle.synth_cpu import CpuCircuit, cpu_setup_pk
    o = Oracle()
    t0 = time.perf_counter()
    circ = CpuCircuit(o, args.log_m, seed=CIRCUIT_SEED)
    pk = cpu_setup_pk(o, circ, seed=KEY_SEED)
    prep_s = time.perf_counter() - t0
    ref = RefLib.get() if RefLib.available() else None
    kind, threads = ("reference" if ref else "port"), (os.cpu_count() or 1)
    stages, st = cpu_prove_stages(o, pk, circ.w, R_INT, S_INT, ref=ref)
    per = {name: [] for name, _ in stages}
    warm = {name: [] for name, _ in stages}
    timed = 0.0
    proof = None
    for i in range(args.warmup + args.steps):
        name, fn = stages[i % len(stages)]
        t = time.perf_counter()
        fn()
        dt = time.perf_counter() - t
        (per if i >= args.warmup else warm)[name].append(dt)
        if i >= args.warmup:
            timed += dt
        if proof is None and "proof" in st:
            proof = st["proof"].copy()
    for name, _, in stages:  # a stage the timed steps did not reach: its warm-up time
        if not per[name]:
            if not warm[name]:
                fn = dict(stages)[name]
                t = time.perf_counter()
                fn()
                warm[name].append(time.perf_counter() - t)
            per[name] = warm[name]
    stage_s = {k: statistics.mean(v) for k, v in per.items()}
    s_proof = sum(stage_s.values())
    val = 1.0 / s_proof
    if proof is None:
        proof = st.get("proof")
    line = {"metric": METRIC, "impl": "reference", "value": round(val, 6), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(timed * 1e3 / args.steps, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32x8 (256-bit Montgomery integers)",
            "data": "synthetic: the benchmark circuit and key, built on the CPU from the same seeds",
            "config": {"workload": f"Groth16 prove, synthetic R1CS 2^{args.log_m} constraints "
                                   f"(domain 2^{args.log_m}), fixed r,s",
                       "n_vars": circ.n_vars, "domain": 1 << args.log_m,
                       "step": "one stage of the proving sequence; 7 stages make one proof"},
            "steps_per_proof": len(stages), "s_per_proof": round(s_proof, 2),
            "stages_s": {k: round(v, 3) for k, v in stage_s.items()},
            "prep_s": round(prep_s, 1),
            "cpu_baseline": {"value": round(val, 6), "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": "stages of 2^20-constraint proofs, one per step, all host threads"},
            "e2e": {"value": round(val, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if proof is not None:
        line["proof_sha256"] = proof_sha256(proof)
        line["pairing"] = bool(verify(pk["vk"], proof, circ.public_inputs))
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--slots", type=int, default=3, help="concurrent proofs of the served engine")
    ap.add_argument("--no-mix", action="store_true", help="skip the mixed-size served leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-MSM leg")
    ap.add_argument("--mix-requests", type=int, default=96)
    ap.add_argument("--log-m", type=int, default=LOG_M,
                    help="constraint domain of the proving workload (the metric is quoted on 2^20)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup()
    run_ours(args, world, rank, local)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
