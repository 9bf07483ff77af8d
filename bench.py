#!/usr/bin/env python
"""Benchmark: stationary distributions per second on the n=20 precision network x 512
held-out rate sets (the learned-warm-start workload's held-out sweep).

One step = the whole hot path for one batch: bit-sliced transition table, SCC /
levels / reordering, terminal kernels, transient solve and x_inf + marginals for
512 (rate set, x0) pairs, inputs resident in HBM.  `value` = solves/s over all
ranks (max device time over ranks); `e2e` = the same through the public Python API
with pinned host inputs copied in and the results (marginals + terminal-state
probabilities, i.e. every nonzero of x_inf) copied back inside the timed region.

The metric compares the learned-warm-start + mixed-precision form with the plain FP64
form.  The headline (`--method direct`, default) is the plain FP64 level sweep, the
faster of the two on this workload; the learned+mixed form is timed the same way in
the same run (`learned_mixed`), after its network is trained outside the timed region
on the plain solves' occupations of the 3,584 training rate sets.  After the headline
(outside its steps) the many-network workload runs once through esl_solve_many
(`many_networks`: 48 networks, n 12-18, 64 x 16 systems each; --no-many skips it).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--method direct|learned|mixed|fp64]
    python bench.py --impl reference ...   # the CPU FP64 oracle on the host cores

Synthetic data: seeded random network (paraexastolog_b200.synth), no dataset.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

from paraexastolog_b200 import shards, synth  # noqa: E402

METRIC = "solves/s, n=20 x 512 rate sets, learned+mixed vs FP64 sparse LU at L1<=1e-9"
BATCH = 512


N_TRAIN = 3584


def workload(rank: int = 0, world: int = 1):
    """(network, this rank's rate sets, x0, training rate sets, [begin, end) of the
    rank's slice of the global sweep).  Weak scaling: the global sweep is the 512
    held-out rate sets followed, for world > 1, by further seeded log-uniform draws
    (shards.global_sweep); rank r solves its shard_bounds slice, BATCH rate sets."""
    w = synth.config_learned(n_rate_sets=4096)
    net = w.networks[0]
    held = np.ascontiguousarray(w.rates[0][-BATCH:])

    def draw(seed, count):
        return synth.log_uniform_rates(np.random.default_rng(10_000 + seed), net.n, count)

    rates, bounds = shards.rank_rate_sets(held, rank, world, draw)
    return (net, rates, np.ascontiguousarray(w.x0[0]), np.ascontiguousarray(w.rates[0][:N_TRAIN]), bounds)


def train_warm_start(esl, torch, ctx, net, x0, train_rates, steps: int, device: int):
    """Outside the timed region: plain FP64 (direct) occupations of the training rate sets,
    in chunks of BATCH, each followed by Adam steps of the warm-start network on it."""
    mlp = esl.Mlp(ctx, net, seed=0)
    occ = torch.empty((BATCH, net.N), dtype=torch.float64, device=f"cuda:{device}")
    t0 = time.perf_counter()
    chunks = (len(train_rates) + BATCH - 1) // BATCH
    loss = None
    for c in range(chunks):
        r = train_rates[c * BATCH:(c + 1) * BATCH]
        esl.solve_batch(ctx, net, r, x0, method=esl.METHOD_DIRECT, tol=1e-10, occupation=occ[: len(r)],
                        marginals=False)
        loss = mlp.train(r, occ[: len(r)], steps=steps // chunks, batch=16384, lr=2e-3)
    torch.cuda.synchronize(device)
    del occ
    return mlp, {"train_rate_sets": len(train_rates), "adam_steps": steps // chunks * chunks, "batch": 16384,
                 "final_loss": loss, "seconds": time.perf_counter() - t0, "targets": mlp.n_targets}


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def bf16_peak():
    """Measured dense bf16 tensor throughput (TFLOP/s, burst), or the fallback."""
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f).get("bf16_tflops", 1590.0))
    return 1590.0


def traffic_per_byte():
    """DRAM bytes per algorithmic byte of the largest group's Schur operator from the
    committed ncu capture summary (64 systems, two 32-system tiles), or None."""
    path = os.path.join(REPO, "profiles", "schur_operator_largest_group_n20_x64_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f).get("dram_bytes_per_algorithmic_byte")


class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
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
        reasons = sorted({names[j] for r in rows for j in range(4) if r[5 + j].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def kernel_rooflines(entries):
    """Per kernel class of one profiled step: launches, device ms, algorithmic bytes
    and GB/s.  For the Schur operator and the BiCGStab updates, records of the largest
    level group (at least half the class's largest per-launch bytes) are listed apart."""
    out = []
    classes = sorted({e[0] for e in entries})
    for name in classes:
        rec = [e for e in entries if e[0] == name]
        groups = [("all", rec)]
        if name in ("schur_operator", "bicgstab_update"):
            cut = 0.5 * max(e[2] for e in rec)
            groups.append(("largest_level_group", [e for e in rec if e[2] >= cut]))
        for scope, rr in groups:
            ms = sum(e[1] for e in rr)
            by = sum(e[2] for e in rr)
            out.append({"kernel": name, "scope": scope, "launches": len(rr), "ms": ms,
                        "bytes_per_launch": by / len(rr), "achieved": by / (ms * 1e-3) / 1e9 if ms > 0 else None,
                        "unit": "GB/s"})
    return out


def table_rooflines(esl, torch, ctx, model, rates, label, repeats: int = 5):
    """k_flip_masks (out-masks only) and k_emit_csc of esl_table_build, best of
    `repeats` builds (the first one untimed)."""
    esl.table(ctx, model, rates, with_cols=False)
    best = {}
    for _ in range(repeats):
        ctx.set_profiling(True)
        esl.table(ctx, model, rates, with_cols=False)
        for name, ms, by in ctx.profile_entries():
            if name not in best or ms < best[name][0]:
                best[name] = (ms, by)
        ctx.set_profiling(False)
    torch.cuda.synchronize()
    return [{"kernel": name, "scope": label, "launches": 1, "ms": ms, "bytes_per_launch": by,
             "achieved": by / (ms * 1e-3) / 1e9 if ms > 0 else None, "unit": "GB/s", "timing": "best of 5"}
            for name, (ms, by) in sorted(best.items())]


def run_ours(args, rank, world, device):
    import torch
    import torch.distributed as dist

    import paraexastolog_b200 as esl

    torch.cuda.set_device(device)
    # one stream for torch's copies and the library's kernels, so that events on it time
    # the library's work and copies are ordered with it
    stream = torch.cuda.Stream(device)
    torch.cuda.set_stream(stream)
    ctx = esl.Context(device, stream)
    net_g, rates, x0, train_rates, bounds = workload(rank, world)
    model = esl.Model.parse(net_g.bnet)
    d_rates = torch.tensor(rates, device=f"cuda:{device}")
    d_x0 = torch.tensor(x0, device=f"cuda:{device}")
    N = 1 << model.n
    learned = args.method == "learned"
    solve_method = {"fp64": esl.METHOD_FP64, "mixed": esl.METHOD_MIXED, "direct": esl.METHOD_DIRECT,
                    "learned": esl.METHOD_MIXED}[args.method]
    mlp, train_info, warm_buf = None, None, None
    if learned or not args.no_compare:
        net0 = esl.Net.build(ctx, model, rates[0])
        mlp, train_info = train_warm_start(esl, torch, ctx, net0, x0, train_rates, args.train_steps, device)
        warm_buf = torch.empty((BATCH, N), dtype=torch.float64, device=f"cuda:{device}")

    def step(method=solve_method, use_warm=learned, dr=d_rates, dx=d_x0):
        net = esl.Net.build(ctx, model, rates[0])
        warm = mlp.predict(dr, out=warm_buf) if use_warm else None
        res = esl.solve_batch(ctx, net, dr, dx, method=method, tol=args.tol, warm=warm)
        return net, res

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(device)

    def timed(fn, steps):
        barrier()
        l0 = esl.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(device) as clk:
            e0.record(stream)
            for _ in range(steps):
                out = fn()
            e1.record(stream)
            barrier()
        return out, e0.elapsed_time(e1), esl.launch_count() - l0, clk.summary()

    tuning = None
    if not args.no_autotune and not args.profile_run:
        # level-sweep tiling for this batch, picked by timing (outside the timed region)
        tuning = esl.Net.build(ctx, model, rates[0]).autotune(d_rates, d_x0, method=solve_method, tol=args.tol)
    for _ in range(args.warmup):
        net, res = step()
    if args.profile_run:
        step()
        torch.cuda.synchronize(device)
        return None, None
    (net, res), ms, launches, clocks = timed(step, args.steps)
    iters, relres = res.report.iterations, res.report.relres
    last_xinf = res.x_inf

    # the other form of the metric's comparison, timed the same way on the same GPU and batch:
    # learned warm start + mixed precision when the headline is the plain FP64 form, and the
    # plain FP64 form otherwise
    other, other_xinf = None, None
    if not args.no_compare:
        if learned or args.method != "direct":
            o_step = lambda: step(method=esl.METHOD_DIRECT, use_warm=False)  # noqa: E731
            o_name = "direct"
        else:
            o_step = lambda: step(method=esl.METHOD_MIXED, use_warm=True)  # noqa: E731
            o_name = "learned+mixed"
        for _ in range(max(1, args.warmup - 1)):
            o_step()
        (_, ores), oms, _, _ = timed(o_step, args.steps)
        # the other form's results of its last timed step, for its error against the oracle
        other_xinf = ores.x_inf
        other = {"method": o_name, "value": BATCH * args.steps * world / (oms * 1e-3),
                 "ms_per_step": oms / args.steps, "iterations": ores.report.iterations,
                 "relres": ores.report.relres}
        if mlp is not None:
            # iterations of the mixed solve without the warm start, and the inference time alone
            cres = esl.solve_batch(ctx, net, d_rates, d_x0, method=esl.METHOD_MIXED, tol=args.tol)
            other["mixed_without_warm_start_iterations"] = cres.report.iterations
            _, pms, _, _ = timed(lambda: mlp.predict(d_rates, out=warm_buf), 3)
            other["warm_start_inference_ms"] = pms / 3
            # the inference's own roofline: layer 2 (128 x 128) on the tensor cores per
            # (target state, rate set) sample; layers 1 and 3 are per-sample vector work
            samples = mlp.n_targets * BATCH
            flops = 2.0 * 128 * 128 * samples
            tf = flops / (pms / 3 * 1e-3) / 1e12
            bf16 = bf16_peak()
            other["warm_start_inference_roofline"] = {
                "bound": "tensor", "kernel": "k_mlp_predict_tc (tcgen05.mma kind::f16, BF16 -> FP32 in TMEM, layer 2)",
                "samples": samples, "flop_per_sample": 2 * 128 * 128, "achieved": tf, "unit": "TFLOP/s",
                "peak": bf16, "frac": tf / bf16,
                "peak_kind": "measured dense bf16 (cuBLAS burst)"}
            other["warm_start_training"] = train_info

    # rooflines from live CUDA events on the library's stream: every hot kernel class of
    # one step (table masks, graph sweeps, Schur operator, BiCGStab updates), and the CSC
    # emission of the transition table of this network and of the n=22 drop-in network
    ctx.set_profiling(True)
    step()
    entries = ctx.profile_entries()
    ctx.set_profiling(False)
    kernels = kernel_rooflines(entries)
    kernels += table_rooflines(esl, torch, ctx, model, rates[0], "n20_bench_network")
    scale = synth.config_scale()
    m22 = esl.Model.parse(scale.networks[0].bnet)
    kernels += table_rooflines(esl, torch, ctx, m22, scale.rates[0][0], "n22_drop_in_network")
    del m22
    op = [e for e in entries if e[0] == "schur_operator"]
    op_ms, op_bytes = sum(e[1] for e in op), sum(e[2] for e in op)
    # the applications of the largest level group (the one that dominates the step)
    big_cut = 0.5 * max((e[2] for e in op), default=0.0)
    big = [e for e in op if e[2] >= big_cut]
    big_ms, big_bytes, big_n = sum(e[1] for e in big), sum(e[2] for e in big), len(big)

    # end to end through the public API: pinned host inputs, results back to host
    h_rates = torch.tensor(rates).pin_memory()
    h_x0 = torch.tensor(x0).pin_memory()
    term_idx = None
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h2d = d2h = 0
    f0.record(stream)
    t_wall = time.perf_counter()
    for _ in range(args.steps):
        dr = h_rates.to(f"cuda:{device}", non_blocking=True)
        dx = h_x0.to(f"cuda:{device}", non_blocking=True)
        h2d = dr.numel() * 8 + dx.numel() * 8
        net, res = step(dr=dr, dx=dx)
        if term_idx is None:
            order, _, _, _ = net.export()
            term_idx = order[: net.terminal_states].long()
        probs = res.x_inf[:, 0, :].index_select(1, term_idx).cpu()
        marg = res.marginals.cpu()
        d2h = probs.numel() * 8 + marg.numel() * 8
    f1.record(stream)
    barrier()
    e2e_ms = f0.elapsed_time(f1)
    e2e_wall = time.perf_counter() - t_wall

    ms, e2e_ms = shards.max_over_ranks([ms, e2e_ms], world, device=f"cuda:{device}")
    out = None
    if rank == 0:
        solves = BATCH * args.steps * world
        peak, peak_kind = peaks()
        for k in kernels:
            k["peak"] = peak
            k["frac"] = k["achieved"] / peak if k.get("achieved") else None
        achieved_all = op_bytes / (op_ms * 1e-3) / 1e9 if op_ms > 0 else None
        achieved = big_bytes / (big_ms * 1e-3) / 1e9 if big_ms > 0 else None
        tpb = traffic_per_byte()
        value = solves / (ms * 1e-3)
        out = {
            "metric": METRIC,
            "value": value,
            "unit": "solves/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": {"direct": "f64", "fp64": "f64"}.get(args.method, "f32+f64"),
            "data": "synthetic (seeded random Boolean network, log-uniform rates)",
            "config": {"workload": f"n20_precision_network_x_{BATCH}_heldout_rate_sets", "n_nodes": model.n,
                       "states": N, "batch_rate_sets": BATCH, "initial_distributions": 1,
                       "method": "learned+mixed" if learned else args.method, "tol_relres": args.tol,
                       "l2": "working set > L2 (x_inf alone is 4 GB per step)",
                       "parallelism": f"replicas x{world} (rate-set shards)",
                       "sweep": f"rank 0 solves rate sets [{bounds[0]}, {bounds[1]}) of a {BATCH * world}-set "
                                "global sweep (the 512 held-out sets, then seeded draws for world > 1)",
                       "denominator": "the plain FP64 form is a level sweep of FP64 BiCGStab on the odd-row "
                                      "Schur complement of each level group (no sparse LU factorisation)",
                       "step": ("table + SCC/levels/order + terminal kernels + " +
                                ("warm-start inference + " if learned else "") +
                                "transient solve + x_inf/marginals")},
            "e2e": {"value": solves / (e2e_ms * 1e-3), "unit": "solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "wall_s": e2e_wall},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm",
                         "kernel": "schur_operator (k_sw_elim_pr + k_sw_apply_pr, paired rows) of the largest level group",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None,
                         "peak_kind": peak_kind,
                         "traffic": (big_bytes / big_n) * tpb if (tpb and big_n) else None,
                         "algorithmic_bytes_per_launch": big_bytes / big_n if big_n else None,
                         "launches": big_n,
                         "all_groups": {"achieved": achieved_all,
                                        "frac": achieved_all / peak if achieved_all else None,
                                        "launches": len(op),
                                        "note": "first poll window of every Krylov group; small groups "
                                                "are launch-latency bound"},
                         "kernels": kernels},
            "solver": {"iterations": iters, "relres": relres},
            "clocks": clocks,
        }
        if tuning:
            out["config"]["tiling"] = tuning
        if other:
            other["value_over_headline"] = other["value"] / value
            out["learned_mixed" if other["method"] == "learned+mixed" else "plain_fp64"] = other
    if out is not None and other_xinf is not None:
        out["_other_xinf"] = other_xinf
    return out, last_xinf


def cpu_baseline(sample: int, rank: int = 0, world: int = 1, threads: int = 0):
    """The CPU FP64 oracle on this host's cores over a bounded sample of the rank's rate
    sets; returns (baseline record, seconds, the oracle's x_inf of the sample)."""
    import oracle as O

    net_g, rates, x0, _, _ = workload(rank, world)
    m = O.Model(text=net_g.bnet)
    sym = m.analyse(rates[0])
    threads = threads or min(os.cpu_count() or 1, sample)
    r = rates[:sample]
    xs = np.broadcast_to(x0, (sample, x0.size)).copy()
    t = time.perf_counter()
    ref, _ = sym.solve_many(r, xs, threads=threads)
    dt = time.perf_counter() - t
    return {"value": sample / dt, "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"{sample} of the 512 held-out rate sets, oracle symbolic analysis excluded"}, dt, ref


def many_networks(device: int, reps: int = 2):
    """The many-network workload (48 random networks, n = 12..18, 64 rate sets x 16
    initial distributions each: 49,152 solves) through one esl_solve_many call over four
    contexts.  Net.build runs outside the timing; rates and x0 are resident on the
    device.  Wall clock with the device synchronised on both sides, best of `reps`
    after one untimed call.  Returns (record, results of the last call)."""
    import torch

    import paraexastolog_b200 as esl
    w = synth.config_batch()
    dev = f"cuda:{device}"
    ctxs = [esl.Context(device, torch.cuda.Stream(device)) for _ in range(4)]
    jobs = []
    for i, (net_g, rates, xs) in enumerate(zip(w.networks, w.rates, w.x0)):
        net = esl.Net.build(ctxs[i % len(ctxs)], esl.Model.parse(net_g.bnet), rates[0])
        jobs.append((net, torch.tensor(rates, device=dev), torch.tensor(xs, device=dev)))
    res = esl.solve_many(ctxs, jobs, method=esl.METHOD_DIRECT, tol=1e-10)
    times = []
    for _ in range(reps):
        del res
        torch.cuda.synchronize(device)
        t = time.perf_counter()
        res = esl.solve_many(ctxs, jobs, method=esl.METHOD_DIRECT, tol=1e-10)
        torch.cuda.synchronize(device)
        times.append(time.perf_counter() - t)
    solves = sum(int(r.x_inf.shape[0]) * int(r.x_inf.shape[1]) for r in res)
    rec = {"workload": "batch48_n12_18: 48 random networks, n 12-18, 64 rate sets x 16 x0 each",
           "value": solves / min(times), "unit": "solves/s", "solves": solves, "seconds": min(times),
           "timing": "wall clock around one esl_solve_many call (4 contexts), device synchronised on both "
                     "sides; Net.build outside",
           "converged": all(r.report.converged == 1 and r.status == 0 for r in res)}
    return rec, w, res


def cpu_baseline_many(w, res, n_sample: int = 6):
    """CPU baseline and accuracy of the many-network workload: the FP64 oracle on a seeded
    sample of (network, rate set, x0) triples, one host thread each."""
    from concurrent.futures import ThreadPoolExecutor

    import oracle as O
    rng = np.random.default_rng(48)
    picks = [(int(i), int(rng.integers(0, 64)), int(rng.integers(0, 16)))
             for i in rng.choice(len(w.networks), n_sample, replace=False)]

    def one(p):
        i, b, q = p
        sym = O.Model(text=w.networks[i].bnet).analyse(w.rates[i][b])
        t = time.perf_counter()
        ox, _ = sym.solve(w.x0[i][q], w.rates[i][b])
        return ox, time.perf_counter() - t

    with ThreadPoolExecutor(n_sample) as ex:
        refs = list(ex.map(one, picks))
    l1 = max(float(np.abs(res[i].x_inf[b, q].cpu().numpy() - ox).sum()) for (i, b, q), (ox, _) in zip(picks, refs))
    cpu_s = sum(dt for _, dt in refs)
    return ({"value": n_sample / cpu_s, "unit": "solves/s", "cores": 1, "kind": "port",
             "sample": f"{n_sample} (network, rate set, x0) triples, one thread each; per-core rate, oracle "
                       "symbolic analysis excluded"},
            {"solves": n_sample, "l1_max": l1, "target_l1": 1e-9})


def run_reference(args):
    # one rate set per host thread, up to 128 threads (~60 MB each): a step takes about
    # one oracle solve (~35 s) however many threads run
    sample = max(8, min(os.cpu_count() or 8, 128))
    for _ in range(min(args.warmup, 1)):
        cpu_baseline(sample)
    total, solves = 0.0, 0
    for _ in range(args.steps):
        cb, dt, _ = cpu_baseline(sample)
        total += dt
        solves += sample
    value = solves / total
    cb["value"] = value
    # n_gpus is the N this arm was launched with (so that it pairs with our arm's line);
    # the work itself runs on the host cores of rank 0 only
    return {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "n20_precision_network_x_512_heldout_rate_sets", "sample_per_step": sample,
                       "device": "host cores of rank 0 (no GPU)"},
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    global BATCH
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--method", default="direct", choices=["direct", "learned", "mixed", "fp64"],
                    help="headline form: direct = plain FP64 level sweep (the fastest here); "
                         "learned = learned warm start + mixed precision")
    ap.add_argument("--train-steps", type=int, default=1400, help="Adam steps of the warm-start network")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip timing the other form of the comparison (learned+mixed vs plain FP64)")
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-many", action="store_true",
                    help="skip the many-network workload (48 networks, n 12-18, 64 x 16 systems each)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default level-sweep tiling")
    ap.add_argument("--batch", type=int, default=BATCH, help="held-out rate sets per step (profiling of smaller cases)")
    ap.add_argument("--profile-run", action="store_true",
                    help="run --warmup steps and then exactly one step, nothing else (for ncu launch lists)")
    ap.add_argument("--profile-table", action="store_true",
                    help="build the CSC transition tables of the n=20 bench network and of the n=22 drop-in "
                         "network once each, nothing else (for ncu captures of the table kernels)")
    ap.add_argument("--profile-mlp", action="store_true",
                    help="run the warm-start inference (untrained weights) of the n=20 bench network on 64 rate "
                         "sets twice, nothing else (for ncu captures of the tensor-core kernel)")
    args = ap.parse_args()
    BATCH = args.batch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.profile_table:
        import torch

        import paraexastolog_b200 as esl
        ctx = esl.Context(local)
        net_g, rates, _, _, _ = workload(0, 1)
        scale = synth.config_scale()
        for text, r in ((net_g.bnet, rates[0]), (scale.networks[0].bnet, scale.rates[0][0])):
            esl.table(ctx, esl.Model.parse(text), r, with_cols=False)
        torch.cuda.synchronize()
        return

    if args.profile_mlp:
        import torch

        import paraexastolog_b200 as esl
        ctx = esl.Context(local)
        net_g, rates, _, _, _ = workload(0, 1)
        net = esl.Net.build(ctx, esl.Model.parse(net_g.bnet), rates[0])
        mlp = esl.Mlp(ctx, net, seed=3)
        mlp.set_params(mlp.get_params(), 0.0, 1.0)
        d_rates = torch.tensor(rates[:64], device=f"cuda:{local}")
        for _ in range(2):
            mlp.predict(d_rates)
        torch.cuda.synchronize()
        return

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)))
        return

    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    out, xinf = run_ours(args, rank, world, local)
    if args.profile_run:
        return
    if not args.no_cpu_baseline:
        # error of this run's results against the FP64 oracle on a sample of every rank's
        # rate sets; at N=1 the same oracle run is the timed CPU baseline
        if world == 1:
            sample = max(8, min(os.cpu_count() or 8, 16))
            cb, _, ref = cpu_baseline(sample)
        else:
            sample = 2
            cb, _, ref = cpu_baseline(sample, rank, world, threads=max(1, (os.cpu_count() or 2) // world))
        got = xinf[:sample, 0].cpu().numpy()
        diff = np.abs(got - ref.reshape(sample, -1))
        other = out.pop("_other_xinf", None) if out is not None else None
        odiff = np.abs(other[:sample, 0].cpu().numpy() - ref.reshape(sample, -1)) if other is not None else None
        l1, mx, ol1, omx = shards.max_over_ranks(
            [diff.sum(1).max(), diff.max(), odiff.sum(1).max() if odiff is not None else -1.0,
             odiff.max() if odiff is not None else -1.0], world, device=f"cuda:{local}")
        if rank == 0:
            if world == 1:
                out["cpu_baseline"] = cb
            out["accuracy_vs_fp64_oracle"] = {"rate_sets": sample * world, "l1_max": l1, "maxabs": mx,
                                              "target_l1": 1e-9, "ranks": world}
            for key in ("learned_mixed", "plain_fp64"):
                if key in out and ol1 >= 0.0:
                    out[key]["accuracy_vs_fp64_oracle"] = {"rate_sets": sample * world, "l1_max": ol1,
                                                           "maxabs": omx, "target_l1": 1e-9}
    if out is not None:
        out.pop("_other_xinf", None)
    if world == 1 and not args.no_many and out is not None:
        # the many-network workload, after the headline (outside its timed steps)
        del xinf
        many, w, mres = many_networks(local)
        if not args.no_cpu_baseline:
            many["cpu_baseline"], many["accuracy_vs_fp64_oracle"] = cpu_baseline_many(w, mres)
        del mres
        out["many_networks"] = many
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
