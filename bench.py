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
on the plain solves' occupations of the 3,584 training rate sets.

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

from paraexastolog_b200 import synth  # noqa: E402

METRIC = "solves/s, n=20 x 512 rate sets, learned+mixed vs FP64 sparse LU at L1<=1e-9"
BATCH = 512


N_TRAIN = 3584


def workload(rank: int):
    """(network, held-out rate sets of this rank, x0, training rate sets)."""
    w = synth.config_learned(n_rate_sets=4096)
    net = w.networks[0]
    rates = w.rates[0][-BATCH:]
    if rank > 0:  # weak scaling: further seeded rate sets of the same distribution
        rng = np.random.default_rng(10_000 + rank)
        rates = synth.log_uniform_rates(rng, net.n, BATCH)
    return (net, np.ascontiguousarray(rates), np.ascontiguousarray(w.x0[0]),
            np.ascontiguousarray(w.rates[0][:N_TRAIN]))


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


def traffic_per_byte():
    """DRAM bytes per algorithmic byte of the Schur operator from the committed ncu
    capture summary (profiles/schur_operator_traffic.json), or None."""
    path = os.path.join(REPO, "profiles", "schur_operator_traffic.json")
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
    net_g, rates, x0, train_rates = workload(rank)
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
    other = None
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
        other = {"method": o_name, "value": BATCH * args.steps * world / (oms * 1e-3),
                 "ms_per_step": oms / args.steps, "iterations": ores.report.iterations,
                 "relres": ores.report.relres}
        if mlp is not None:
            # iterations of the mixed solve without the warm start, and the inference time alone
            cres = esl.solve_batch(ctx, net, d_rates, d_x0, method=esl.METHOD_MIXED, tol=args.tol)
            other["mixed_without_warm_start_iterations"] = cres.report.iterations
            _, pms, _, _ = timed(lambda: mlp.predict(d_rates, out=warm_buf), 3)
            other["warm_start_inference_ms"] = pms / 3
            other["warm_start_training"] = train_info

    # roofline of the dominant kernel pair (Schur operator) from live CUDA events
    ctx.set_profiling(True)
    for _ in range(max(1, min(args.steps, 2))):
        step()
    op_ms, op_bytes, op_launches = ctx.profile()
    rec_ms, rec_bytes = ctx.profile_records()
    ctx.set_profiling(False)
    # the applications of the largest level group (the one that dominates the step)
    big = rec_bytes >= 0.5 * rec_bytes.max() if rec_bytes.size else rec_bytes.astype(bool)
    big_ms, big_bytes, big_n = float(rec_ms[big].sum()), float(rec_bytes[big].sum()), int(big.sum())

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

    t = torch.tensor([ms, e2e_ms, float(launches)], device=f"cuda:{device}")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, e2e_ms = float(t[0]), float(t[1])
    out = None
    if rank == 0:
        solves = BATCH * args.steps * world
        peak, peak_kind = peaks()
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
                       "step": ("table + SCC/levels/order + terminal kernels + " +
                                ("warm-start inference + " if learned else "") +
                                "transient solve + x_inf/marginals")},
            "e2e": {"value": solves / (e2e_ms * 1e-3), "unit": "solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "wall_s": e2e_wall},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm",
                         "kernel": "schur_operator (k_sw_elim + k_sw_apply) of the largest level group",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None,
                         "peak_kind": peak_kind,
                         "traffic": (big_bytes / big_n) * tpb if (tpb and big_n) else None,
                         "algorithmic_bytes_per_launch": big_bytes / big_n if big_n else None,
                         "launches": big_n,
                         "all_groups": {"achieved": achieved_all,
                                        "frac": achieved_all / peak if achieved_all else None,
                                        "launches": op_launches,
                                        "note": "first poll window of every Krylov group; small groups "
                                                "are launch-latency bound"}},
            "solver": {"iterations": iters, "relres": relres},
            "clocks": clocks,
        }
        if tuning:
            out["config"]["tiling"] = tuning
        if other:
            other["value_over_headline"] = other["value"] / value
            out["learned_mixed" if other["method"] == "learned+mixed" else "plain_fp64"] = other
    return out, last_xinf


def cpu_baseline(sample: int):
    """The CPU FP64 oracle on this host's cores over a bounded sample of rate sets;
    returns (baseline record, seconds, the oracle's x_inf of the sample)."""
    import oracle as O

    net_g, rates, x0, _ = workload(0)
    m = O.Model(text=net_g.bnet)
    sym = m.analyse(rates[0])
    threads = min(os.cpu_count() or 1, sample)
    r = rates[:sample]
    xs = np.broadcast_to(x0, (sample, x0.size)).copy()
    t = time.perf_counter()
    ref, _ = sym.solve_many(r, xs, threads=threads)
    dt = time.perf_counter() - t
    return {"value": sample / dt, "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"{sample} of the 512 held-out rate sets, oracle symbolic analysis excluded"}, dt, ref


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
    ap.add_argument("--no-autotune", action="store_true", help="keep the default level-sweep tiling")
    ap.add_argument("--batch", type=int, default=BATCH, help="held-out rate sets per step (profiling of smaller cases)")
    ap.add_argument("--profile-run", action="store_true",
                    help="run --warmup steps and then exactly one step, nothing else (for ncu launch lists)")
    args = ap.parse_args()
    BATCH = args.batch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

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
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:
            sample = max(8, min(os.cpu_count() or 8, 16))
            out["cpu_baseline"], _, ref = cpu_baseline(sample)
            # error of this run's results against the FP64 oracle on the sampled rate sets
            got = xinf[:sample, 0].cpu().numpy()
            diff = np.abs(got - ref.reshape(sample, -1))
            out["accuracy_vs_fp64_oracle"] = {"rate_sets": sample, "l1_max": float(diff.sum(1).max()),
                                              "maxabs": float(diff.max()), "target_l1": 1e-9}
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
