#!/usr/bin/env python
"""Benchmark of the FINFLO per-iteration hot path on B200.

One step = one full single-grid iteration of the reference's CYCLES on one
block (STATIM/BOUNDI, RESIDU + RESL2, IMPS with LU-SGS, FIN + limits, SUBIN).
Metric: cell-iters/s = interior cells x completed cycles / seconds (device
time from CUDA events on the library's stream, max over ranks).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs as N independent replicas (one block per GPU, no data-path
collective; the batched multi-block exchange is a separate path), reported as
weak scaling.  The reference arm times the CPU restatement of the reference
routines (the Fortran reference has no compiler here) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(ni=65, nj=33, nk=33)   # node counts -> 64 x 32 x 32 cells
WORKLOAD_NAME = ("bump channel 64x32x32 cells, laminar Re=1e4 M=0.5, Roe+MUSCL(INTER=3), "
                 "full NS, LU-SGS, single grid, FP64")


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        self.path = os.path.join("/tmp", f"ff_clocks_{os.getpid()}.csv")
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 6 and parts[0].isdigit():
                rows.append(parts)
        if not rows:
            return None
        sm = [int(r[0]) for r in rows]
        reasons = set()
        for r in rows:
            for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), r[2:6]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][1]), "reasons": sorted(reasons)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _allreduce_max(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_oracle_rate(seconds=15.0, wl=WORKLOAD, procs=1):
    """Cell-iters/s of the CPU oracle on the bench workload (bounded sample)."""
    from finflo_b200 import case
    from oracle.oracle import Oracle
    blk, prm, fs = case.bump_case(wl["ni"], wl["nj"], wl["nk"])
    o = Oracle(blk, prm)
    o.start()
    o.cycle(1)
    n = 0
    t0 = time.perf_counter()
    while True:
        o.cycle(n + 2)
        n += 1
        el = time.perf_counter() - t0
        if el > seconds:
            break
    return blk.interior_cells * n / el, n


def _cpu_worker(args):
    seconds, wl = args
    sys.path.insert(0, ROOT)
    r, n = cpu_oracle_rate(seconds, wl)
    return r, n


def cpu_all_cores(seconds=15.0, wl=WORKLOAD):
    import multiprocessing as mp
    ncores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(ncores) as pool:
        res = pool.map(_cpu_worker, [(seconds, wl)] * ncores)
    return sum(r for r, _ in res), ncores, sum(n for _, n in res)


def run_reference(args):
    ws, rank, local = _dist()
    if rank != 0:
        return 0
    seconds = max(5.0, min(20.0, 2.0 * args.steps))
    rate, cores, ncyc = cpu_all_cores(seconds)
    line = {
        "metric": "cell-iters/s", "value": rate, "unit": "cell-iters/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded bump-channel grid and noisy free stream)",
        "config": {"workload": WORKLOAD_NAME, "parallelism": f"{cores} host processes (replicas)"},
        "impl": "reference",
        "cpu_baseline": {"value": rate, "unit": "cell-iters/s", "cores": cores, "kind": "port",
                         "sample": f"{ncyc} cycles total over {cores} replica processes, ~{seconds:.0f}s each"},
        "e2e": {"value": rate, "unit": "cell-iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_ours(args):
    ws, rank, local = _dist()
    if ws > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    from finflo_b200 import case
    from finflo_b200.gpu import GpuSolver, FF_STAGE_RESIDUAL
    wl = dict(WORKLOAD)
    if args.grid:
        wl["ni"], wl["nj"], wl["nk"] = (int(x) for x in args.grid.split(","))
    blk, prm, fs = case.bump_case(wl["ni"], wl["nj"], wl["nk"])
    g = GpuSolver(local)
    bid = g.add_block(blk, prm)
    g.upload(bid)
    g.start(bid)
    g.cycles(1 + args.warmup, bid, icycle0=1)   # warm-up incl. graph capture
    g.sync()
    ncell = blk.interior_cells
    # ---- device-timed cycles -------------------------------------------
    clk = ClockSampler(local)
    _barrier(ws)
    clk.start()
    ms = g.time_cycles(args.steps, bid)
    clocks = clk.stop()
    _barrier(ws)
    ms = _allreduce_max(ms, ws)
    value = ncell * args.steps * ws / (ms * 1e-3)
    # ---- dominant kernel: the fused residual ---------------------------
    ms_res = g.time_stage(FF_STAGE_RESIDUAL, reps=20, bid=bid)
    bytes_per_cell = 288.0   # algorithmic bytes of the laminar FP64 residual
    achieved = bytes_per_cell * ncell / (ms_res * 1e-3) / 1e9
    peak, kind = _peaks()
    launches = g.cycle_launches(bid) * args.steps
    lk = g.lusgs_kind(bid)
    sweep = dict(g.sweep_tuning(bid), chosen="cluster lines" if lk % 100 == 1 else "cooperative hyperplane")
    # ---- end to end through the C-ABI with host buffers ----------------
    names_in = ["TEMP", "U", "V", "W", "PDIFF"]
    host = {n: blk.arrays[n] for n in names_in}
    h2d = d2h = 0
    t0 = time.perf_counter()
    for s in range(0 if args.no_e2e else args.steps):
        g.upload(bid, names_in)
        h2d += 8 * blk.ntot * len(names_in)
        hist = g.cycles(1, bid, icycle0=2)
        g.download(bid, names_in, into=host)
        d2h += 8 * blk.ntot * len(names_in) + hist.nbytes
    g.sync()
    e2e_s = time.perf_counter() - t0
    e2e_s = _allreduce_max(e2e_s, ws)
    e2e = ncell * args.steps * ws / e2e_s if not args.no_e2e else None
    line = {
        "metric": "cell-iters/s", "value": value, "unit": "cell-iters/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded bump-channel grid and noisy free stream)",
        "config": {"workload": WORKLOAD_NAME if not args.grid else f"bump channel {blk.imax}x{blk.jmax}x{blk.kmax} cells (profiling size)",
                   "cells_per_gpu": ncell, "parallelism": f"replicas x{ws}",
                   "l2": "working set < L2 (cycle state resident)", "lusgs_sweep": sweep},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": "k_residual", "achieved": achieved, "peak": peak,
                     "peak_kind": kind, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                     "ms_per_launch": ms_res, "bytes_per_cell": bytes_per_cell},
        "e2e": {"value": e2e, "unit": "cell-iters/s", "h2d_bytes_per_step": h2d // max(1, args.steps),
                "d2h_bytes_per_step": d2h // max(1, args.steps)},
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu and not args.grid:
        rate, ncyc = cpu_oracle_rate(seconds=min(15.0, max(3.0, args.cpu_seconds)))
        line["cpu_baseline"] = {"value": rate, "unit": "cell-iters/s", "cores": 1, "kind": "port",
                                "sample": f"{ncyc} oracle cycles on the same 64x32x32 workload"}
    if rank == 0:
        print(json.dumps(line))
    g.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


BOX_NAME = ("periodic box, 24 blocks (4x3x2, seeded uneven 1:1 cuts, ~5.9M cells), inviscid M=0.3 "
            "entropy wave, FP64 residual + FP32 LU-SGS, device CONNEC, graph-captured multi-block cycle")


def run_box(args):
    """The batched multi-block workload: every block's chain of stages as
    concurrent branches of one captured cycle, the 1:1 exchange on device;
    with N > 1 the blocks are spread over the GPUs (strong scaling) and the
    halos move by NCCL send/recv once per cycle."""
    ws, rank, local = _dist()
    import torch
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    from finflo_b200 import case
    from finflo_b200 import dist as fd
    from finflo_b200.gpu import FF_STAGE_RESIDUAL
    nb = tuple(int(x) for x in args.blocks.split(","))
    blocks, prms, fs = case.periodic_box_case(nb=nb, lusgs_fp32=True)
    total = sum(b.interior_cells for b in blocks)
    backend = fd.GpuBackend(local)
    if ws > 1:
        db = fd.DistributedBlocks(blocks, prms, backend)
        db.start()
        mine = [blocks[g] for g in db.plan.local]
        db.cycles(1 + args.warmup)
        g = backend.solver
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.ExternalStream(g.stream_handle(), device=backend.device)
        clk = ClockSampler(local)
        _barrier(ws)
        clk.start()
        ev0.record(stream)
        for i in range(args.steps):
            g.mb_phase(fd.PHASE_CYCLE_A, 2 + args.warmup + i, True)
            db.exchange()
            g.mb_phase(fd.PHASE_B, 2 + args.warmup + i, True)
            g.mb_phase(fd.PHASE_RECORD, 2 + args.warmup + i, True)
        ev1.record(stream)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1)
        clocks = clk.stop()
        launches = None
    else:
        g = backend.solver
        for b, p in zip(blocks, prms):
            bid = g.add_block(b, p)
            g.upload(bid)
        mine = blocks
        g.start_all()
        g.cycles_all(1 + args.warmup, icycle0=1)
        g.sync()
        clk = ClockSampler(local)
        clk.start()
        ms, per_cycle = g.time_cycles_all(args.steps)
        clocks = clk.stop()
        launches = per_cycle * args.steps
    _barrier(ws)
    ms = _allreduce_max(ms, ws)
    value = total * args.steps / (ms * 1e-3)
    # residual stage of every local block, timed one by one
    ms_res = sum(g.time_stage(FF_STAGE_RESIDUAL, reps=5, bid=i) for i in range(len(mine)))
    cells_mine = sum(b.interior_cells for b in mine)
    bytes_per_cell = 216.0   # inviscid residual: 9 state + 13 metric reads, 5 writes (FP64)
    achieved = bytes_per_cell * cells_mine / (ms_res * 1e-3) / 1e9
    peak, kind = _peaks()
    line = {
        "metric": "cell-iters/s", "value": value, "unit": "cell-iters/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "strong" if ws > 1 else "weak", "vs_baseline": None,
        "dtype": "f64 residual / f32 LU-SGS", "data": "synthetic (seeded block split and entropy-wave phase)",
        "config": {"workload": BOX_NAME, "blocks": len(blocks), "cells": total,
                   "parallelism": f"blocks over {ws} GPU(s)", "l2": "inputs larger than L2"},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": "k_residual (all blocks)", "achieved": achieved, "peak": peak,
                     "peak_kind": kind, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                     "ms_per_launch": ms_res / max(1, len(mine)), "bytes_per_cell": bytes_per_cell},
        "e2e": None,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line))
    backend.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--grid", default="", help="node counts ni,nj,nk (profiling runs)")
    ap.add_argument("--workload", default="bump", choices=["bump", "box"])
    ap.add_argument("--blocks", default="4,3,2", help="block arrangement of the box workload")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "box":
        return run_box(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
