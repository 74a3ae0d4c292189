#!/usr/bin/env python
"""Benchmark: time to optimal of the B200 dual simplex, learned vs plain pricing.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload learned|plain_small|plain_large] [--pricing learned|dse]

One step = --concurrency (8) complete solves (phase 1 + phase 2 to an optimal
status) of seeded LPs from the workload's distribution (default: m=2000,
n=4000, 1% N(0,1) entries, b = A x0 + U[0.1,1], c ~ U[0,1]; seeds 2000+, never
used in training), one host thread and CUDA stream per LP.  Each rank solves
its own seeds (independent LPs: replicas, weak scaling, no collective).
`value` is LPs solved to optimality per second: solved LPs / the max over
ranks of the summed per-step device time (CUDA events), every LP already
resident in HBM.  `time_to_optimal` times --tto-lps of the same LPs solved
alone on the GPU with the chosen pricing and with plain DSE pricing (same
seeds, objectives compared).  `e2e` is `value` measured through the public C
ABI from pinned host buffers (ds_load_typed -> ds_solve -> ds_get_primal /
ds_get_dual).  `--impl reference` solves the same LPs to optimality with the
CPU port of the reference's sequential dual simplex on the host cores.
Rank 0 prints one JSON line.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-optimal & iters/s: learned vs plain GPU dual simplex, obj rel-err ≤1e-9"
BATCH = {
    "batched": dict(count=4096, m_lo=32, m_hi=512, density=0.10, seed=7000),
    "batched_small": dict(count=65536, m_lo=16, m_hi=64, density=0.10, seed=9000),
}
WORKLOADS = {
    "batched": dict(desc="4096 LPs, m~U{32..512}, n=2m, density 10% N(0,1), A x <= b, x >= 0, seed+i"),
    "batched_small": dict(desc="65,536 LPs, m~U{16..64}, n=2m, density 10% N(0,1), A x <= b, x >= 0, seed+i"),
    "learned": dict(desc="LP m=2000 n=4000 density 1% N(0,1), A x <= b, x >= 0", m=2000, n=4000),
    "plain_small": dict(desc="LP m=200 n=400 density 5% N(0,1), A x <= b, x >= 0", m=200, n=400),
    "plain_large": dict(desc="LP m=50000 n=100000 8 nnz/col N(0,1), A x <= b, x >= 0", m=50000, n=100000),
}


def gen(workload, seed):
    from parallel_ds_b200 import lp as L
    return {"learned": L.learned, "plain_small": L.plain_small, "plain_large": L.plain_large}[workload](seed)


def lp_bytes(t):
    return sum(int(t[k].nbytes) for k in ("row_ptr", "col_idx", "val", "c", "col_type", "col_lb", "col_ub",
                                          "row_type", "row_lb", "row_ub"))


class Clocks(threading.Thread):
    """nvidia-smi sampling during the timed region (SM clock, throttle reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        super().__init__(daemon=True)
        self.dev, self.rows, self.stop_ev, self.proc = dev, [], threading.Event(), None

    def run(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            for line in self.proc.stdout:
                self.rows.append([x.strip() for x in line.split(",")])
                if self.stop_ev.is_set():
                    break
        except Exception:
            pass

    def stop(self):
        self.stop_ev.set()
        if self.proc:
            self.proc.terminate()
        self.join(timeout=3)
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


def pinned_copy(t):
    """The typed LP's arrays in page-locked host memory (torch allocator)."""
    import numpy as np
    import torch
    out = {}
    for k, v in t.items():
        if isinstance(v, np.ndarray):
            buf = torch.empty(v.shape, dtype=torch.from_numpy(v[:0].copy()).dtype, pin_memory=True)
            buf.numpy()[...] = v
            out[k] = buf.numpy()
        else:
            out[k] = v
    return out


def our_arm(args, rank, world, local_rank):
    import numpy as np
    import torch
    from concurrent.futures import ThreadPoolExecutor
    from parallel_ds_b200 import _lib
    from parallel_ds_b200 import learned as LN
    from parallel_ds_b200 import lp as L
    from parallel_ds_b200._lib import DsOptions, DsStats, ptr

    torch.cuda.set_device(local_rank)
    lib = _lib.lib()
    Cc = args.concurrency
    learned = args.pricing == "learned"

    def options(pricing_learned):
        o = DsOptions()
        lib.ds_default_options(C.byref(o))
        o.device = local_rank
        o.pricing = _lib.PRICING_LEARNED if pricing_learned else _lib.PRICING_DSE
        return o

    model = C.c_void_p()
    if learned:
        with np.load(args.weights) as f:
            params = np.ascontiguousarray(f["params"], dtype=np.float32)
        assert lib.ds_model_create(local_rank, C.byref(model)) == 0
        assert lib.ds_model_set_params(model, ptr(params, C.c_float), len(params)) == 0

    def new_handle(pricing_learned=learned):
        h = C.c_void_p()
        o = options(pricing_learned)
        assert lib.ds_create(C.byref(o), C.byref(h)) == 0
        if pricing_learned:
            assert lib.ds_set_model(h, model) == 0
        return h

    def load(h, t):
        rc = lib.ds_load_typed(h, t["m"], t["n"], ptr(t["row_ptr"], C.c_int), ptr(t["col_idx"], C.c_int),
                               ptr(t["val"], C.c_double), ptr(t["c"], C.c_double), ptr(t["col_type"], C.c_int),
                               ptr(t["col_lb"], C.c_double), ptr(t["col_ub"], C.c_double),
                               ptr(t["row_type"], C.c_int), ptr(t["row_lb"], C.c_double),
                               ptr(t["row_ub"], C.c_double))
        assert rc == 0, lib.ds_last_error(h)

    def stats(h):
        s = DsStats()
        lib.ds_get_stats(h, C.byref(s))
        return s

    def solve(h):
        rc = lib.ds_solve(h)
        assert rc == 0, lib.ds_last_error(h)
        return h

    K, W = args.steps, args.warmup
    seeds = [[2000 + (rank * K + s) * Cc + c for c in range(Cc)] for s in range(K)]
    wseeds = [[1000 + (rank * W + s) * Cc + c for c in range(Cc)] for s in range(W)]
    lps = [[pinned_copy(L.typed(gen(args.workload, x))) for x in row] for row in seeds]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > L2
    pool = ThreadPoolExecutor(max_workers=Cc)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # warm-up (untimed): same handles and concurrency as the timed steps, and one plain solve
    handles = [new_handle() for _ in range(Cc)]
    for row in wseeds:
        ts = [L.typed(gen(args.workload, x)) for x in row]
        for h, t in zip(handles, ts):
            load(h, t)
        list(pool.map(solve, handles))
    hp = new_handle(False)
    load(hp, L.typed(gen(args.workload, 999)))
    solve(hp)

    # ---- time to optimal, one LP alone on the GPU: learned vs plain on the same seeds
    tto = []
    h1 = new_handle()
    tto_seeds = [3000 + rank * args.tto_lps + i for i in range(args.tto_lps)]
    for x in tto_seeds:
        t = L.typed(gen(args.workload, x))
        load(h1, t); solve(h1)
        a = dict(ms=stats(h1).solve_ms, it=stats(h1).iterations, obj=lib.ds_get_objective(h1),
                 st=_status(lib.ds_get_status(h1)), pdhg_ms=stats(h1).pdhg_ms)
        load(hp, t); solve(hp)
        b = dict(ms=stats(hp).solve_ms, it=stats(hp).iterations, obj=lib.ds_get_objective(hp),
                 st=_status(lib.ds_get_status(hp)))
        tto.append((a, b))
    roof = profile_roofline(lib, h1)
    lib.ds_destroy(h1)
    tto_block = None
    if tto:
        ta, tb = sum(a["ms"] for a, _ in tto), sum(b["ms"] for _, b in tto)
        ia, ib = sum(a["it"] for a, _ in tto), sum(b["it"] for _, b in tto)
        ratios = sorted(b["ms"] / a["ms"] for a, b in tto)
        # short on purpose: the whole JSON line must stay readable in a log tail
        tto_block = {
            "speedup_vs_plain": round(tb / ta, 4), "mean_ms": round(ta / len(tto), 3),
            "plain_mean_ms": round(tb / len(tto), 3), "lps": len(tto), "pricing": args.pricing,
            "iters_per_s": round(ia / (ta / 1e3), 1), "plain_iters_per_s": round(ib / (tb / 1e3), 1),
            "mean_iterations": round(ia / len(tto), 1), "plain_mean_iterations": round(ib / len(tto), 1),
            "per_lp_speedup_min_median_max": [round(ratios[0], 3), round(ratios[len(ratios) // 2], 3),
                                              round(ratios[-1], 3)],
            "mean_pdhg_ms": round(sum(a.get("pdhg_ms", 0.0) for a, _ in tto) / len(tto), 3),
            "max_obj_rel_err_vs_plain": max(abs(a["obj"] - b["obj"]) / max(1.0, abs(b["obj"])) for a, b in tto),
            "statuses": sorted({a["st"] for a, _ in tto} | {b["st"] for _, b in tto}),
            "seeds": f"{tto_seeds[0]}..{tto_seeds[-1]}",
        }

    # ---- value: LPs resident in HBM, K steps of Cc concurrent solves
    step_handles = []
    for row in lps:
        hs = [new_handle() for _ in row]
        for h, t in zip(hs, row):
            load(h, t)
        step_handles.append(hs)
    torch.cuda.synchronize()
    clk = Clocks(local_rank) if rank == 0 else None
    if clk:
        clk.start(); time.sleep(0.6)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    barrier(); torch.cuda.synchronize()
    launches0 = lib.ds_kernel_launch_count()
    for s, hs in enumerate(step_handles):
        flush.fill_(float(s))                 # evict the previous step's working set from L2
        ev[s][0].record()
        list(pool.map(solve, hs))
        ev[s][1].record()
    torch.cuda.synchronize(); barrier()
    launches = lib.ds_kernel_launch_count() - launches0
    clocks = clk.stop() if clk else None
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t_ms = sum(step_ms)
    allh = [h for hs in step_handles for h in hs]
    iters = sum(stats(h).iterations for h in allh)
    statuses = [lib.ds_get_status(h) for h in allh]
    lp_ms = [stats(h).solve_ms for h in allh]
    n_solved = sum(1 for x in statuses if x == 1)

    # ---- e2e: public API from pinned host buffers, H2D + D2H inside the timed region
    h2d = sum(lp_bytes(t) for row in lps for t in row) // (K * Cc) * Cc
    d2h = (8 * (lps[0][0]["n"] + lps[0][0]["m"]) + 8 * lps[0][0]["m"]) * Cc
    outs = [(np.zeros(lps[0][0]["n"]), np.zeros(lps[0][0]["m"])) for _ in range(Cc)]

    def e2e_one(args_):
        h, t, (x, y) = args_
        load(h, t)
        solve(h)
        lib.ds_get_primal(h, ptr(x, C.c_double), None)
        lib.ds_get_dual(h, ptr(y, C.c_double))
        return 1 if lib.ds_get_status(h) == 1 else 0

    barrier(); torch.cuda.synchronize()
    ee = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    e0 = time.perf_counter()
    ee[0].record()
    e_solved = 0
    for row in lps:
        e_solved += sum(pool.map(e2e_one, zip(handles, row, outs)))
    ee[1].record()
    torch.cuda.synchronize(); barrier()
    e_wall_ms = (time.perf_counter() - e0) * 1e3
    e_ms = max(ee[0].elapsed_time(ee[1]), e_wall_ms)
    for h in allh + handles + [hp]:
        lib.ds_destroy(h)
    if learned:
        lib.ds_model_destroy(model)
    pool.shutdown()

    if world > 1:
        tt = torch.tensor([t_ms, e_ms], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        it = torch.tensor([iters, n_solved, e_solved], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(it, op=torch.distributed.ReduceOp.SUM)
        t_ms, e_ms = [float(v) for v in tt.tolist()]
        iters, n_solved, e_solved = [int(v) for v in it.tolist()]
    if rank != 0:
        return None
    res = {
        "metric": METRIC,
        "value": n_solved / (t_ms / 1e3),
        "unit": "LPs/s",
        "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": t_ms / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: seeded generator, N(0,1) entries, x0~U[0,1], b=A x0+U[0.1,1], c~U[0,1]",
        "config": {"workload": WORKLOADS[args.workload]["desc"], "pricing": args.pricing,
                   "scorer": os.path.relpath(args.weights, ROOT) if learned else None,
                   "lps_per_step": Cc, "seeds_rank0": f"{seeds[0][0]}..{seeds[-1][-1]}", "refactor_interval": 100,
                   "parallelism": f"replicas x{world}, {Cc} concurrent solves per GPU",
                   "l2": "256 MB buffer written between steps (flush); each step solves its LPs to optimality",
                   "step": f"{Cc} complete solves to optimality (status optimal), one host thread and CUDA "
                           f"stream each"},
        "iters_per_s": iters / (t_ms / 1e3),
        "iterations": iters,
        "time_to_optimal": tto_block,
        "lp_time_to_optimal_ms": {"mean": round(statistics.mean(lp_ms), 3), "max": round(max(lp_ms), 3)},
        "statuses": sorted({_status(x) for x in statuses}),
        "e2e": {"value": e_solved / (e_ms / 1e3), "unit": "LPs/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e_ms / K},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if roof:
        res["roofline"] = roof
    return res


def large_arm(args, rank, world, local_rank):
    """The large eta-file workload (m=50,000, n=100,000, 8 nonzeros per column):
    one step = the first --large-iters iterations of a plain DSE solve of one
    seeded LP from its slack basis (refactorisations every 100 iterations by
    the sparse LU included), LP resident in HBM.  Metric: iterations/s."""
    import numpy as np
    import torch
    from parallel_ds_b200 import _lib
    from parallel_ds_b200 import lp as L
    from parallel_ds_b200._lib import DsOptions, DsStats, ptr

    torch.cuda.set_device(local_rank)
    lib = _lib.lib()
    cap = args.large_iters

    def new_handle():
        h = C.c_void_p()
        o = DsOptions()
        lib.ds_default_options(C.byref(o))
        o.device = local_rank
        o.max_iterations = cap
        assert lib.ds_create(C.byref(o), C.byref(h)) == 0
        return h

    def load(h, t):
        rc = lib.ds_load_typed(h, t["m"], t["n"], ptr(t["row_ptr"], C.c_int), ptr(t["col_idx"], C.c_int),
                               ptr(t["val"], C.c_double), ptr(t["c"], C.c_double), ptr(t["col_type"], C.c_int),
                               ptr(t["col_lb"], C.c_double), ptr(t["col_ub"], C.c_double),
                               ptr(t["row_type"], C.c_int), ptr(t["row_lb"], C.c_double),
                               ptr(t["row_ub"], C.c_double))
        assert rc == 0, lib.ds_last_error(h)

    def stats(h):
        st = DsStats()
        lib.ds_get_stats(h, C.byref(st))
        return st

    K, W = args.steps, args.warmup
    seeds = [2000 + rank * K + s for s in range(K)]
    lps = [pinned_copy(L.typed(gen(args.workload, x))) for x in seeds]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    hw = new_handle()
    for s in range(W):
        load(hw, L.typed(gen(args.workload, 1000 + rank * W + s)))
        assert lib.ds_solve(hw) == 0, lib.ds_last_error(hw)
    hs = [new_handle() for _ in lps]
    for h, t in zip(hs, lps):
        load(h, t)
    torch.cuda.synchronize()
    clk = Clocks(local_rank) if rank == 0 else None
    if clk:
        clk.start(); time.sleep(0.6)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = lib.ds_kernel_launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    for s, h in enumerate(hs):
        flush.fill_(float(s))
        ev[s][0].record()
        assert lib.ds_solve(h) == 0, lib.ds_last_error(h)
        ev[s][1].record()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    launches = lib.ds_kernel_launch_count() - launches0
    clocks = clk.stop() if clk else None
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    iters = sum(stats(h).iterations for h in hs)
    refac_ms = sum(stats(h).refactor_ms for h in hs)
    st0 = stats(hs[0])
    # e2e: load from pinned host buffers, solve, read x and y back
    x, y = np.zeros(lps[0]["n"]), np.zeros(lps[0]["m"])
    torch.cuda.synchronize()
    e0 = time.perf_counter()
    e_it = 0
    for t in lps:
        load(hw, t)
        assert lib.ds_solve(hw) == 0, lib.ds_last_error(hw)
        lib.ds_get_primal(hw, ptr(x, C.c_double), None)
        lib.ds_get_dual(hw, ptr(y, C.c_double))
        e_it += stats(hw).iterations
    torch.cuda.synchronize()
    e_ms = (time.perf_counter() - e0) * 1e3
    roof = profile_roofline(lib, hs[0])
    for h in hs + [hw]:
        lib.ds_destroy(h)
    if world > 1:
        tt = torch.tensor([t_ms, e_ms], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        it = torch.tensor([iters, e_it], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(it, op=torch.distributed.ReduceOp.SUM)
        t_ms, e_ms = [float(v) for v in tt.tolist()]
        iters, e_it = [int(v) for v in it.tolist()]
    if rank != 0:
        return None
    res = {
        "metric": "iterations/s of the plain GPU dual simplex (eta file + sparse LU), first %d iterations" % cap,
        "value": iters / (t_ms / 1e3), "unit": "iterations/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": t_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded generator, 8 N(0,1) entries per column at uniform random rows",
        "config": {"workload": WORKLOADS[args.workload]["desc"], "pricing": "dse", "iterations_per_step": cap,
                   "refactor_interval": 100, "seeds_rank0": f"{seeds[0]}..{seeds[-1]}",
                   "l2": "256 MB buffer written between steps (flush)",
                   "step": f"one LP, its first {cap} iterations from the slack basis"},
        "refactor_ms_per_step": refac_ms / K,
        "last_factor": {"bump": st0.bump_size, "kernel": st0.lu_kernel, "dense_block": st0.lu_dense,
                        "levels_ftran_btran": st0.lu_levels, "markowitz_rounds": st0.lu_rounds},
        "e2e": {"value": e_it / (e_ms / 1e3), "unit": "iterations/s",
                "h2d_bytes_per_step": int(lp_bytes(lps[0])),
                "d2h_bytes_per_step": int(8 * (lps[0]["n"] + lps[0]["m"])), "ms_per_step": e_ms / K},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if roof:
        res["roofline"] = roof
    return res


def large_cpu_sample(workload, iters=300):
    """The oracle running the first `iters` iterations of the same LP on one core."""
    from oracle import pyoracle as po
    from parallel_ds_b200 import lp as L
    t = L.typed(gen(workload, 2000))
    t0 = time.perf_counter()
    r = po.solve_typed(t, max_iterations=iters)
    dt = time.perf_counter() - t0
    return {"value": r["iterations"] / dt, "unit": "iterations/s", "cores": 1, "kind": "port",
            "sample": f"oracle runs the first {r['iterations']} iterations of seed 2000 ({r['status']}), {dt:.1f} s"}


def batch_arm(args, rank, world, local_rank):
    """Batched workloads: one step = one persistent launch solving the whole
    batch (`count` LPs per GPU, weak scaling: rank r solves seeds
    seed + r*count + i)."""
    import numpy as np
    import torch
    from parallel_ds_b200 import _lib
    from parallel_ds_b200.batch import BatchSolver, gen_arrays, rank_seed

    torch.cuda.set_device(local_rank)
    lib = _lib.lib()
    cfg = BATCH[args.workload]
    count = args.batch_count or cfg["count"]
    seed = rank_seed(cfg["seed"], rank, count)

    def pinned(shape, dtype):
        return torch.empty(int(shape), dtype=torch.from_numpy(np.zeros(0, dtype)).dtype, pin_memory=True).numpy()

    arr = gen_arrays(count, cfg["m_lo"], cfg["m_hi"], cfg["density"], seed, alloc=pinned)
    bs = BatchSolver(local_rank)
    bs.load_arrays(arr)
    if not args.no_tune:
        bs.tune()                               # untimed: the autotuner picks the schedule
    for _ in range(args.warmup):
        bs.solve()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    clk = Clocks(local_rank) if rank == 0 else None
    if clk:
        clk.start(); time.sleep(0.6)
    barrier(); torch.cuda.synchronize()
    launches0 = lib.ds_kernel_launch_count()
    step_ms = []
    for s in range(args.steps):
        flush.fill_(float(s)); torch.cuda.synchronize()        # L2 flush between steps
        bs.solve()                                             # CUDA events on the batch's stream
        step_ms.append(bs.stats()["solve_ms"])
    torch.cuda.synchronize(); barrier()
    launches = lib.ds_kernel_launch_count() - launches0
    clocks = clk.stop() if clk else None
    st, obj, its = bs.results()
    solved = int((st == 1).sum())
    t_ms = sum(step_ms)
    # algorithmic bytes of the launch: per pivot 16 m^2 (B^-1 read + write), the
    # FTRAN's B^-1 columns (8 m per nonzero of a_q), the pivot row's CSC (12 nnz
    # + 4 n) and the O(m) vectors
    m = arr["m"].astype(np.float64); n = arr["n"].astype(np.float64)
    cpo = np.concatenate([[0], np.cumsum(arr["n"].astype(np.int64) + 1)])
    nnz = arr["col_ptr"][cpo[1:] - 1].astype(np.float64)
    per_it = 16 * m * m + 8 * m * (nnz / n) + 12 * nnz + 4 * n + 24 * m
    alg_bytes = float(np.sum(its * per_it))
    stats = bs.stats()

    # e2e: the public C ABI from pinned host buffers: load (H2D) + solve + results (D2H)
    h2d = sum(int(v.nbytes) for v in arr.values())
    d2h = count * (4 + 8 + 4)
    barrier(); torch.cuda.synchronize()
    e0 = time.perf_counter()
    e_solved = 0
    for _ in range(args.steps):
        bs.load_arrays(arr)
        bs.solve()
        st2, _, _ = bs.results()
        e_solved += int((st2 == 1).sum())
    e_ms = (time.perf_counter() - e0) * 1e3
    barrier()

    if world > 1:
        tt = torch.tensor([t_ms, e_ms], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        cn = torch.tensor([solved, e_solved, launches], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(cn, op=torch.distributed.ReduceOp.SUM)
        t_ms, e_ms = [float(v) for v in tt.tolist()]
        solved, e_solved, launches = [int(v) for v in cn.tolist()]
    if rank != 0:
        return None
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = alg_bytes / (stats["solve_ms"] * 1e-3) / 1e9
    return {
        "metric": METRIC, "value": solved * args.steps / (t_ms / 1e3), "unit": "LPs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded generator per instance (seed+i), N(0,1) entries, b=A x0+U[0.1,1], c~U[0,1]",
        "config": {"workload": WORKLOADS[args.workload]["desc"], "lps_per_gpu": count, "seed_rank0": cfg["seed"],
                   "schedule": stats["schedule"], "tune_ms": stats["tune_ms"],
                   "parallelism": f"replicas x{world} (each GPU its own {count} LPs), one persistent launch each",
                   "l2": "256 MB buffer written between steps; the batch (B^-1 slots + instances) exceeds L2",
                   "step": "one CUDA-graph replay of the persistent launch solving every LP of the batch"},
        "statuses": {_status(k): int(v) for k, v in zip(*np.unique(st, return_counts=True))},
        "iterations": {"mean": float(its.mean()), "max": int(its.max()), "total": int(its.sum())},
        "e2e": {"value": e_solved / (e_ms / 1e3), "unit": "LPs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e_ms / args.steps},
        "roofline": {"bound": "hbm", "kernel": "k_batch_solve", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": BATCH_TRAFFIC_PER_ALG_BYTE * alg_bytes,
                     "peak_source": "measured" if peaks else "fallback",
                     "algorithmic_bytes_per_launch": alg_bytes},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }


def batch_cpu_sample(workload, seconds=15.0, threads=1, max_lps=4096):
    """The oracle solving the batch's first instances (generated before the
    clock starts) on `threads` host threads until about `seconds` have passed."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import lpgen as G
    from oracle import pyoracle as po
    cfg = BATCH[workload]
    total = min(max_lps, cfg["count"])
    # instances from the oracle's restatement of the generator (bit-identical
    # to the library's), made in chunks outside the timed solves
    dt = 0.0
    done, statuses = 0, set()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        while dt < seconds and done < total:
            chunk = [G.typed(G.batched_instance(cfg["seed"], i, cfg["m_lo"], cfg["m_hi"], cfg["density"]))
                     for i in range(done, min(total, done + 4 * threads))]
            t0 = time.perf_counter()
            for r in ex.map(po.solve_typed, chunk):
                statuses.add(r["status"])
            dt += time.perf_counter() - t0
            done += len(chunk)
    return {"value": done / dt, "unit": "LPs/s", "cores": threads, "kind": "port",
            "sample": f"oracle solves the batch's first {done} instances ({sorted(statuses)}) on {threads} "
                      f"thread(s), {dt:.1f} s"}


def _status(code):
    from parallel_ds_b200._lib import STATUS
    return STATUS.get(code, str(code))


# DRAM bytes (read + write) per launch from one ncu capture of the kernel:
# profiles/dense_iteration_kernels_learned_m2000.md (k_binv_update, m=2000:
# B^-1 read from DRAM cold under ncu, its writes still in L2 at kernel end) and
# profiles/k_batch_solve_batched_256.md (151 GB DRAM for 211 GB algorithmic
# bytes on 256 LPs; applied to a full batch in that proportion).
NCU_TRAFFIC = {"k_binv_update": 32.062464e6}
BATCH_TRAFFIC_PER_ALG_BYTE = 151.0 / 211.0


def profile_roofline(lib, h):
    """Per-kernel device times measured by the engine's replay profiler."""
    import json as _j
    buf = C.create_string_buffer(1 << 16)
    if lib.ds_profile_solve(h, buf, len(buf)) != 0:
        return None
    prof = _j.loads(buf.value.decode())
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    top = max(prof["kernels"], key=lambda k: k["share"])
    achieved = top["bytes"] / (top["avg_us"] * 1e-6) / 1e9
    return {"bound": "hbm", "kernel": top["name"], "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": NCU_TRAFFIC.get(top["name"]),
            "peak_source": "measured" if peaks else "fallback",
            "kernels": {k["name"]: {"avg_us": round(k["avg_us"], 2), "gbs": round(k["gbs"], 1),
                                    "share": round(k["share"], 3)} for k in prof["kernels"]}}


def cpu_sample(workload):
    """The oracle (CPU port of the reference) solving one LP of the workload to
    optimality on one host core."""
    from oracle import pyoracle as po
    from parallel_ds_b200 import lp as L
    t = L.typed(gen(workload, 2000))
    t0 = time.perf_counter()
    r = po.solve_typed(t)
    dt = time.perf_counter() - t0
    return {"value": 1.0 / dt, "unit": "LPs/s", "cores": 1, "kind": "port",
            "sample": f"oracle solves seed 2000 to {r['status']} in {r['iterations']} iterations, {dt:.1f} s "
                      f"({r['iterations'] / dt:.0f} iterations/s)"}


def reference_arm(args):
    """The reference's CPU algorithm (the oracle port: sequential dual simplex
    with DSE pricing) solving the GPU arm's LPs to optimality, one LP per host
    thread on all host cores."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import lpgen as G
    from oracle import pyoracle as po
    cores = os.cpu_count() or 1
    K, W = args.steps, args.warmup
    per_step = max(1, min(args.concurrency, cores))
    # inputs from the oracle's restatement of the generator (bit-identical to
    # the GPU arm's), so this arm maps no product library
    ref_gen = {"learned": G.learned, "plain_small": G.plain_small,
               "plain_large": lambda sd: G.generate(1, 50000, 100000, per_col=8, seed=sd)}[args.workload]
    lps = [[G.typed(ref_gen(2000 + s * args.concurrency + c)) for c in range(per_step)]
           for s in range(K)]
    po.solve_typed(G.typed(G.plain_small(1000)))      # warm-up: load the library, fault in pages
    large = args.workload == "plain_large"
    # the large workload is timed like the GPU arm's line, over each LP's first
    # iterations (a bounded sample: 300, the CPU port's dense LU grows with the bump)
    cap = min(args.large_iters, 300) if large else None
    solve = (lambda t: po.solve_typed(t, max_iterations=cap)) if large else po.solve_typed
    rs = []
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=per_step) as ex:
        for row in lps:
            rs += list(ex.map(solve, row))
    dt = time.perf_counter() - t0
    if large:
        its = sum(r["iterations"] for r in rs)
        v = its / dt
        return {
            "metric": "iterations/s of the plain GPU dual simplex (eta file + sparse LU), first %d iterations"
                      % args.large_iters,
            "value": v, "unit": "iterations/s", "n_gpus": 0, "steps": K, "warmup": W, "ms_per_step": dt * 1e3 / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
            "data": "synthetic: the GPU arm's seeded LPs",
            "config": {"workload": WORKLOADS[args.workload]["desc"], "pricing": "dse",
                       "step": f"{per_step} LPs, their first {cap} iterations, one per host thread"},
            "cpu_baseline": {"value": v, "unit": "iterations/s", "cores": per_step, "kind": "port",
                             "sample": f"{len(rs)} LPs, first {cap} iterations each, {its} iterations, {dt:.1f} s"},
            "e2e": {"value": v, "unit": "iterations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "statuses": sorted({r["status"] for r in rs}),
        }
    solved = sum(1 for r in rs if r["status"] == "optimal")
    v = solved / dt
    return {
        "metric": METRIC, "value": v, "unit": "LPs/s", "n_gpus": 0, "steps": K, "warmup": W,
        "ms_per_step": dt * 1e3 / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "impl": "reference",
        "data": "synthetic: the GPU arm's seeded LPs",
        "config": {"workload": WORKLOADS[args.workload]["desc"], "pricing": "dse",
                   "step": f"{per_step} LPs solved to optimality, one per host thread"},
        "cpu_baseline": {"value": v, "unit": "LPs/s", "cores": per_step, "kind": "port",
                         "sample": f"{len(rs)} LPs (seeds of the GPU arm's steps) solved to optimality, "
                                   f"{sum(r['iterations'] for r in rs)} iterations, {dt:.1f} s"},
        "e2e": {"value": v, "unit": "LPs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "iters_per_s": sum(r["iterations"] for r in rs) / dt,
        "statuses": sorted({r["status"] for r in rs}),
    }


def solve_one(args):
    """One LP of the workload (seed --solve-one) solved alone, stats as JSON:
    the small, fixed command that profiler captures run."""
    import numpy as np
    from parallel_ds_b200 import learned as LN
    from parallel_ds_b200 import lp as L
    from parallel_ds_b200 import solver as S
    lp = gen(args.workload, args.solve_one)
    if args.pdhg_estimate:
        s = S.CudaDualSimplex(S.problem_from_lp(lp), pdhg_cluster=0 if args.no_pdhg_cluster else 1)
        s.initDualSimplex()
        x, y = s.pdhg_estimate(args.pdhg_estimate)
        print(json.dumps({"workload": args.workload, "seed": args.solve_one, "pdhg_iterations": args.pdhg_estimate,
                          "objective_estimate": float(np.dot(lp["c"], x))}))
        return
    model = LN.LeavingRowScorer.load(args.weights) if args.pricing == "learned" else None
    out = []
    for rep in range(args.repeat):
        kw = {"max_iterations": args.max_iterations} if args.max_iterations else {}
        s = S.CudaDualSimplex(S.problem_from_lp(lp), pricing=args.pricing, model=model, **kw)
        s.initDualSimplex()
        sol = s.solve()
        out.append(dict(status=s.status(), objective=sol.Z, **{k: v for k, v in s.stats().items()}))
    print(json.dumps({"workload": args.workload, "seed": args.solve_one, "pricing": args.pricing, "solves": out}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="learned", choices=sorted(WORKLOADS))
    ap.add_argument("--pricing", default="learned", choices=["dse", "learned"])
    ap.add_argument("--weights", default=os.path.join(ROOT, "parallel_ds_b200", "weights",
                                                      "scorer_m2000_n4000_d1.npz"))
    ap.add_argument("--tto-lps", type=int, default=32, help="held-out LPs timed alone, learned and plain")
    ap.add_argument("--concurrency", type=int, default=8, help="LPs solved at once per GPU")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--solve-one", type=int, default=None, metavar="SEED",
                    help="solve one LP of the workload alone and print its stats (profiling)")
    ap.add_argument("--repeat", type=int, default=1, help="--solve-one: solves of the same LP")
    ap.add_argument("--pdhg-estimate", type=int, default=0, metavar="ITERS",
                    help="--solve-one: run only the PDHG warm-start estimate for ITERS iterations")
    ap.add_argument("--no-pdhg-cluster", action="store_true", help="PDHG on the launch-per-step graph path")
    ap.add_argument("--no-tune", action="store_true", help="batched workloads: default schedule, no autotuning")
    ap.add_argument("--max-iterations", type=int, default=0, help="--solve-one: iteration cap (0: none)")
    ap.add_argument("--large-iters", type=int, default=3000,
                    help="plain_large workload: iterations of each step's solve (iteration cap)")
    ap.add_argument("--batch-count", type=int, default=0,
                    help="batched workloads: LPs per GPU (default: the workload's 4096 / 65,536)")
    args = ap.parse_args()
    if args.solve_one is not None:
        solve_one(args)
        return
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        if rank == 0:
            if args.workload in BATCH:
                r = batch_cpu_sample(args.workload, seconds=20.0 * args.steps / 3, threads=os.cpu_count() or 1)
                print(json.dumps({"metric": METRIC, "value": r["value"], "unit": "LPs/s", "n_gpus": 0,
                                  "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
                                  "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                                  "impl": "reference", "data": "synthetic: the GPU arm's instances",
                                  "config": {"workload": WORKLOADS[args.workload]["desc"]}, "cpu_baseline": r,
                                  "e2e": {"value": r["value"], "unit": "LPs/s", "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}))
            else:
                print(json.dumps(reference_arm(args)))
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    arm = batch_arm if args.workload in BATCH else (large_arm if args.workload == "plain_large" else our_arm)
    res = arm(args, rank, world, local_rank)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            res["cpu_baseline"] = (batch_cpu_sample(args.workload) if args.workload in BATCH
                                   else large_cpu_sample(args.workload) if args.workload == "plain_large"
                                   else cpu_sample(args.workload))
        print(json.dumps(res))
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
