"""Train the leaving-row network on plain-solver traces and evaluate it.

    python -m parallel_ds_b200.train_scorer --train-seeds 0:64 --eval-seeds 100000:100200

1. Solve the training LPs (m=2000, n=4000, density 1% unless overridden) with
   the plain DSE path, recording candidate-row features every --every
   iterations; label a record 1 when its basic variable is nonbasic at the
   optimum.
2. Train the network on the GPU (tensor-core forward/backward, Adam).
3. Solve the held-out LPs with plain and learned pricing; report iterations,
   device time to optimal and the objective difference.
4. Write the parameters (and the evaluation summary) to --out.
"""
import argparse
import json
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import learned as LN
from . import lp as L
from . import solver as S


def seed_range(text):
    a, b = text.split(":")
    return list(range(int(a), int(b)))


def make_lp(seed, m, n, density):
    return L.generate(m=m, n=n, density=density, seed=seed)


def trace_one(args):
    seed, m, n, density, every, cap = args
    lp = make_lp(seed, m, n, density)
    res, F, y, M = LN.solve_with_trace(lp, every=every, cap=cap)
    return seed, res, F, y


def solve_one(lp, model=None, **kw):
    s = S.CudaDualSimplex(S.problem_from_lp(lp), model=model,
                          pricing="learned" if model is not None else "dse", **kw)
    s.initDualSimplex()
    sol = s.solve()
    st = s.stats()
    return dict(status=s.status(), objective=sol.Z, iterations=st["iterations"], solve_ms=st["solve_ms"],
                pdhg_ms=st["pdhg_ms"], learned_used=st["learned_used"], learned_fallback=st["learned_fallback"])


def evaluate(model, seeds, m, n, density, margin, mix, time_seeds=8, concurrency=8, log=print):
    """Iterations and objectives of plain vs learned solves on every held-out
    seed (solved concurrently), and time to optimal of each solved alone on the
    first `time_seeds` seeds (after one warm-up solve of each kind)."""
    def pair(seed):
        lp = make_lp(seed, m, n, density)
        a = solve_one(lp)
        b = solve_one(lp, model=model, learned_margin=margin, learned_mix=mix)
        rel = abs(a["objective"] - b["objective"]) / max(1.0, abs(a["objective"]))
        return dict(seed=seed, plain=a, learned=b, rel_err=rel)

    with ThreadPoolExecutor(max_workers=concurrency) as ex:
        rows = list(ex.map(pair, seeds))
    it_ratio = sum(r["plain"]["iterations"] for r in rows) / max(1, sum(r["learned"]["iterations"] for r in rows))
    per_lp = [r["plain"]["iterations"] / r["learned"]["iterations"] for r in rows]
    warm = make_lp(seeds[0] + 10**6, m, n, density)
    wa = solve_one(warm)
    wb = solve_one(warm, model=model, learned_margin=margin, learned_mix=mix)
    log(f"warm-up: plain {wa['solve_ms']:.0f} ms, learned {wb['solve_ms']:.0f} ms (pdhg {wb['pdhg_ms']:.1f} ms)")
    timed = []
    for seed in seeds[:time_seeds]:
        r = pair(seed)
        timed.append(r)
        log(f"time {seed}: plain {r['plain']['iterations']} it {r['plain']['solve_ms']:.0f} ms | learned "
            f"{r['learned']['iterations']} it {r['learned']['solve_ms']:.0f} ms (pdhg {r['learned']['pdhg_ms']:.1f} ms, "
            f"used {r['learned']['learned_used']}, fallback {r['learned']['learned_fallback']})")
    t_ratio = (sum(r["plain"]["solve_ms"] for r in timed) / max(1e-9, sum(r["learned"]["solve_ms"] for r in timed))
               if timed else None)
    return dict(seeds=f"{seeds[0]}:{seeds[-1] + 1}", lps=len(rows), iteration_ratio=it_ratio,
                iteration_ratio_min=min(per_lp), iteration_ratio_max=max(per_lp),
                time_ratio=t_ratio, timed=[dict(seed=r["seed"], plain_ms=r["plain"]["solve_ms"],
                                                learned_ms=r["learned"]["solve_ms"],
                                                pdhg_ms=r["learned"]["pdhg_ms"]) for r in timed],
                max_rel_err=max(r["rel_err"] for r in rows),
                all_optimal=all(r["plain"]["status"] == r["learned"]["status"] == "optimal" for r in rows),
                mean_plain_iterations=float(np.mean([r["plain"]["iterations"] for r in rows])),
                mean_learned_iterations=float(np.mean([r["learned"]["iterations"] for r in rows])))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--m", type=int, default=2000)
    ap.add_argument("--n", type=int, default=4000)
    ap.add_argument("--density", type=float, default=0.01)
    ap.add_argument("--train-seeds", type=seed_range, default=seed_range("0:64"))
    ap.add_argument("--eval-seeds", type=seed_range, default=seed_range("100000:100200"))
    ap.add_argument("--every", type=int, default=16)
    ap.add_argument("--cap", type=int, default=1 << 20)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--margin", type=float, default=0.5)
    ap.add_argument("--mix", type=float, default=0.05)
    ap.add_argument("--concurrency", type=int, default=8)
    ap.add_argument("--init-seed", type=int, default=0)
    ap.add_argument("--time-seeds", type=int, default=8)
    ap.add_argument("--out", default=LN.DEFAULT_WEIGHTS)
    ap.add_argument("--summary", default=None)
    a = ap.parse_args(argv)

    t0 = time.time()
    jobs = [(s, a.m, a.n, a.density, a.every, a.cap) for s in a.train_seeds]
    Xs, ys, its = [], [], []
    with ThreadPoolExecutor(max_workers=a.concurrency) as ex:
        for seed, res, F, y in ex.map(trace_one, jobs):
            if res["status"] != "optimal":
                continue
            Xs.append(F); ys.append(y); its.append(res["iterations"])
    X = np.concatenate(Xs); y = np.concatenate(ys)
    t1 = time.time()
    print(f"traces: {len(Xs)} LPs, {len(y)} records, positive {y.mean():.3f}, "
          f"mean iterations {np.mean(its):.0f}, {t1 - t0:.1f} s")

    model = LN.LeavingRowScorer(LN.init_params(a.init_seed))
    rows = (len(y) // a.batch) * a.batch
    loss = model.train(X[:rows], y[:rows], epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.init_seed)
    z = model.forward(X)
    acc = float(np.mean((z > 0) == (y > 0.5)))
    t2 = time.time()
    print(f"train: loss {loss:.4f}, accuracy {acc:.3f}, {t2 - t1:.1f} s")

    ev = evaluate(model, a.eval_seeds, a.m, a.n, a.density, a.margin, a.mix, time_seeds=a.time_seeds,
                  concurrency=a.concurrency)
    t3 = time.time()
    print(f"eval: {ev['lps']} LPs, iteration ratio {ev['iteration_ratio']:.3f} "
          f"[{ev['iteration_ratio_min']:.2f}, {ev['iteration_ratio_max']:.2f}], time ratio {ev['time_ratio']}, "
          f"max rel err {ev['max_rel_err']:.1e}, all optimal {ev['all_optimal']}, {t3 - t2:.1f} s")
    meta = dict(m=a.m, n=a.n, density=a.density, train_seeds=f"{a.train_seeds[0]}:{a.train_seeds[-1] + 1}",
                every=a.every, epochs=a.epochs, batch=a.batch, lr=a.lr, records=len(y),
                positive=float(y.mean()), train_loss=loss, train_accuracy=acc, margin=a.margin, mix=a.mix)
    model.save(a.out, **meta)
    if a.summary:
        with open(a.summary, "w") as f:
            json.dump(dict(meta=meta, eval=ev), f, indent=1)
    return ev


if __name__ == "__main__":
    main()
