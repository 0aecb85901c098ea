"""Learn per-phase extrinsic weights and evaluate them by BER against the plain
decoder.

    python -m sogrand_b200.learn --steps 60 --batch 4096 --train-ebn0 1.5 --loss phases \
        --eval-ebn0 1.25,1.5,1.75,2.0 --eval-cw 500000 --eval-imax 5,10,30 --out learned.json

Training: Adam on 3*Imax weights (initialised to the reference's 0.7) with
the BCE of the final APP, or of every phase's APP (--loss phases), on fresh
seeded codewords (sogrand_b200.diff).  Or, with --search, no gradient: every
linear weight ramp alpha_p = a + b*p/(3*Imax-1) of a grid decodes the same
search batch and the ramp with the lowest BER is kept (the BCE gradient
holds the decode's discrete branch fixed, while the weights move BER mostly
through that branch).
Evaluation: the plain decoder (alpha = 0.7, Imax = 30, and at each evaluated
Imax) and the learned weights at each Imax decode the same fresh codewords
(a codeword range of the seeded stream disjoint from training).  Every
decoder sees the same codewords, so BER differences are paired: per
codeword, d = (bit errors of one decoder) - (bit errors of the other), and
the 95% interval of the BER difference is mean(d)/512 +- 1.96 sd(d) /
(512 sqrt(n)).  BER and block error rate come with 95% Wilson intervals.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

Z95 = 1.959963984540054


def _popcount_table():
    import torch

    t = torch.zeros(256, dtype=torch.int16)
    for i in range(256):
        t[i] = bin(i).count("1")
    return t


def evaluate_set(configs: dict, ebn0: float, n_cw: int, seed: int, cw0: int, chunk: int = 100000,
                 pairs=()) -> dict:
    """Decode the same n_cw fresh codewords with every configuration
    (name -> (alpha or None for the reference's 0.7, Imax)).  Returns per
    configuration its totals, and for every (a, b) in pairs the paired BER
    difference BER(a) - BER(b) with its 95% interval."""
    import torch

    import sogrand_b200 as sg

    pop = _popcount_table().cuda()
    params = {}
    for name, (alpha, imax) in configs.items():
        a = np.full(sg.SG_MAX_PHASES, 0.7)
        if alpha is not None:
            a[: min(len(alpha), 3 * imax)] = np.asarray(alpha)[: 3 * imax]
        params[name] = sg.params(Imax=imax, alpha=a)
    tot = {k: {"bit_errors": 0, "block_errors": 0, "iterations": 0.0, "seconds": 0.0} for k in configs}
    acc = {pr: [0.0, 0.0] for pr in pairs}  # sum d, sum d^2
    for off in range(0, n_cw, chunk):
        n = min(chunk, n_cw - off)
        info, llr = sg.gen_llr(seed, cw0 + off, n, ebn0_db=ebn0, device="cuda")
        errs = {}
        for name, p in params.items():
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            bits, raw, _ = sg.decode(llr, p)
            e1.record()
            torch.cuda.synchronize()
            tot[name]["seconds"] += e0.elapsed_time(e1) / 1000.0
            e = pop[(bits ^ info).long()].sum(dim=1).to(torch.int64)
            errs[name] = e
            tot[name]["bit_errors"] += int(e.sum().item())
            tot[name]["block_errors"] += int((e > 0).sum().item())
            tot[name]["iterations"] += float(sg.stats_from_device(raw)["iterations"].sum())
        for a, b in pairs:
            d = (errs[a] - errs[b]).to(torch.float64)
            acc[(a, b)][0] += float(d.sum().item())
            acc[(a, b)][1] += float((d * d).sum().item())
        del info, llr
    out = {"ebn0_db": ebn0, "codewords": n_cw, "configs": {}, "paired": []}
    for name, t in tot.items():
        nb = n_cw * 512
        lo, hi = sg.wilson_interval(t["bit_errors"], nb)
        blo, bhi = sg.wilson_interval(t["block_errors"], n_cw)
        out["configs"][name] = {
            "imax": configs[name][1], "learned": configs[name][0] is not None, "bit_errors": t["bit_errors"],
            "ber": t["bit_errors"] / nb, "ber_ci95": [lo, hi], "block_errors": t["block_errors"],
            "bler": t["block_errors"] / n_cw, "bler_ci95": [blo, bhi],
            "avg_iterations": t["iterations"] / n_cw, "codewords_per_s": n_cw / t["seconds"]}
    for (a, b), (s1, s2) in acc.items():
        mean = s1 / n_cw
        var = max(s2 / n_cw - mean * mean, 0.0) * n_cw / max(n_cw - 1, 1)
        se = math.sqrt(var / n_cw)
        d = mean / 512
        out["paired"].append({"a": a, "b": b, "ber_diff": d,
                              "ci95": [d - Z95 * se / 512, d + Z95 * se / 512],
                              "rel": d / out["configs"][b]["ber"] if out["configs"][b]["ber"] else None})
    return out


def schedule(a: float, b: float, imax: int) -> np.ndarray:
    """Per-phase weights alpha_p = a + b * p / (3*Imax - 1), p = 0 .. 3*Imax-1
    (a linear ramp over the decode; b = 0 is a constant, and a = 0.7, b = 0
    the reference's weights), clipped to [0.05, 1.5]."""
    n = 3 * imax
    t = np.arange(n) / max(n - 1, 1)
    return np.clip(a + b * t, 0.05, 1.5)


def search_schedules(imax: int, ebn0: float, n_cw: int, seed: int, a_grid, b_grid, chunk: int = 100000) -> dict:
    """Derivative-free search for weights: every ramp (a, b) of the grid and
    the reference's weights decode the same n_cw codewords at Imax; each
    ramp is scored by its paired BER difference from the reference's.
    Returns the table and the best ramp (lowest BER)."""
    configs = {"plain": (None, imax)}
    names = {}
    for a in a_grid:
        for b in b_grid:
            k = f"a{a:.2f}_b{b:+.2f}"
            names[k] = (float(a), float(b))
            configs[k] = (schedule(a, b, imax), imax)
    row = evaluate_set(configs, ebn0, n_cw, seed, 0, chunk=chunk, pairs=[(k, "plain") for k in names])
    table = []
    for pr in row["paired"]:
        a, b = names[pr["a"]]
        c = row["configs"][pr["a"]]
        table.append({"a": a, "b": b, "ber": c["ber"], "ber_diff_vs_plain": pr["ber_diff"], "ci95": pr["ci95"],
                      "avg_iterations": c["avg_iterations"]})
    best = min(table, key=lambda r: r["ber"])
    return {"imax": imax, "ebn0_db": ebn0, "codewords": n_cw, "seed": seed,
            "plain_ber": row["configs"]["plain"]["ber"], "table": table, "best": best}


def search_schedules_multi(imax: int, points, seed: int, a_grid, b_grid) -> dict:
    """search_schedules at several (Eb/N0, codewords) points; the kept ramp
    is the one whose worst relative BER change from the reference's weights
    over the points is lowest (below 0: better at every point)."""
    runs = [search_schedules(imax, eb, n, seed + 1000 * i, a_grid, b_grid) for i, (eb, n) in enumerate(points)]
    score = {}
    for run in runs:
        for r in run["table"]:
            rel = r["ber"] / run["plain_ber"] - 1.0 if run["plain_ber"] else 0.0
            key = (r["a"], r["b"])
            score[key] = max(score.get(key, -math.inf), rel)
    (a, b), worst = min(score.items(), key=lambda kv: kv[1])
    return {"imax": imax, "points": [{"ebn0_db": eb, "codewords": n} for eb, n in points], "runs": runs,
            "worst_relative_ber_change": [{"a": k[0], "b": k[1], "worst": v} for k, v in score.items()],
            "best": {"a": a, "b": b, "worst_relative_ber_change": worst}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--train-ebn0", type=float, default=1.5)
    ap.add_argument("--imax-train", type=int, default=30)
    ap.add_argument("--lr", type=float, default=0.02)
    ap.add_argument("--loss", default="final", choices=["final", "phases"])
    ap.add_argument("--weights", default=None, help="json with learned weights (skip training)")
    ap.add_argument("--val-cw", type=int, default=0, help="validation codewords (keep the best weights)")
    ap.add_argument("--val-every", type=int, default=10)
    ap.add_argument("--eval-ebn0", default="1.25,1.5,1.75,2.0")
    ap.add_argument("--eval-cw", type=int, default=500000)
    ap.add_argument("--eval-imax", default="5,10,30")
    ap.add_argument("--no-plain-same-imax", action="store_true",
                    help="compare only against the plain decoder at Imax 30")
    ap.add_argument("--search", action="store_true",
                    help="instead of gradient training, pick the best linear weight ramp by BER (search_schedules)")
    ap.add_argument("--search-cw", default="200000",
                    help="search codewords, one number or one per --search-ebn0 point")
    ap.add_argument("--search-ebn0", default=None,
                    help="search points (dB, comma list; default --train-ebn0); several: minimax over them")
    ap.add_argument("--search-a", default="0.5,0.6,0.7,0.8,0.9,1.0")
    ap.add_argument("--search-b", default="-0.4,-0.2,0,0.2,0.4")
    ap.add_argument("--seed", type=int, default=90210)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()

    from sogrand_b200 import diff

    t0 = time.perf_counter()
    search = None
    if args.weights:
        alpha = np.array(json.load(open(args.weights))["weights"])
        hist = []
    elif args.search:
        agrid = [float(x) for x in args.search_a.split(",")]
        bgrid = [float(x) for x in args.search_b.split(",")]
        ebs = [float(x) for x in args.search_ebn0.split(",")] if args.search_ebn0 else [args.train_ebn0]
        cws = [int(x) for x in args.search_cw.split(",")]
        cws = cws * len(ebs) if len(cws) == 1 else cws
        if len(ebs) == 1:
            search = search_schedules(args.imax_train, ebs[0], cws[0], args.seed, agrid, bgrid)
            tables = [search]
        else:
            search = search_schedules_multi(args.imax_train, list(zip(ebs, cws)), args.seed, agrid, bgrid)
            tables = search["runs"]
        for run in tables:
            for r in run["table"]:
                print(f"{run['ebn0_db']} dB a {r['a']:.2f} b {r['b']:+.2f} BER {r['ber']:.4e} vs plain "
                      f"{r['ber_diff_vs_plain']:+.3e} [{r['ci95'][0]:+.2e}, {r['ci95'][1]:+.2e}]", flush=True)
        alpha = schedule(search["best"]["a"], search["best"]["b"], args.imax_train)
        hist = []
    else:
        alpha, hist = diff.train_weights(steps=args.steps, batch=args.batch, ebn0_db=args.train_ebn0,
                                         imax=args.imax_train, lr=args.lr, seed=args.seed, val_cw=args.val_cw,
                                         val_every=args.val_every, loss=args.loss,
                                         log=lambda s, l, v: print(f"step {s} loss {l:.4f} val {v}", flush=True))
    train_s = time.perf_counter() - t0
    res = {"weights": [float(x) for x in alpha],
           "train": {"steps": args.steps, "batch": args.batch, "val_cw": args.val_cw, "loss": args.loss,
                     "ebn0_db": args.train_ebn0, "imax": args.imax_train, "lr": args.lr, "history": hist,
                     "seconds": train_s},
           "search": search, "eval": []}
    eval_seed = args.seed + 1  # a stream disjoint from training
    imaxes = [int(x) for x in args.eval_imax.split(",")]
    configs = {"plain30": (None, 30)}
    pairs = []
    for im in imaxes:
        configs[f"learned{im}"] = (alpha, im)
        pairs.append((f"learned{im}", "plain30"))
        if im != 30 and not args.no_plain_same_imax:
            configs[f"plain{im}"] = (None, im)
            pairs.append((f"learned{im}", f"plain{im}"))
    for eb in [float(x) for x in args.eval_ebn0.split(",") if x.strip()]:
        row = evaluate_set(configs, eb, args.eval_cw, eval_seed, 0, pairs=pairs)
        res["eval"].append(row)
        print(json.dumps(row), flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
