"""Learn per-phase extrinsic weights and evaluate them by BER against the plain
decoder.

    python -m sogrand_b200.learn --steps 60 --batch 4096 --train-ebn0 1.5 \
        --eval-ebn0 1.25,1.5,1.75,2.0 --eval-cw 500000 --eval-imax 5,10,30 --out learned.json

Training: Adam on 3*Imax weights (initialised to the reference's 0.7) with
the BCE of the final APP on fresh seeded codewords (sogrand_b200.diff).
Evaluation: the plain decoder (alpha = 0.7, Imax = 30) and the learned
weights at each Imax decode the same fresh codewords (a codeword range of
the seeded stream disjoint from training); BER and block error rate come
with 95% Wilson intervals, and the difference of BERs with a 95% interval
(normal approximation of the two independent-sample difference).
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

Z95 = 1.959963984540054


def evaluate(alpha, imax: int, ebn0: float, n_cw: int, seed: int, cw0: int, chunk: int = 100000, variant=None):
    import torch

    import sogrand_b200 as sg

    a = np.full(sg.SG_MAX_PHASES, 0.7)
    if alpha is not None:
        a[: min(len(alpha), 3 * imax)] = np.asarray(alpha)[: 3 * imax]
    p = sg.params(Imax=imax, alpha=a)
    tot = {k: 0 for k in sg.SUMMARY_DTYPE.names}
    t = 0.0
    for off in range(0, n_cw, chunk):
        n = min(chunk, n_cw - off)
        info, llr = sg.gen_llr(seed, cw0 + off, n, ebn0_db=ebn0, device="cuda")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s, _ = sg.decode_summary(llr, p, ref_info=info)
        t += time.perf_counter() - t0
        for k in tot:
            tot[k] += s[k]
        del info, llr
    ber = tot["bit_errors"] / tot["bits_compared"]
    lo, hi = sg.wilson_interval(tot["bit_errors"], tot["bits_compared"])
    blo, bhi = sg.wilson_interval(tot["block_errors"], tot["blocks"])
    return {"imax": imax, "ebn0_db": ebn0, "codewords": tot["blocks"], "bit_errors": tot["bit_errors"],
            "ber": ber, "ber_ci95": [lo, hi], "block_errors": tot["block_errors"],
            "bler": tot["block_errors"] / tot["blocks"], "bler_ci95": [blo, bhi],
            "avg_iterations": tot["total_iterations"] / tot["blocks"], "codewords_per_s": tot["blocks"] / t}


def ber_difference(a: dict, b: dict) -> dict:
    """BER(a) - BER(b) with a 95% normal-approximation interval."""
    na = a["codewords"] * 512
    nb = b["codewords"] * 512
    pa, pb = a["ber"], b["ber"]
    se = math.sqrt(pa * (1 - pa) / na + pb * (1 - pb) / nb)
    d = pa - pb
    return {"diff": d, "ci95": [d - Z95 * se, d + Z95 * se]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--train-ebn0", type=float, default=1.5)
    ap.add_argument("--imax-train", type=int, default=30)
    ap.add_argument("--lr", type=float, default=0.02)
    ap.add_argument("--weights", default=None, help="json with learned weights (skip training)")
    ap.add_argument("--val-cw", type=int, default=0, help="validation codewords (keep the best weights)")
    ap.add_argument("--val-every", type=int, default=10)
    ap.add_argument("--eval-ebn0", default="1.25,1.5,1.75,2.0")
    ap.add_argument("--eval-cw", type=int, default=500000)
    ap.add_argument("--eval-imax", default="5,10,30")
    ap.add_argument("--seed", type=int, default=90210)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()

    from sogrand_b200 import diff

    t0 = time.perf_counter()
    if args.weights:
        alpha = np.array(json.load(open(args.weights))["weights"])
        hist = []
    else:
        alpha, hist = diff.train_weights(steps=args.steps, batch=args.batch, ebn0_db=args.train_ebn0,
                                         imax=args.imax_train, lr=args.lr, seed=args.seed, val_cw=args.val_cw,
                                         val_every=args.val_every,
                                         log=lambda s, l, v: print(f"step {s} loss {l:.4f} val {v}", flush=True))
    train_s = time.perf_counter() - t0
    res = {"weights": [float(x) for x in alpha], "train": {"steps": args.steps, "batch": args.batch,
                                                          "val_cw": args.val_cw,
                                                          "ebn0_db": args.train_ebn0, "imax": args.imax_train,
                                                          "lr": args.lr, "loss": hist, "seconds": train_s},
           "eval": []}
    eval_seed = args.seed + 1  # a stream disjoint from training
    for eb in [float(x) for x in args.eval_ebn0.split(",")]:
        plain = evaluate(None, 30, eb, args.eval_cw, eval_seed, 0)
        row = {"ebn0_db": eb, "plain_imax30": plain, "learned": [], "plain": []}
        for im in [int(x) for x in args.eval_imax.split(",")]:
            r = evaluate(alpha, im, eb, args.eval_cw, eval_seed, 0)
            r["ber_minus_plain_imax30"] = ber_difference(r, plain)
            pl = plain if im == 30 else evaluate(None, im, eb, args.eval_cw, eval_seed, 0)
            r["ber_minus_plain_same_imax"] = ber_difference(r, pl)
            row["learned"].append(r)
            row["plain"].append(pl)
        res["eval"].append(row)
        print(json.dumps(row), flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
