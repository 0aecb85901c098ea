"""BER / throughput sweep over Eb/N0: the reference flow's
generate_bin -> cubic_encoder -> channel_sim -> cubic_decoder -> comparator
(SOGRAND_C/cubic_flow.sh) at scale, on the device.

    python -m sogrand_b200.sweep --ebn0 1.0:3.0:0.25 --n-cw 100000 --out sweep.json

For every Eb/N0 point, n codewords of the seeded stream are generated,
encoded and sent through the BPSK/AWGN channel on the GPU, decoded, and
compared with the transmitted information bits on the GPU
(sg_decode_summary_device).  Reported per point: codewords/s of the
decode-and-compare call (CUDA events), BER and block error rate with 95%
Wilson intervals, average iterations (the reference's units) and NG per
codeword.
"""
from __future__ import annotations

import argparse
import json


def parse_points(spec: str) -> list[float]:
    """'a:b:step' (inclusive) or a comma list."""
    if ":" in spec:
        a, b, st = (float(x) for x in spec.split(":"))
        n = int(round((b - a) / st)) + 1
        return [round(a + i * st, 10) for i in range(n)]
    return [float(x) for x in spec.split(",")]


def sweep(points, n_cw: int, seed: int = 20261203, chunk: int = 100000, params=None):
    import torch

    import sogrand_b200 as sg

    p = params or sg.params()
    rows = []
    for eb in points:
        tot = {k: 0 for k in sg.SUMMARY_DTYPE.names}
        ms = 0.0
        for off in range(0, n_cw, chunk):
            n = min(chunk, n_cw - off)
            info, llr = sg.gen_llr(seed, off, n, ebn0_db=eb, device="cuda")
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            s, _ = sg.decode_summary(llr, p, ref_info=info)
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            for k in tot:
                tot[k] += s[k]
            del info, llr
        ber_lo, ber_hi = sg.wilson_interval(tot["bit_errors"], tot["bits_compared"])
        bl_lo, bl_hi = sg.wilson_interval(tot["block_errors"], tot["blocks"])
        rows.append({
            "ebn0_db": eb, "codewords": tot["blocks"], "codewords_per_s": tot["blocks"] / (ms / 1e3),
            "ber": tot["bit_errors"] / tot["bits_compared"], "ber_ci95": [ber_lo, ber_hi],
            "bler": tot["block_errors"] / tot["blocks"], "bler_ci95": [bl_lo, bl_hi],
            "avg_iterations": tot["total_iterations"] / tot["blocks"],
            "ng_per_codeword": tot["total_ng"] / tot["blocks"],
            "nonfinite": tot["nonfinite"],
        })
    return rows


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--ebn0", default="1.0:3.0:0.25", help="a:b:step or a comma list (dB)")
    ap.add_argument("--n-cw", type=int, default=100000, help="codewords per point")
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    rows = sweep(parse_points(args.ebn0), args.n_cw, args.seed)
    print(f"{'Eb/N0':>6} {'cw/s':>9} {'BER':>10} {'95% CI':>23} {'BLER':>9} {'iter':>6} {'NG/cw':>10}")
    for r in rows:
        print(f"{r['ebn0_db']:6.2f} {r['codewords_per_s']:9.0f} {r['ber']:10.3e} "
              f"[{r['ber_ci95'][0]:9.2e},{r['ber_ci95'][1]:9.2e}] {r['bler']:9.2e} {r['avg_iterations']:6.2f} "
              f"{r['ng_per_codeword']:10.0f}", flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(rows, f, indent=1)


if __name__ == "__main__":
    main()
