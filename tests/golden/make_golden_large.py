"""Large reference-pinned fixtures and the reference-vs-restatement survey.

Run from the repository root where the reference sources are available
(after `make -C oracle all crq ref && make -C sogrand_b200/csrc`):

    python tests/golden/make_golden_large.py [--procs N]

For each set below, every codeword is decoded by
  ref   the unmodified reference (oracle/_ref/libsgref.so: the reference's
        SOGRAND_bitSO / early_termination / hard_decision, glibc exp/log),
  twin  the restatement with the decoder's own exp/log (libsg_oracle_twin.so),
  crq   the restatement with correctly rounded exp/log (libsg_oracle_crq.so),
and the discrete results (decoded bits, iterations, NG, NG_p, converged) are
written to tests/golden/golden_large.npz.  The restatements differ from the
reference only through the last bits of exp/log, so the count of codewords
whose statistics differ measures what each exp/log choice costs in
reference parity.  Inputs are sogrand_b200.gen_llr's seeded channel outputs,
checked at test time by SHA-256.
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import multiprocessing as mp
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

LIBS = {
    "ref": os.path.join(ROOT, "oracle", "_ref", "libsgref.so"),
    "twin": os.path.join(ROOT, "oracle", "libsg_oracle_twin.so"),
    "crq": os.path.join(ROOT, "oracle", "libsg_oracle_crq.so"),
}
OUT = os.path.join(ROOT, "tests", "golden", "golden_large.npz")
UINT64_MAX = (1 << 64) - 1
THRES = 1.0 - 1e-5

# (name, seed, n_cw, Eb/N0 dB)
SETS = [
    ("large_2.0dB", 20261204, 4096, 2.0),
    ("large_1.5dB", 20261205, 4096, 1.5),
]

_cache: dict = {}


def _decode(kind, llr):
    """One codeword -> (bits[64] u8, iterations, ng, ng_p, converged)."""
    if kind == "ref":
        lib = _cache.get("ref")
        if lib is None:
            lib = _cache["ref"] = C.CDLL(LIBS["ref"])
            dp = np.ctypeslib.ndpointer(np.float64, flags="C")
            u8 = np.ctypeslib.ndpointer(np.uint8, flags="C")
            u64 = np.ctypeslib.ndpointer(np.uint64, flags="C")
            i32 = np.ctypeslib.ndpointer(np.int32, flags="C")
            lib.sgref_decode.argtypes = [dp, C.c_size_t, C.c_int, C.c_int, C.c_uint64, C.c_double, dp, u8,
                                         C.c_void_p, dp, u64, u64, i32]
        bits = np.zeros(64, np.uint8)
        it = np.zeros(1)
        ng = np.zeros(1, np.uint64)
        ngp = np.zeros(1, np.uint64)
        cv = np.zeros(1, np.int32)
        lib.sgref_decode(np.ascontiguousarray(llr), 1, 3, 30, UINT64_MAX, THRES, np.full(100, 0.7), bits, None,
                         it, ng, ngp, cv)
        return bits, float(it[0]), int(ng[0]), int(ngp[0]), int(cv[0])
    from oracle_api import Oracle

    o = _cache.get(kind)
    if o is None:
        o = _cache[kind] = Oracle(LIBS[kind])
    b, st, _ = o.decode(llr)
    s = st[0]
    return b[0], s[0], int(s[1]), int(s[2]), int(s[3])


def _job(args):
    kind, llr = args
    return _decode(kind, llr)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--procs", type=int, default=max(1, (os.cpu_count() or 2) - 1))
    ap.add_argument("--n-cw", type=int, default=0, help="override the codewords per set (testing the script)")
    args = ap.parse_args()
    for f in LIBS.values():
        if not os.path.exists(f):
            sys.exit(f"missing {f}: run `make -C oracle all crq ref` first")
    import sogrand_b200 as sg

    out = {}
    t0 = time.time()
    ctx = mp.get_context("spawn")
    with ctx.Pool(args.procs) as pool:
        for name, seed, n, snr in SETS:
            n = args.n_cw or n
            info, llr = sg.gen_llr(seed, 0, n, ebn0_db=snr)
            out[f"{name}/meta"] = np.array([seed, n], np.int64)
            out[f"{name}/ebn0_db"] = np.array(snr)
            out[f"{name}/llr_sha256"] = np.array(hashlib.sha256(llr.tobytes()).hexdigest())
            out[f"{name}/info_sha256"] = np.array(hashlib.sha256(info.tobytes()).hexdigest())
            for kind in LIBS:
                res = pool.map(_job, [(kind, llr[i]) for i in range(n)], chunksize=4)
                out[f"{name}/{kind}_bits"] = np.stack([r[0] for r in res]).astype(np.uint8)
                out[f"{name}/{kind}_iterations"] = np.array([r[1] for r in res])
                out[f"{name}/{kind}_ng"] = np.array([r[2] for r in res], np.uint64)
                out[f"{name}/{kind}_ng_p"] = np.array([r[3] for r in res], np.uint64)
                out[f"{name}/{kind}_converged"] = np.array([r[4] for r in res], np.int8)
                print(f"{name} {kind}: {time.time() - t0:.0f}s", flush=True)
            for kind in ("twin", "crq"):
                d = np.zeros(n, bool)
                for f in ("iterations", "ng", "ng_p", "converged"):
                    d |= out[f"{name}/{kind}_{f}"] != out[f"{name}/ref_{f}"]
                d |= (out[f"{name}/{kind}_bits"] != out[f"{name}/ref_bits"]).any(axis=1)
                print(f"{name}: {kind} differs from the reference on {d.sum()} of {n} codewords: "
                      f"{np.flatnonzero(d).tolist()}", flush=True)
    # Bits agree between the three decoders except where recorded; store the
    # reference bits once and the others only where they differ.
    for name, *_ in SETS:
        rb = out[f"{name}/ref_bits"]
        for kind in ("twin", "crq"):
            kb = out.pop(f"{name}/{kind}_bits")
            idx = np.flatnonzero((kb != rb).any(axis=1))
            out[f"{name}/{kind}_bits_diff_idx"] = idx
            out[f"{name}/{kind}_bits_diff"] = kb[idx]
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} in {time.time() - t0:.0f}s")


if __name__ == "__main__":
    main()
