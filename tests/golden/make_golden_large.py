"""Large reference-pinned fixtures and the glibc / correctly-rounded survey.

Run from the repository root where the reference sources are available
(after `make -C oracle all ref REF=<reference root>` and
`make -C sogrand_b200/csrc`):

    python tests/golden/make_golden_large.py [--procs N] [--kinds ref,ref_cr,twin] [--sets a,b]

For each set below, every codeword is decoded by
  ref     the unmodified reference (oracle/_ref/libsgref.so: the reference's
          SOGRAND_bitSO / early_termination / hard_decision, glibc exp/log),
  ref_cr  the same unmodified source under a correctly rounded exp/log
          (oracle/_ref/libsgref_cr.so) -- the decoder's exact target,
  twin    the restatement with the table-driven exp/log of sg_math.h
          (within 0.51 ulp, not correctly rounded; libsg_oracle_twin.so),
          the decoder's default math mode,
and the discrete results (decoded bits, iterations, NG, NG_p, converged)
are written to tests/golden/golden_large.npz.  Under a finite Tmax a line
decode that lists no codeword makes the reference read an uninitialised
list size (cubic_decoder_final.c:524); such codewords are flagged
(`<kind>_undefined`) and left out of the comparisons with the reference.  ref and ref_cr differ only
through glibc's misrounded last bits, twin only through its own, so the count
of codewords whose results differ from ref measures what each exp/log
choice costs in parity with the glibc-linked reference.  Results already in
the output file for the same inputs (same LLR SHA-256) are reused for kinds
not listed in --kinds, and sets not listed in --sets are carried over
unchanged.  Inputs are sogrand_b200.gen_llr's seeded channel
outputs, checked at test time by SHA-256.
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
    "ref_cr": os.path.join(ROOT, "oracle", "_ref", "libsgref_cr.so"),
    "twin": os.path.join(ROOT, "oracle", "libsg_oracle_twin.so"),
}
OUT = os.path.join(ROOT, "tests", "golden", "golden_large.npz")
UINT64_MAX = (1 << 64) - 1
THRES = 1.0 - 1e-5
FIELDS = ("iterations", "ng", "ng_p", "converged")

# (name, seed, n_cw, Eb/N0 dB, Tmax)
SETS = [
    ("large_2.0dB", 20261204, 4096, 2.0, UINT64_MAX),
    ("large_1.5dB", 20261205, 4096, 1.5, UINT64_MAX),
    ("large_1.0dB", 20261206, 1024, 1.0, UINT64_MAX),
    ("large_2.5dB", 20261207, 2048, 2.5, UINT64_MAX),
    ("large_tmax1000_1.5dB", 20261208, 1024, 1.5, 1000),
]

_cache: dict = {}


def _decode(kind, llr, tmax):
    """One codeword -> (bits[64] u8, iterations, ng, ng_p, converged,
    undefined).  undefined: a line decode of the reference read its
    uninitialised list size (possible only under a finite Tmax; the
    reference's output is undefined then; the restatement's is defined)."""
    if kind in ("ref", "ref_cr"):
        lib = _cache.get(kind)
        if lib is None:
            lib = _cache[kind] = C.CDLL(LIBS[kind])
            dp = np.ctypeslib.ndpointer(np.float64, flags="C")
            u8 = np.ctypeslib.ndpointer(np.uint8, flags="C")
            u64 = np.ctypeslib.ndpointer(np.uint64, flags="C")
            i32 = np.ctypeslib.ndpointer(np.int32, flags="C")
            lib.sgref_decode.argtypes = [dp, C.c_size_t, C.c_int, C.c_int, C.c_uint64, C.c_double, dp, u8,
                                         C.c_void_p, dp, u64, u64, i32]
            lib.sgref_decode_checked.argtypes = [dp, C.c_size_t, C.c_int, C.c_int, C.c_uint64, C.c_double, dp,
                                                 u8, C.c_void_p, dp, u64, u64, i32, i32]
        bits = np.zeros(64, np.uint8)
        it = np.zeros(1)
        ng = np.zeros(1, np.uint64)
        ngp = np.zeros(1, np.uint64)
        cv = np.zeros(1, np.int32)
        und = np.zeros(1, np.int32)
        if tmax == UINT64_MAX:
            lib.sgref_decode(np.ascontiguousarray(llr), 1, 3, 30, tmax, THRES, np.full(100, 0.7), bits, None,
                             it, ng, ngp, cv)
        else:
            lib.sgref_decode_checked(np.ascontiguousarray(llr), 1, 3, 30, tmax, THRES, np.full(100, 0.7), bits,
                                     None, it, ng, ngp, cv, und)
        return bits, float(it[0]), int(ng[0]), int(ngp[0]), int(cv[0]), int(und[0] != 0)
    from oracle_api import Oracle

    o = _cache.get(kind)
    if o is None:
        o = _cache[kind] = Oracle(LIBS[kind])
    b, st, _ = o.decode(llr, Tmax=tmax)
    s = st[0]
    return b[0], s[0], int(s[1]), int(s[2]), int(s[3]), 0


def _job(args):
    kind, llr, tmax = args
    return _decode(kind, llr, tmax)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--procs", type=int, default=max(1, (os.cpu_count() or 2) - 1))
    ap.add_argument("--kinds", default="ref,ref_cr,twin")
    ap.add_argument("--sets", default="", help="compute only these sets (comma list); the others are carried over")
    ap.add_argument("--n-cw", type=int, default=0, help="override the codewords per set (testing the script)")
    ap.add_argument("--out", default=OUT)
    args = ap.parse_args()
    kinds = args.kinds.split(",")
    for k in kinds:
        if not os.path.exists(LIBS[k]):
            sys.exit(f"missing {LIBS[k]}: run `make -C oracle all ref REF=...` first")
    import sogrand_b200 as sg

    old = dict(np.load(args.out)) if os.path.exists(args.out) else {}
    out = {}
    t0 = time.time()
    ctx = mp.get_context("spawn")
    only = set(args.sets.split(",")) if args.sets else None
    with ctx.Pool(args.procs) as pool:
        for name, seed, n, snr, tmax in SETS:
            if only is not None and name not in only:
                for k, v in old.items():
                    if k.startswith(name + "/"):
                        out[k] = v
                continue
            n = args.n_cw or n
            info, llr = sg.gen_llr(seed, 0, n, ebn0_db=snr)
            sha = hashlib.sha256(llr.tobytes()).hexdigest()
            out[f"{name}/meta"] = np.array([seed, n], np.int64)
            out[f"{name}/ebn0_db"] = np.array(snr)
            out[f"{name}/tmax"] = np.array(tmax, np.uint64)
            out[f"{name}/llr_sha256"] = np.array(sha)
            out[f"{name}/info_sha256"] = np.array(hashlib.sha256(info.tobytes()).hexdigest())
            same_inputs = str(old.get(f"{name}/llr_sha256", "")) == sha
            full = {}
            for kind in ("ref", "ref_cr", "twin"):
                if kind not in kinds:
                    if same_inputs and f"{name}/{kind}_ng" in old:
                        bits = old[f"{name}/ref_bits"].copy()
                        if kind != "ref":
                            bits[old[f"{name}/{kind}_bits_diff_idx"]] = old[f"{name}/{kind}_bits_diff"]
                        full[kind] = {"bits": bits, **{f: old[f"{name}/{kind}_{f}"] for f in FIELDS},
                                      "undefined": old.get(f"{name}/{kind}_undefined", np.zeros(n, np.int8))}
                    continue
                res = pool.map(_job, [(kind, llr[i], tmax) for i in range(n)], chunksize=4)
                full[kind] = {"bits": np.stack([r[0] for r in res]).astype(np.uint8),
                              "iterations": np.array([r[1] for r in res]),
                              "ng": np.array([r[2] for r in res], np.uint64),
                              "ng_p": np.array([r[3] for r in res], np.uint64),
                              "converged": np.array([r[4] for r in res], np.int8),
                              "undefined": np.array([r[5] for r in res], np.int8)}
                print(f"{name} {kind}: {time.time() - t0:.0f}s", flush=True)
            # the reference's bits stored once, the others where they differ
            rb = full["ref"]["bits"]
            out[f"{name}/ref_bits"] = rb
            for kind, d in full.items():
                for f in FIELDS:
                    out[f"{name}/{kind}_{f}"] = d[f]
                out[f"{name}/{kind}_undefined"] = d["undefined"]
                if kind == "ref":
                    continue
                idx = np.flatnonzero((d["bits"] != rb).any(axis=1))
                out[f"{name}/{kind}_bits_diff_idx"] = idx
                out[f"{name}/{kind}_bits_diff"] = d["bits"][idx]
                diff = (d["bits"] != rb).any(axis=1)
                for f in FIELDS:
                    diff |= d[f] != full["ref"][f]
                # only where both outputs are defined
                defined = (full["ref"]["undefined"] == 0) & (d["undefined"] == 0)
                diff &= defined
                out[f"{name}/ref_vs_{kind}_idx"] = np.flatnonzero(diff)
                print(f"{name}: {kind} differs from the glibc-linked reference on {diff.sum()} of {defined.sum()} "
                      f"defined codewords ({n - defined.sum()} undefined): {np.flatnonzero(diff).tolist()}",
                      flush=True)
    np.savez_compressed(args.out, **out)
    print(f"wrote {args.out} in {time.time() - t0:.0f}s")


if __name__ == "__main__":
    main()
