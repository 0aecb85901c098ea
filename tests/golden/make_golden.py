"""Generate the golden fixtures of the parity tests.

Run from the repository root (needs the reference sources, so it runs where
the reference is available, not on the GPU machine):

    make -C oracle all ref && make -C sogrand_b200/csrc
    python tests/golden/make_golden.py

Inputs are the seeded synthetic channel outputs of sogrand_b200.gen_llr
(regenerated bit-identically at test time and checked against the SHA-256
recorded here).  Expected outputs come from
  - "ref": the unmodified reference SOGRAND_C/cubic_decoder_final.c with the
    system libm (glibc), through oracle/_ref/libsgref.so (reference functions
    + a per-codeword driver) and, for the main fixture, through the
    unmodified flow binary oracle/_ref/cubic_decoder_final (decoded file and
    printed averages);
  - "ref_cr": the same unmodified source compiled against a correctly
    rounded exp/log (oracle/_ref/libsgref_cr.so, oracle/cr_libm.c) -- the
    bit-exact target of the decoder's reference-exact math mode, soft values
    included (the generator checks that the restatement with the decoder's
    correctly rounded exp/log, oracle/libsg_oracle_twin_cr.so, equals it in
    every recorded value where the reference is defined);
  - "twin": the oracle restatement with the decoder's default, table-driven
    exp/log (oracle/libsg_oracle_twin.so) -- the bit-exact target of the
    default math mode.
"ref" differs from "ref_cr" only where glibc's exp/log are not correctly
rounded, and from "twin" only where glibc's or the table routines' last
bits differ; the counts of codewords where that moves a discrete result are
recorded per set.  Per-line known answers come from both reference builds,
with and without a Tmax cap; a line that lists no codeword under the cap
makes the reference read an uninitialised list size, so only its N_guess is
recorded there.
Writes tests/golden/golden.json and tests/golden/kat_lines.npz.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import multiprocessing as mp
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

REF_SO = os.path.join(ROOT, "oracle", "_ref", "libsgref.so")
REF_CR_SO = os.path.join(ROOT, "oracle", "_ref", "libsgref_cr.so")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "cubic_decoder_final")
TWIN_SO = os.path.join(ROOT, "oracle", "libsg_oracle_twin.so")
TWIN_CR_SO = os.path.join(ROOT, "oracle", "libsg_oracle_twin_cr.so")
OUT_DIR = os.path.join(ROOT, "tests", "golden")
UINT64_MAX = (1 << 64) - 1
THRES = 1.0 - 1e-5

# (name, seed, n_cw, ebn0 dB or (lo, hi), Tmax)
SETS = [
    ("cfg1_2dB_100", 20261203, 100, 2.0, UINT64_MAX),
    ("snr_1.0dB", 101, 24, 1.0, UINT64_MAX),
    ("snr_1.5dB", 102, 24, 1.5, UINT64_MAX),
    ("snr_2.5dB", 103, 24, 2.5, UINT64_MAX),
    ("snr_3.0dB", 104, 24, 3.0, UINT64_MAX),
    ("mixed_1to3dB", 105, 24, (1.0, 3.0), UINT64_MAX),
    # the Tmax-capped mode (the cap is checked once per logistic weight)
    ("tmax1000_2dB", 106, 64, 2.0, 1000),
    ("tmax1000_1.5dB", 107, 64, 1.5, 1000),
]
# per-line known answers under a Tmax cap
KAT_TMAX = (10, 100, 1000)


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def gen(seed, n, snr):
    import sogrand_b200 as sg

    if isinstance(snr, tuple):
        return sg.gen_llr(seed, 0, n, ebn0_range=snr)
    return sg.gen_llr(seed, 0, n, ebn0_db=snr)


class Params(C.Structure):
    _fields_ = [("L", C.c_int), ("Imax", C.c_int), ("Tmax", C.c_uint64), ("thres", C.c_double),
                ("alpha", C.c_double * 150)]


class Stats(C.Structure):
    _fields_ = [("iterations", C.c_double), ("ng", C.c_uint64), ("ng_p", C.c_uint64),
                ("converged", C.c_int), ("phases", C.c_int)]


def ref_one(args):
    """Reference decode of one codeword -> (bits, iters, ng, ngp, conv, lapp
    sha, line decodes that read the reference's uninitialised list size).
    args: (llr, Tmax[, reference library])."""
    llr, tmax = args[:2]
    lib = C.CDLL(args[2] if len(args) > 2 else REF_SO)
    dp = np.ctypeslib.ndpointer(np.float64, flags="C")
    u8 = np.ctypeslib.ndpointer(np.uint8, flags="C")
    u64 = np.ctypeslib.ndpointer(np.uint64, flags="C")
    i32 = np.ctypeslib.ndpointer(np.int32, flags="C")
    lib.sgref_decode_checked.argtypes = [dp, C.c_size_t, C.c_int, C.c_int, C.c_uint64, C.c_double, dp, u8, dp,
                                         dp, u64, u64, i32, i32]
    bits = np.zeros(64, np.uint8)
    lapp = np.zeros(4096)
    it = np.zeros(1)
    ng = np.zeros(1, np.uint64)
    ngp = np.zeros(1, np.uint64)
    cv = np.zeros(1, np.int32)
    und = np.zeros(1, np.int32)
    lib.sgref_decode_checked(np.ascontiguousarray(llr), 1, 3, 30, tmax, THRES, np.full(100, 0.7), bits, lapp, it,
                             ng, ngp, cv, und)
    return (bits.tobytes().hex(), float(it[0]), int(ng[0]), int(ngp[0]), int(cv[0]), sha(lapp.tobytes()),
            int(und[0]))


def twin_one(args):
    """Restatement decode of one codeword; args: (llr, Tmax[, library])."""
    llr, tmax = args[:2]
    lib = C.CDLL(args[2] if len(args) > 2 else TWIN_SO)
    dp = np.ctypeslib.ndpointer(np.float64, flags="C")
    u8 = np.ctypeslib.ndpointer(np.uint8, flags="C")
    lib.sgo_default_params.argtypes = [C.POINTER(Params)]
    lib.sgo_decode.argtypes = [dp, C.c_size_t, C.POINTER(Params), u8, dp, C.POINTER(Stats)]
    p = Params()
    lib.sgo_default_params(C.byref(p))
    p.Tmax = tmax
    st = (Stats * 1)()
    bits = np.zeros(64, np.uint8)
    lapp = np.zeros(4096)
    lib.sgo_decode(np.ascontiguousarray(llr), 1, C.byref(p), bits, lapp, st)
    s = st[0]
    return bits.tobytes().hex(), s.iterations, int(s.ng), int(s.ng_p), int(s.converged), sha(lapp.tobytes())


def kat_lines(rng, cubes):
    """Per-line inputs: slices of decoded-looking cubes at several scales plus
    constructed edge cases (ties, equal magnitudes, zeros, large IC)."""
    lines = []
    n = cubes.shape[0]
    for _ in range(384):
        c = rng.integers(0, n)
        b = rng.integers(0, 4096 - 16)
        lines.append(cubes[c, b:b + 16] * rng.choice([0.5, 1.0, 2.0, 4.0, 8.0, 16.0]))
    # exact ties between magnitudes (the reference's sort order decides)
    for _ in range(48):
        v = rng.normal(0, 2, 16)
        k = rng.integers(2, 8)
        idx = rng.choice(16, k, replace=False)
        v[idx] = np.abs(v[idx[0]]) * rng.choice([-1, 1], k)
        lines.append(v)
    # all magnitudes equal (beta = 0 -> IC = 0 through the int cast)
    for _ in range(16):
        lines.append(rng.choice([-1, 1], 16) * rng.uniform(0.1, 5))
    # exact zeros (hard decision 1, |L| = 0)
    for _ in range(16):
        v = rng.normal(0, 1.5, 16)
        v[rng.choice(16, rng.integers(1, 5), replace=False)] = 0.0
        lines.append(v)
    # nearly equal small magnitudes -> large IC
    for _ in range(32):
        v = rng.choice([-1, 1], 16) * (rng.uniform(5, 30) + rng.uniform(0, 1e-3, 16) * rng.choice([1, 100], 16))
        lines.append(v)
    # very reliable lines (P_notGuess cancels to ~0)
    for _ in range(16):
        lines.append(rng.choice([-1, 1], 16) * rng.uniform(20, 60, 16))
    return np.ascontiguousarray(np.array(lines, dtype=np.float64))


def main():
    for f in (REF_SO, REF_CR_SO, REF_BIN, TWIN_SO, TWIN_CR_SO):
        if not os.path.exists(f):
            sys.exit(f"missing {f}: run `make -C oracle all ref` first")
    golden = {"generator": "sogrand_b200.gen_llr (splitmix counter RNG, polar Gaussian, sg_log)",
              "thres": THRES, "L": 3, "Imax": 30, "sets": {}}
    ctx = mp.get_context("spawn")
    t0 = time.time()
    with ctx.Pool(os.cpu_count()) as pool:
        for name, seed, n, snr, tmax in SETS:
            info, llr = gen(seed, n, snr)
            jobs = [(llr[i], tmax) for i in range(n)]
            ref = pool.map(ref_one, jobs)
            ref_cr = pool.map(ref_one, [(llr[i], tmax, REF_CR_SO) for i in range(n)])
            twin = pool.map(twin_one, jobs)
            twin_cr = pool.map(twin_one, [(llr[i], tmax, TWIN_CR_SO) for i in range(n)])
            for i in range(n):  # the restatement equals the reference under a correctly rounded libm
                if ref_cr[i][6] == 0:
                    assert twin_cr[i][:6] == ref_cr[i][:6], (name, i, twin_cr[i][:5], ref_cr[i][:5])
            entry = {
                "seed": seed, "n_cw": n, "ebn0_db": snr, "Tmax": tmax,
                "llr_sha256": sha(llr.tobytes()), "info_sha256": sha(info.tobytes()),
                "ref": {"bits": [r[0] for r in ref], "iterations": [r[1] for r in ref],
                        "ng": [r[2] for r in ref], "ng_p": [r[3] for r in ref],
                        "converged": [r[4] for r in ref], "lapp_sha256": [r[5] for r in ref],
                        "undefined_lines": [r[6] for r in ref]},
                "ref_cr": {"bits": [r[0] for r in ref_cr], "iterations": [r[1] for r in ref_cr],
                           "ng": [r[2] for r in ref_cr], "ng_p": [r[3] for r in ref_cr],
                           "converged": [r[4] for r in ref_cr], "lapp_sha256": [r[5] for r in ref_cr],
                           "undefined_lines": [r[6] for r in ref_cr]},
                "twin": {"bits": [r[0] for r in twin], "iterations": [r[1] for r in twin],
                         "ng": [r[2] for r in twin], "ng_p": [r[3] for r in twin],
                         "converged": [r[4] for r in twin], "lapp_sha256": [r[5] for r in twin]},
            }
            # over the codewords the reference defines (no line reading its
            # uninitialised list size)
            mism = sum(1 for a, b in zip(ref, ref_cr) if a[6] == 0 and a[:5] != b[:5])
            entry["glibc_vs_cr_mismatches"] = mism
            entry["glibc_vs_twin_mismatches"] = sum(1 for a, b in zip(ref, twin) if a[6] == 0 and a[:5] != b[:5])
            ber = np.mean(np.unpackbits(np.frombuffer(b"".join(bytes.fromhex(r[0]) for r in ref), np.uint8))
                          != np.unpackbits(info.ravel()))
            entry["ref_ber"] = float(ber)
            golden["sets"][name] = entry
            print(f"{name}: {n} cw, glibc-vs-correctly-rounded reference mismatches {mism}, BER {ber:.3g}, "
                  f"avg it {np.mean([r[1] for r in ref]):.2f}, {time.time() - t0:.0f}s", flush=True)

    # the unmodified flow binary on the main fixture: decoded file + averages
    name, seed, n, snr, _ = SETS[0]
    _, llr = gen(seed, n, snr)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "llr.bin"), os.path.join(td, "dec.bin")
        llr.tofile(fin)
        out = subprocess.run([REF_BIN, fin, fout], check=True, capture_output=True, text=True).stdout
        dec = open(fout, "rb").read()
    e = golden["sets"][name]
    assert dec == b"".join(bytes.fromhex(b) for b in e["ref"]["bits"]), "flow binary bits differ from harness"
    lines = {l.split(":")[0]: l.split(":")[1].strip() for l in out.splitlines() if ":" in l}
    assert lines["Average NG per block"] == "%.2f" % (sum(e["ref"]["ng"]) / n)
    assert lines["Average iterations per block"] == "%.2f" % (sum(e["ref"]["iterations"]) / n)
    assert lines["Average NG_p per block"] == "%.2f" % (sum(e["ref"]["ng_p"]) / n)
    e["flow_binary_stdout"] = [l for l in out.splitlines() if not l.startswith("Total CPU time")]
    print("flow binary agrees with the harness on", name)

    # per-line known answers
    rng = np.random.default_rng(7)
    _, cubes = gen(SETS[1][1], 8, SETS[1][3])
    lines = kat_lines(rng, cubes)
    dp = np.ctypeslib.ndpointer(np.float64, flags="C")
    kat = {"llr": lines}
    runs = [(3, UINT64_MAX, "L3"), (1, UINT64_MAX, "L1"), (4, UINT64_MAX, "L4")]
    runs += [(3, t, f"T{t}") for t in KAT_TMAX]
    # tag "<run>_..." from the reference with glibc, "<run>_cr_..." from it
    # under a correctly rounded exp/log
    runs = [(L, t, tag, REF_SO) for L, t, tag in runs] + [(L, t, tag + "_cr", REF_CR_SO) for L, t, tag in runs]
    for L, tmax, tag, so in runs:
        ref = C.CDLL(so)
        ref.sgref_bitso.argtypes = [dp, C.c_int, C.c_uint64, C.c_double, dp, dp, C.POINTER(C.c_int)]
        ref.sgref_line_undefined.argtypes = [dp, C.c_int, C.c_uint64, C.c_double, C.POINTER(C.c_double)]
        lapp = np.zeros_like(lines)
        le = np.zeros_like(lines)
        ng = np.zeros(len(lines), np.int32)
        undef = np.zeros(len(lines), np.int8)
        for i in range(len(lines)):
            a = np.zeros(16)
            b = np.zeros(16)
            k = C.c_int()
            # a line that lists no codeword makes the reference read its
            # uninitialised list size: its soft output is undefined there
            # (only N_guess is), and is recorded as NaN
            undef[i] = ref.sgref_line_undefined(lines[i], L, tmax, THRES, None)
            ref.sgref_bitso(lines[i], L, tmax, THRES, a, b, C.byref(k))
            if undef[i]:
                a[:] = np.nan
                b[:] = np.nan
            lapp[i], le[i], ng[i] = a, b, k.value
        kat[f"{tag}_lapp"], kat[f"{tag}_le"], kat[f"{tag}_nguess"] = lapp, le, ng
        if tmax != UINT64_MAX:
            kat[f"{tag}_undefined"] = undef
            print(f"KAT Tmax={tmax}: {int(undef.sum())} of {len(lines)} lines list no codeword", flush=True)
    np.savez_compressed(os.path.join(OUT_DIR, "kat_lines.npz"), **kat)
    with open(os.path.join(OUT_DIR, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1)
    print("wrote golden.json and kat_lines.npz in %.0fs" % (time.time() - t0))


if __name__ == "__main__":
    main()
