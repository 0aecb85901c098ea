"""Benchmark of the B200 SOGRAND cubic decoder (one JSON line on rank 0).

Workload (the 2.0 dB point of the "plain method at scale" configuration):
100,000 codewords of the (16,8)^3 cubic product code per GPU, i.i.d. info
bits, BPSK over AWGN at Eb/N0 = 2.0 dB (sigma of channel_sim.c), float64 LLR
cubes generated on the device by the seeded generator; L = 3, Imax = 30,
Tmax = UINT64_MAX.  A step decodes the whole batch.  The 3.3 GB of LLRs per
GPU are larger than L2, so no flush is needed between steps.

  value  codewords/s over all ranks, inputs resident in HBM, timed with CUDA
         events on the decode stream, max over ranks
  e2e    the same through the public C ABI with host buffers
         (sg_decode_host: pinned host LLRs in, bits + statistics out)

`--impl reference` times the reference's own CPU decoder
(SOGRAND_C/cubic_decoder_final.c built from its sources into oracle/_ref,
else the oracle restatement) on all host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "codewords/s & info Mb/s on 1 B200 at Eb/N0 2 dB, BER-matched vs plain & CPU"
UNIT = "codewords/s"
SEED = 20260101
EBN0 = 2.0
# bytes per codeword the decode must move: 4096 float64 in, 64 bytes of bits out
ALG_BYTES_PER_CW = 4096 * 8 + 64
# the reference's published decoder throughput at Eb/N0 2 dB: its CUDA decoder
# on an RTX 4070 Laptop GPU, 1000 codewords in 75.8 s (reference README.md:137-143)
PUBLISHED_CW_PER_S = 13.19
# DRAM bytes (read + write) per codeword of the decode kernel, from one ncu
# capture of 2368 codewords at 2 dB (profiles/): traffic grows with the
# codewords a launch decodes (the cubes are read once), so a full launch's
# traffic is this times its codewords.
DRAM_BYTES_PER_CW = {"batch": (78.752e6 + 2.577e6) / 2368, "plain": (78.98e6 + 1.63e6) / 2368}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons = [], [], set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names[1:], f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def ref_inputs(td, n):
    """LLR files for the CPU legs: codewords [0, n) of the bench stream, one
    file per codeword.  They are made by the twin oracle's build of the
    library's generator (bit-identical to sogrand_b200.gen_llr), so the
    process timing the reference never loads the library."""
    lib = C.CDLL(os.path.join(ROOT, "oracle", "libsg_oracle_twin.so"))
    lib.sgo_gen_llr.argtypes = [C.c_uint64, C.c_uint64, C.c_size_t, C.c_double, C.c_void_p, C.c_void_p]
    lib.sgo_sigma.restype = C.c_double
    lib.sgo_sigma.argtypes = [C.c_double]
    sigma = lib.sgo_sigma(EBN0)
    files = []
    llr = np.zeros(4096)
    for c in range(n):
        lib.sgo_gen_llr(SEED, c, 1, sigma, None, llr.ctypes.data)
        f = os.path.join(td, f"cw{c}.bin")
        llr.tofile(f)
        files.append(f)
    return files


def ref_kind():
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "cubic_decoder_final_O2")
    return ("reference", ref_bin) if os.path.exists(ref_bin) else ("port", None)


def run_queue(files, workers, kind, ref_bin):
    """Decode every file with `workers` concurrent decoders, each taking the
    next codeword from a shared queue as soon as it is free (no core waits
    on a fixed shard while others idle).  Returns the wall time."""
    nxt = iter(files)
    lock = threading.Lock()
    failed = []

    def worker():
        while True:
            with lock:
                f = next(nxt, None)
            if f is None:
                return
            if kind == "reference":
                rc = subprocess.run([ref_bin, f, f + ".dec"], stdout=subprocess.DEVNULL).returncode
            else:
                rc = subprocess.run([sys.executable, __file__, "--port-worker", f]).returncode
            if rc != 0:
                failed.append(f)

    t0 = time.perf_counter()
    th = [threading.Thread(target=worker) for _ in range(workers)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    dt = time.perf_counter() - t0
    if failed:
        raise RuntimeError(f"CPU decoder failed on {failed[:3]}")
    return dt


def cpu_sample_text(kind, n, per_core, cores):
    who = ("an unmodified cubic_decoder_final process (reference source built at -O2)" if kind == "reference"
           else "the oracle restatement")
    return (f"{n} codewords per step ({per_core} per core) at {EBN0} dB; {cores} workers take one codeword "
            f"at a time from a shared queue, each decoded by {who}")


def run_reference(args, rank, world):
    """CPU reference arm: rank 0 times the reference decoder on all host
    cores; the other ranks exit without work."""
    if rank != 0:
        return
    cores = len(os.sched_getaffinity(0))
    per_core = args.ref_cw_per_core
    kind, ref_bin = ref_kind()
    n = cores * per_core
    with tempfile.TemporaryDirectory() as td:
        files = ref_inputs(td, n)
        # warm-up steps (page in the binary and the inputs) decode one
        # codeword per worker; the timed steps decode the whole sample
        for _ in range(args.warmup):
            run_queue(files[:cores], cores, kind, ref_bin)
        times = [run_queue(files, cores, kind, ref_bin) for _ in range(args.steps)]
    value = n / statistics.mean(times)
    sample = cpu_sample_text(kind, n, per_core, cores)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * statistics.mean(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(args, args.n_cw, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "info_mbps": value * 512 / 1e6,
        "step_seconds": {"min": min(times), "max": max(times)},
    }
    print(json.dumps(line), flush=True)


def port_worker(path):
    """Decode one LLR file with the oracle restatement (CPU legs, used only
    when the reference could not be built)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_api import Oracle

    llr = np.fromfile(path)
    Oracle(os.path.join(ROOT, "oracle", "libsg_oracle.so")).decode(llr)


def cpu_baseline(args):
    """Bounded CPU sample on the host cores, the same measurement as the
    reference arm's step."""
    cores = len(os.sched_getaffinity(0))
    per_core = args.cpu_cw_per_core
    kind, ref_bin = ref_kind()
    n = cores * per_core
    with tempfile.TemporaryDirectory() as td:
        files = ref_inputs(td, n)
        dt = run_queue(files, cores, kind, ref_bin)
    return {"value": n / dt, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": cpu_sample_text(kind, n, per_core, cores) + f"; {dt:.1f} s wall"}


_REF_LIB = None


def _ref_harness_decode(args):
    """Pool worker: one codeword through the reference's own functions
    (oracle/_ref/libsgref.so, glibc libm) at the given Tmax; returns the
    packed bits and whether a line decode read the reference's
    uninitialised list size (possible only under a finite Tmax; the
    reference's output is undefined then).  The check runs each line's
    search once more, so it is done only when Tmax is finite."""
    global _REF_LIB
    llr, tmax = args
    if _REF_LIB is None:
        _REF_LIB = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libsgref.so"))
        dp = np.ctypeslib.ndpointer(np.float64, flags="C")
        u8 = np.ctypeslib.ndpointer(np.uint8, flags="C")
        i32 = np.ctypeslib.ndpointer(np.int32, flags="C")
        _REF_LIB.sgref_decode.argtypes = [dp, C.c_size_t, C.c_int, C.c_int, C.c_uint64, C.c_double, dp, u8,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _REF_LIB.sgref_decode_checked.argtypes = [dp, C.c_size_t, C.c_int, C.c_int, C.c_uint64, C.c_double, dp,
                                                  u8, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                  i32]
    bits = np.zeros(64, np.uint8)
    und = np.zeros(1, np.int32)
    if tmax == (1 << 64) - 1:
        _REF_LIB.sgref_decode(np.ascontiguousarray(llr), 1, 3, 30, tmax, 1.0 - 1e-5, np.full(100, 0.7), bits,
                              None, None, None, None, None)
    else:
        _REF_LIB.sgref_decode_checked(np.ascontiguousarray(llr), 1, 3, 30, tmax, 1.0 - 1e-5, np.full(100, 0.7),
                                      bits, None, None, None, None, None, und)
    return bits, int(und[0])


def run_sweep(args):
    """Eb/N0 sweep of the plain method at scale: per point and Tmax, the GPU
    decode-and-compare of n codewords (codewords/s, BER with 95% interval,
    iterations, NG; sogrand_b200.sweep) and, beside it, the reference's own
    decoder on all host cores over the first cores x cpu_cw_per_core
    codewords of the same stream (one codeword per task from a shared
    queue), with its decoded bits checked against the GPU's."""
    import multiprocessing as mp

    import torch

    import sogrand_b200 as sg
    from sogrand_b200.sweep import parse_points, sweep

    torch.cuda.set_device(0)
    cores = len(os.sched_getaffinity(0))
    n_cpu = cores * args.cpu_cw_per_core
    points = parse_points(args.ebn0)
    tmaxes = [(1 << 64) - 1 if t == "inf" else int(t) for t in args.tmax.split(",")]
    have_ref = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libsgref.so"))
    rows = []
    with mp.get_context("spawn").Pool(cores) as pool:
        for tmax in tmaxes:
            p = sg.params(Tmax=tmax)
            for eb in points:
                row = sweep([eb], args.n_cw, seed=args.seed, params=p)[0]
                row["tmax"] = "inf" if tmax == (1 << 64) - 1 else tmax
                if have_ref and n_cpu > 0:
                    _, llr = sg.gen_llr(args.seed, 0, n_cpu, ebn0_db=eb)
                    gbits, _, _ = sg.decode(llr, p)
                    t0 = time.perf_counter()
                    res = pool.map(_ref_harness_decode, [(llr[i], tmax) for i in range(n_cpu)], chunksize=1)
                    dt = time.perf_counter() - t0
                    und = [r[1] > 0 for r in res]
                    row["cpu_reference"] = {
                        "codewords_per_s": n_cpu / dt, "codewords": n_cpu, "cores": cores,
                        "how": "reference functions (oracle/_ref/libsgref.so, -O2, glibc), one codeword per "
                               "task from a shared queue over all host cores"
                               + ("" if tmax == (1 << 64) - 1 else "; each line's search run twice to detect "
                                  "the reference's undefined (uninitialised list size) lines, so the rate is "
                                  "understated"),
                        "codewords_undefined_in_reference": int(sum(und)),
                        "defined_codewords_with_bits_differing_from_gpu": int(sum(
                            not np.array_equal(r[0], b) for r, b, u in zip(res, gbits, und) if not u))}
                rows.append(row)
                c = row.get("cpu_reference", {})
                print(f"Tmax {row['tmax']:>5} {eb:5.2f} dB  GPU {row['codewords_per_s']:9.0f} cw/s  "
                      f"BER {row['ber']:.3e}  it {row['avg_iterations']:5.2f}  NG {row['ng_per_codeword']:9.0f}  "
                      f"CPU {c.get('codewords_per_s', 0):7.2f} cw/s (undefined {c.get('codewords_undefined_in_reference')}, "
                      f"differing {c.get('defined_codewords_with_bits_differing_from_gpu')})", flush=True)
    print(json.dumps({"sweep": rows}), flush=True)


def run_ref_gpu(args):
    """The reference's own GPU decoder (SOGRAND_CUDA/cubic_decoder1.cu built
    unmodified for sm_100a into oracle/_ref) on this GPU, beside this
    library on the same codewords: the first n codewords of the bench
    stream at 2 dB as one LLR file.  Reports both decoders' device-timed
    codewords/s (the reference's own "Total GPU time" line, which brackets
    its kernel launches with CUDA events; this library's sg_decode_device
    with CUDA events) and how many codewords' decoded bits differ."""
    import torch

    import sogrand_b200 as sg
    from sogrand_b200 import autotune

    exe = os.path.join(ROOT, "oracle", "_ref", "cubic_decoder1_sm100a")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference_gpu", "unavailable": "oracle/_ref/cubic_decoder1_sm100a not built"}))
        return
    n = args.ref_gpu_cw
    _, llr = sg.gen_llr(SEED, 0, n, ebn0_db=EBN0)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "llr.bin"), os.path.join(td, "dec.bin")
        llr.tofile(fin)
        t0 = time.perf_counter()
        out = subprocess.run([exe, fin, fout], capture_output=True, text=True, timeout=1800)
        wall = time.perf_counter() - t0
        if out.returncode != 0:
            print(json.dumps({"impl": "reference_gpu", "unavailable": f"exit {out.returncode}: "
                              + out.stderr.strip()[-200:]}))
            return
        lines = {l.split(":")[0].strip(): l.split(":", 1)[1].strip() for l in out.stdout.splitlines() if ":" in l}
        ref_bits = np.fromfile(fout, np.uint8).reshape(n, 64)
    gpu_s = float(lines["Total GPU time"].split()[0])
    torch.cuda.set_device(0)
    d = torch.from_numpy(llr).cuda()
    sg.decode(d)  # warm-up
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    bits, _, _ = sg.decode(d)
    e1.record()
    torch.cuda.synchronize()
    ours = e0.elapsed_time(e1) / 1000.0
    bits = bits.cpu().numpy()
    print(json.dumps({
        "impl": "reference_gpu", "codewords": n, "ebn0_db": EBN0,
        "reference_gpu": {"codewords_per_s": n / gpu_s, "gpu_seconds": gpu_s, "process_wall_s": wall,
                          "avg_iterations": float(lines["Average iterations per block"]),
                          "avg_ng": float(lines["Average NG per block"]),
                          "build": "SOGRAND_CUDA/cubic_decoder1.cu, nvcc -O3 -use_fast_math, sm_100a"},
        "this_library": {"codewords_per_s": n / ours, "gpu_seconds": ours, "api": "sg_decode_device",
                         "variant": autotune.get_variant()},
        "speedup": gpu_s / ours,
        "codewords_with_different_bits": int((ref_bits != bits).any(axis=1).sum()),
        "note": "the reference GPU decoder swaps the C decoder's first two phase axes and uses CUDA's "
                "exp/log with FMA contraction, so its results may differ from the C reference's"}), flush=True)


def bench_config(args, n, world):
    return {"workload": f"cubic (16,8)^3 SOGRAND decode, {n} codewords per GPU per step, "
                        + (f"Eb/N0 {EBN0} dB" if args.workload == "2dB" else "Eb/N0 U[1,3] dB per codeword")
                        + ", L=3 Imax=30 Tmax=inf",
            "codewords_per_gpu": n, "ebn0_db": EBN0 if args.workload == "2dB" else [1.0, 3.0],
            "form": args.form, "parallelism": f"replicas{world}",
            "l2": f"inputs ({n * 32768 / 1e9:.1f} GB per GPU) larger than L2; no flush"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sogrand", choices=["sogrand", "reference"])
    ap.add_argument("--n-cw", type=int, default=100000, help="codewords per GPU per step")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-cw-per-core", type=int, default=32)
    ap.add_argument("--ref-cw-per-core", type=int, default=32)
    ap.add_argument("--form", default="batch", choices=["plain", "batch"],
                    help="plain: one CTA per codeword (sg_decode_device); batch: persistent kernel replayed "
                         "from a CUDA graph (sg_batch_*)")
    ap.add_argument("--workload", default="2dB", choices=["2dB", "mixed"],
                    help="2dB: Eb/N0 2.0 dB; mixed: per-codeword Eb/N0 uniform in [1, 3] dB")
    ap.add_argument("--variant", default=None, help="decoder kernel variant (name or index)")
    ap.add_argument("--autotune", action="store_true", help="measure all variants first, keep the fastest")
    ap.add_argument("--sweep", action="store_true",
                    help="instead of the bench line: Eb/N0 x Tmax sweep with a CPU reference column")
    ap.add_argument("--ebn0", default="1.0:3.0:0.25", help="sweep points, a:b:step or a comma list (dB)")
    ap.add_argument("--tmax", default="inf,1000", help="sweep Tmax values, comma list ('inf' = none)")
    ap.add_argument("--seed", type=int, default=20261203, help="sweep stream seed")
    ap.add_argument("--ref-gpu", action="store_true",
                    help="instead of the bench line: the reference's own GPU decoder beside this library")
    ap.add_argument("--ref-gpu-cw", type=int, default=1000)
    ap.add_argument("--math", type=int, default=0, choices=[0, 1],
                    help="math mode: 0 table-driven exp/log, 1 correctly rounded (reference-exact)")
    ap.add_argument("--port-worker", default=None, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.port_worker:
        port_worker(args.port_worker)
        return
    if args.sweep:
        run_sweep(args)
        return
    if args.ref_gpu:
        run_ref_gpu(args)
        return
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch

    import sogrand_b200 as sg
    from sogrand_b200 import _lib

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    from sogrand_b200 import autotune

    from sogrand_b200 import batch as B

    sg.set_math_mode(args.math)

    tune = None
    snr_kw = dict(ebn0_db=EBN0) if args.workload == "2dB" else dict(ebn0_range=(1.0, 3.0))
    if args.variant is not None:
        setv = B.set_variant if args.form == "batch" else autotune.set_variant
        setv(int(args.variant) if args.variant.isdigit() else args.variant)
    elif args.autotune:
        tune = (autotune.autotune_batch if args.form == "batch" else autotune.autotune)(device=local, **snr_kw)
    # every rank decodes its own codeword range of the same stream (no data-path collective)
    from sogrand_b200.replicas import codeword_range, max_over_ranks

    n = args.n_cw
    cw0, _ = codeword_range(rank, world, n_per_rank=n)
    stream = torch.cuda.Stream(dev)
    p = sg.params()
    lib = _lib.load()
    with torch.cuda.stream(stream):
        info, llr = sg.gen_llr(SEED, cw0, n, device=dev, stream=stream.cuda_stream, **snr_kw)
        bits = torch.empty((n, 64), dtype=torch.uint8, device=dev)
        stats = torch.empty((n, sg.STATS_DTYPE.itemsize), dtype=torch.uint8, device=dev)
    stream.synchronize()
    batch = None
    if args.form == "batch":
        batch = B.Batch()
        batch.capture(llr, bits, stats, p, stream=stream.cuda_stream)

    def decode_step():
        if batch is not None:
            batch.replay(stream.cuda_stream)
        else:
            _lib.check(lib.sg_decode_device(llr.data_ptr(), n, C.byref(p), bits.data_ptr(), None,
                                            stats.data_ptr(), stream.cuda_stream))

    for _ in range(args.warmup):
        decode_step()
    stream.synchronize()
    if pg:
        pg.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        decode_step()
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    dt = ev0.elapsed_time(ev1) / 1000.0
    t_max = max_over_ranks(dt, device=dev) if pg else dt
    value = world * n * args.steps / t_max

    # results of the timed run (one step's worth) for the sanity fields
    st = sg.stats_from_device(stats)
    ber = float((np.unpackbits(bits.cpu().numpy()) != np.unpackbits(info.cpu().numpy())).mean())
    ng_per_cw = float(st["ng"].mean())

    # end to end through the public C ABI with pinned host buffers
    e2e = None
    if args.e2e_steps > 0:
        llr_h = torch.empty((n, 4096), dtype=torch.float64, pin_memory=True)
        llr_h.copy_(llr)
        bits_h = torch.empty((n, 64), dtype=torch.uint8, pin_memory=True)
        stats_h = np.zeros(n, sg.STATS_DTYPE)
        del llr
        torch.cuda.empty_cache()
        _lib.check(lib.sg_decode_host(llr_h.data_ptr(), n, C.byref(p), bits_h.data_ptr(), None,
                                      stats_h.ctypes.data))  # warm-up
        if pg:
            pg.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            _lib.check(lib.sg_decode_host(llr_h.data_ptr(), n, C.byref(p), bits_h.data_ptr(), None,
                                          stats_h.ctypes.data))
        e2e_dt = (time.perf_counter() - t0) / args.e2e_steps
        if pg:
            e2e_dt = max_over_ranks(e2e_dt, device=dev)
        e2e = {"value": world * n / e2e_dt, "unit": UNIT, "h2d_bytes_per_step": n * 4096 * 8,
               "d2h_bytes_per_step": n * (64 + sg.STATS_DTYPE.itemsize),
               "api": "sg_decode_host (host buffers, copies inside the timed region)"}

    def best_ceiling(mode, runs=3):
        """The per-guess ceiling is the best rate the GPU reaches: the
        maximum of a few ~20 ms measurements (single ones vary by up to 8 %
        between runs)."""
        v = C.c_double()
        best = 0.0
        for _ in range(runs):
            _lib.check(lib.sg_guess_ceiling(20000, mode, C.byref(v)))
            best = max(best, v.value)
        return C.c_double(best)

    ceil, ceil_other = best_ceiling(args.math), best_ceiling(1 - args.math)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    hbm_peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        hbm_peak, peak_src = json.load(open(peaks_path))["hbm_gbs"], "measured"
    achieved = n * ALG_BYTES_PER_CW / (dt / args.steps) / 1e9
    if pg:
        pg.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": value / PUBLISHED_CW_PER_S if args.workload == "2dB" else None,
            "vs_baseline_basis": f"{PUBLISHED_CW_PER_S} codewords/s, the reference's published GPU decoder "
                                 "figure at 2 dB (RTX 4070 Laptop, reference README.md:137-143)",
            "dtype": "f64", "data": "synthetic",
            "config": bench_config(args, n, world),
            "info_mbps": value * 512 / 1e6,
            "ber": ber, "ng_per_codeword": ng_per_cw, "guesses_per_s": value * ng_per_cw,
            "guess_ceiling": {"bound": "fp64 exp per guess", "achieved": value * ng_per_cw / world,
                              "peak": ceil.value, "unit": "guess/s per GPU",
                              "frac": value * ng_per_cw / world / ceil.value,
                              "how": "sg_guess_ceiling: PM add + exp(-PM) + P_notGuess subtract per guess, "
                                     "all SMs, measured on this GPU in this run (best of 3), with the exp of the math "
                                     "mode used (" + ("table-driven" if args.math == 0 else "correctly rounded")
                                     + ")",
                              "peak_other_math_mode": ceil_other.value},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": DRAM_BYTES_PER_CW[args.form] * n,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of 2368 codewords "
                                           "(profiles/), scaled to this launch's codewords",
                         "note": f"peak {peak_src}; the decoder is FP64/issue-bound, see guesses_per_s"},
            "e2e": e2e, "gpu_launches": args.steps, "clocks": clk,
            "form": args.form, "autotune": tune,
            "math_mode": ("table-driven exp/log (default)" if args.math == 0 else
                          "correctly rounded exp/log (reference-exact)"),
            "variant": B.get_variant() if args.form == "batch" else autotune.get_variant(),
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args)
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
