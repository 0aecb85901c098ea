"""Autotuner of the decoder's kernel configuration.

Every variant of the plain decoder computes bit-identical results; they
differ only in speed, which depends on the codeword mix.  The dimensions:
warps per codeword CTA (8 to 16); the channel cube in shared memory (staged
by a bulk copy) or read from global memory; error patterns per lane per step
(G = 1, 2 or 4); lines per warp (1: 32 lanes per line; 2: 16 lanes per
line, the "-l2-" variants).  autotune() decodes one seeded batch of
the caller's workload with each variant, timed with CUDA events, and selects
the fastest for the process.
"""
from __future__ import annotations

import ctypes as C

from . import _lib


def variants() -> list[str]:
    lib = _lib.load()
    return [lib.sg_decoder_variant_name(v).decode() for v in range(lib.sg_decoder_variant_count())]


def set_variant(v: int | str) -> None:
    names = variants()
    idx = names.index(v) if isinstance(v, str) else int(v)
    _lib.check(_lib.load().sg_decoder_set_variant(idx))


def get_variant() -> str:
    lib = _lib.load()
    return lib.sg_decoder_variant_name(lib.sg_decoder_get_variant()).decode()


def autotune(n_cw: int = 148 * 3 * 20, ebn0_db: float | None = None, ebn0_range=None, seed: int = 1,
             device: int = 0, params=None, repeats: int = 1) -> dict:
    """Measure every variant on n_cw synthetic codewords; select the fastest.
    Returns {variant name: codewords/s} plus "best"."""
    import torch

    import sogrand_b200 as sg

    lib = _lib.load()
    dev = torch.device("cuda", device)
    p = params or sg.params()
    if ebn0_db is None and ebn0_range is None:
        ebn0_db = 2.0
    _, llr = sg.gen_llr(seed, 0, n_cw, ebn0_db=ebn0_db, ebn0_range=ebn0_range, device=dev)
    bits = torch.empty((n_cw, sg.SG_INFO_BYTES), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    res = {}
    for v, name in enumerate(variants()):
        _lib.check(lib.sg_decoder_set_variant(v))
        _lib.check(lib.sg_decode_device(llr.data_ptr(), n_cw, C.byref(p), bits.data_ptr(), None, None,
                                        stream.cuda_stream))  # warm-up
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(repeats):
            _lib.check(lib.sg_decode_device(llr.data_ptr(), n_cw, C.byref(p), bits.data_ptr(), None, None,
                                            stream.cuda_stream))
        e1.record(stream)
        torch.cuda.synchronize(dev)
        res[name] = repeats * n_cw / (e0.elapsed_time(e1) / 1000.0)
    best = max(res, key=res.get)
    set_variant(best)
    res["best"] = best
    return res


def autotune_batch(n_cw: int = 148 * 3 * 20, ebn0_db: float | None = None, ebn0_range=None, seed: int = 1,
                   device: int = 0, params=None) -> dict:
    """Measure every batched (persistent) variant; select the fastest."""
    import torch

    import sogrand_b200 as sg
    from . import batch as B

    lib = _lib.load()
    dev = torch.device("cuda", device)
    if ebn0_db is None and ebn0_range is None:
        ebn0_db = 2.0
    _, llr = sg.gen_llr(seed, 0, n_cw, ebn0_db=ebn0_db, ebn0_range=ebn0_range, device=dev)
    b = B.Batch()
    res = {}
    for v, name in enumerate(B.variants()):
        _lib.check(lib.sg_batch_set_variant(v))
        b.decode(llr, params)  # warm-up
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.current_stream(dev)
        e0.record(stream)
        b.decode(llr, params)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        b.check()
        res[name] = n_cw / (e0.elapsed_time(e1) / 1000.0)
    best = max(res, key=res.get)
    B.set_variant(best)
    b.close()
    res["best"] = best
    return res
