"""sogrand_b200 -- B200-native SOGRAND decoder for the (16,8)^3 cubic product code.

Python face of the C ABI in include/sogrand_b200.h.  Host arrays are numpy;
device arrays are torch CUDA tensors (torch is only the device-memory and
stream plumbing).  The names follow the reference:

  decode(...)       the per-codeword loop of cubic_decoder's main()
                    (SOGRAND_C/cubic_decoder_final.c:119-289)
  bitso(...)        SOGRAND_bitSO (cubic_decoder_final.c:521-585) per line
  decode_file(...)  the cubic_decoder process contract (files + statistics)
  gen_llr / encode  seeded stand-ins for generate_bin, cubic_encoder and
                    channel_sim (the reference's own stages use time(NULL))
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import (SG_CUBE, SG_INFO_BYTES, SG_MAX_PHASES, SgCwStats, SgParams,
                   SgRunSummary, SograndError, check)

__all__ = [
    "SG_CUBE", "SG_INFO_BYTES", "STATS_DTYPE", "SograndError", "params", "reference_alpha",
    "decode", "bitso", "decode_file", "decode_summary", "wilson_interval", "SUMMARY_DTYPE", "channel_sigma", "gen_info", "encode", "gen_llr",
    "set_math_mode", "get_math_mode", "set_wait_limit", "get_wait_limit", "check_device", "version",
]

UINT64_MAX = (1 << 64) - 1

STATS_DTYPE = np.dtype(
    [("iterations", "<f8"), ("ng", "<u8"), ("ng_p", "<u8"), ("converged", "<i4"), ("phases", "<i4")]
)
assert STATS_DTYPE.itemsize == C.sizeof(SgCwStats)


def version() -> str:
    return _lib.load().sg_version().decode()


def reference_alpha(alpha100) -> np.ndarray:
    """Per-phase weights from the reference's alpha[100] indexing: the column
    phase of iteration i uses alpha[2i-2], rows and slices alpha[2i-1]
    (cubic_decoder_final.c:149, :188, :227)."""
    a = np.asarray(alpha100, dtype=np.float64)
    out = np.empty(SG_MAX_PHASES)
    for it in range(1, SG_MAX_PHASES // 3 + 1):
        out[3 * (it - 1) + 0] = a[2 * it - 2]
        out[3 * (it - 1) + 1] = a[2 * it - 1]
        out[3 * (it - 1) + 2] = a[2 * it - 1]
    return out


def params(L: int = 3, Imax: int = 30, Tmax: int = UINT64_MAX, thres: float = 1.0 - 1e-5,
           alpha=None) -> SgParams:
    """Decoder parameters; defaults are the reference's (:94-102).
    alpha: None (0.7 everywhere), a scalar, or one weight per phase."""
    p = SgParams()
    _lib.load().sg_params_default(C.byref(p))
    p.L, p.Imax, p.Tmax, p.thres = int(L), int(Imax), int(Tmax), float(thres)
    if alpha is not None:
        a = np.broadcast_to(np.asarray(alpha, dtype=np.float64), (SG_MAX_PHASES,)) if np.ndim(alpha) == 0 \
            else np.asarray(alpha, dtype=np.float64)
        if a.shape[0] < 3 * p.Imax:
            raise ValueError("alpha needs one weight per phase (3*Imax)")
        for i in range(min(SG_MAX_PHASES, a.shape[0])):
            p.alpha[i] = float(a[i])
    return p


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(a) -> int | None:
    if a is None:
        return None
    if _is_torch(a):
        return a.data_ptr()
    return a.ctypes.data


def decode(llr, p: SgParams | None = None, want_lapp: bool = False, stream=None):
    """Decode LLR cubes.

    llr: float64 array of n_cw*4096 values, numpy (host) or a CUDA torch
    tensor (device, asynchronous on `stream`, default torch's current).
    Returns (bits [n_cw, 64] uint8, stats [n_cw] STATS_DTYPE or uint8 view,
    lapp [n_cw, 4096] or None)."""
    p = p or params()
    lib = _lib.load()
    if _is_torch(llr):
        import torch

        assert llr.is_cuda and llr.dtype == torch.float64 and llr.is_contiguous()
        n = llr.numel() // SG_CUBE
        bits = torch.empty((n, SG_INFO_BYTES), dtype=torch.uint8, device=llr.device)
        stats = torch.empty((n, STATS_DTYPE.itemsize), dtype=torch.uint8, device=llr.device)
        lapp = torch.empty((n, SG_CUBE), dtype=torch.float64, device=llr.device) if want_lapp else None
        s = stream if stream is not None else torch.cuda.current_stream(llr.device).cuda_stream
        check(lib.sg_decode_device(_ptr(llr), n, C.byref(p), _ptr(bits), _ptr(lapp), _ptr(stats), s))
        return bits, stats, lapp
    llr = np.ascontiguousarray(llr, dtype=np.float64)
    n = llr.size // SG_CUBE
    bits = np.zeros((n, SG_INFO_BYTES), np.uint8)
    stats = np.zeros(n, STATS_DTYPE)
    lapp = np.zeros((n, SG_CUBE)) if want_lapp else None
    check(lib.sg_decode_host(_ptr(llr), n, C.byref(p), _ptr(bits), _ptr(lapp), _ptr(stats)))
    return bits, stats, lapp


def stats_from_device(raw) -> np.ndarray:
    """Convert the uint8 view returned for device decodes to STATS_DTYPE."""
    return np.frombuffer(raw.cpu().numpy().tobytes(), dtype=STATS_DTYPE)


def bitso(llr_lines, L: int = 3, Tmax: int = UINT64_MAX, thres: float = 1.0 - 1e-5):
    """SOGRAND_bitSO on [n_lines, 16] LLRs (host numpy).
    Returns (L_APP, L_E, N_guess, codewords found)."""
    v = np.ascontiguousarray(llr_lines, dtype=np.float64).reshape(-1, 16)
    n = v.shape[0]
    lapp = np.zeros_like(v)
    le = np.zeros_like(v)
    ng = np.zeros(n, np.int32)
    nc = np.zeros(n, np.int32)
    check(_lib.load().sg_bitso_host(_ptr(v), n, int(L), int(Tmax), float(thres), _ptr(lapp), _ptr(le),
                                    _ptr(ng), _ptr(nc)))
    return lapp, le, ng, nc


def decode_file(in_path: str, out_path: str, p: SgParams | None = None, chunk_cw: int = 0) -> dict:
    p = p or params()
    s = SgRunSummary()
    check(_lib.load().sg_decode_file(in_path.encode(), out_path.encode(), C.byref(p), chunk_cw, C.byref(s)))
    return {k: getattr(s, k) for k, _ in SgRunSummary._fields_}


SUMMARY_DTYPE = np.dtype([("blocks", "<u8"), ("converged", "<u8"), ("nonfinite", "<u8"), ("total_ng", "<u8"),
                          ("total_ng_p", "<u8"), ("bits_compared", "<u8"), ("bit_errors", "<u8"),
                          ("block_errors", "<u8"), ("total_iterations", "<f8"), ("timeouts", "<u8"),
                          ("device_error", "<u4"), ("reserved", "<u4")])


def decode_summary(llr, p: SgParams | None = None, ref_info=None, want_bits: bool = False, stream=None):
    """Decode CUDA-resident cubes and reduce on the device: returns
    (summary dict, bits or None).  ref_info (CUDA uint8 [n, 64]) adds the
    comparator's bit/block error counts."""
    import torch

    p = p or params()
    n = llr.numel() // SG_CUBE
    dev = llr.device
    summ = torch.zeros(SUMMARY_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    bits = torch.empty((n, SG_INFO_BYTES), dtype=torch.uint8, device=dev) if want_bits else None
    s = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    check(_lib.load().sg_decode_summary_device(_ptr(llr), n, C.byref(p), _ptr(ref_info), _ptr(bits), _ptr(summ), s))
    rec = np.frombuffer(summ.cpu().numpy().tobytes(), dtype=SUMMARY_DTYPE)[0]
    return {k: rec[k].item() for k in SUMMARY_DTYPE.names}, bits


def set_wait_limit(limit: int) -> None:
    """Polls / idle rounds before a device-side wait gives up, for launches
    made after the call (process-wide; default and maximum 2^22)."""
    check(_lib.load().sg_set_wait_limit(int(limit)))


def get_wait_limit() -> int:
    return int(_lib.load().sg_get_wait_limit())


def check_device(stream=None) -> None:
    """Synchronise `stream` and raise SograndError(SG_ERR_TIMEOUT) if a
    bounded wait of a plain-decoder kernel gave up on the current device
    since the last check (the flag is cleared)."""
    check(_lib.load().sg_check_device(stream))


def set_math_mode(mode: int) -> None:
    """0: table-driven exp/log (default, fastest); 1: correctly rounded
    exp/log, bit-exact with the reference under a correctly rounded libm.
    Process-wide, for launches made after the call."""
    check(_lib.load().sg_set_math_mode(int(mode)))


def get_math_mode() -> int:
    return int(_lib.load().sg_get_math_mode())


def wilson_interval(k: int, n: int, conf_z: float = 1.959963984540054) -> tuple[float, float]:
    """95% (default) Wilson score interval of the rate k/n."""
    lo, hi = C.c_double(), C.c_double()
    check(_lib.load().sg_wilson_interval(int(k), int(n), float(conf_z), C.byref(lo), C.byref(hi)))
    return lo.value, hi.value


def channel_sigma(ebn0_db: float) -> float:
    """Noise deviation of channel_sim.c:34-39 (cubic code, R = 1/8)."""
    return _lib.load().sg_channel_sigma(float(ebn0_db))


def gen_info(seed: int, cw0: int, n_cw: int) -> np.ndarray:
    out = np.zeros((n_cw, SG_INFO_BYTES), np.uint8)
    check(_lib.load().sg_gen_info_host(seed, cw0, n_cw, _ptr(out)))
    return out


def encode(info) -> np.ndarray:
    """(16,8)^3 systematic encoding: [n, 64] packed info -> [n, 4096] 0/1."""
    info = np.ascontiguousarray(info, dtype=np.uint8).reshape(-1, SG_INFO_BYTES)
    out = np.zeros((info.shape[0], SG_CUBE), np.uint8)
    check(_lib.load().sg_encode_host(_ptr(info), info.shape[0], _ptr(out)))
    return out


def gen_llr(seed: int, cw0: int, n_cw: int, ebn0_db: float | None = None,
            ebn0_range: tuple[float, float] | None = None, device=None, stream=None):
    """Synthetic channel output for codewords [cw0, cw0+n_cw) of stream `seed`.

    Fixed Eb/N0 (the reference's sigma formula) or per-codeword Eb/N0 drawn
    uniformly from ebn0_range.  device=None -> numpy on the host; else a
    torch device -> CUDA tensors generated on the GPU (identical values).
    Returns (info [n, 64] uint8, llr [n, 4096] float64)."""
    if (ebn0_db is None) == (ebn0_range is None):
        raise ValueError("give exactly one of ebn0_db and ebn0_range")
    sigma = channel_sigma(ebn0_db) if ebn0_db is not None else 0.0
    lo, hi = ebn0_range if ebn0_range is not None else (0.0, 0.0)
    lib = _lib.load()
    if device is None:
        info = np.zeros((n_cw, SG_INFO_BYTES), np.uint8)
        llr = np.zeros((n_cw, SG_CUBE))
        check(lib.sg_gen_llr_host(seed, cw0, n_cw, sigma, lo, hi, _ptr(info), _ptr(llr)))
        return info, llr
    import torch

    info = torch.empty((n_cw, SG_INFO_BYTES), dtype=torch.uint8, device=device)
    llr = torch.empty((n_cw, SG_CUBE), dtype=torch.float64, device=device)
    s = stream if stream is not None else torch.cuda.current_stream(info.device).cuda_stream
    check(lib.sg_gen_llr_device(seed, cw0, n_cw, sigma, lo, hi, _ptr(info), _ptr(llr), s))
    return info, llr
