"""Batched persistent decoder (sg_batch_* of the C ABI).

A Batch owns the device work-queue word of the persistent kernel and, after
capture(), a CUDA graph of one whole decode that replay() relaunches.
Outputs are bit-identical to sogrand_b200.decode on the same inputs.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from ._lib import check


def variants() -> list[str]:
    lib = _lib.load()
    return [lib.sg_batch_variant_name(v).decode() for v in range(lib.sg_batch_variant_count())]


def set_variant(v: int | str) -> None:
    idx = variants().index(v) if isinstance(v, str) else int(v)
    check(_lib.load().sg_batch_set_variant(idx))


def get_variant() -> str:
    lib = _lib.load()
    return lib.sg_batch_variant_name(lib.sg_batch_get_variant()).decode()


class Batch:
    def __init__(self):
        self._lib = _lib.load()
        self._h = C.c_void_p()
        check(self._lib.sg_batch_create(C.byref(self._h)))

    def close(self):
        if self._h:
            self._lib.sg_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _stream(dev, stream):
        import torch

        return stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream

    def outputs(self, n: int, device, want_lapp: bool = False):
        import torch

        import sogrand_b200 as sg

        bits = torch.empty((n, sg.SG_INFO_BYTES), dtype=torch.uint8, device=device)
        stats = torch.empty((n, sg.STATS_DTYPE.itemsize), dtype=torch.uint8, device=device)
        lapp = torch.empty((n, sg.SG_CUBE), dtype=torch.float64, device=device) if want_lapp else None
        return bits, stats, lapp

    def decode(self, llr, p=None, want_lapp: bool = False, stream=None):
        """Enqueue one batched decode of CUDA-resident cubes; returns
        (bits, raw stats, lapp or None) as decode() does."""
        import sogrand_b200 as sg

        p = p or sg.params()
        n = llr.numel() // sg.SG_CUBE
        bits, stats, lapp = self.outputs(n, llr.device, want_lapp)
        check(self._lib.sg_batch_decode(self._h, llr.data_ptr(), n, C.byref(p), bits.data_ptr(),
                                        lapp.data_ptr() if lapp is not None else None, stats.data_ptr(),
                                        self._stream(llr.device, stream)))
        return bits, stats, lapp

    def capture(self, llr, bits, stats, p=None, lapp=None, stream=None):
        """Record the decode of `llr` into `bits`/`stats` (and `lapp`) as a
        CUDA graph; the buffers must stay alive while the graph is used."""
        import sogrand_b200 as sg

        p = p or sg.params()
        n = llr.numel() // sg.SG_CUBE
        check(self._lib.sg_batch_capture(self._h, llr.data_ptr(), n, C.byref(p), bits.data_ptr(),
                                         lapp.data_ptr() if lapp is not None else None, stats.data_ptr(),
                                         stream))

    def replay(self, stream=None):
        check(self._lib.sg_batch_replay(self._h, stream))

    def check(self):
        """After completion: raises if a bounded device wait gave up."""
        check(self._lib.sg_batch_check(self._h))
