"""The allocation-free entry point, sg_decode_summary_device_noalloc.

It serves callers that cannot allocate device memory (their allocator is
owned by another component, or all device memory is budgeted at start-up):
every byte it uses beyond the caller's inputs and outputs is static in the
library.  Its results must equal those of sg_decode_summary_device, the
regular entry point, on the same inputs -- here compared exactly (integer
counts, and iteration sums that are exact multiples of 0.5) on two calls in
a row, so that state left in the shared static scratch by the first call
cannot leak into the second.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from sogrand_b200 import _lib

pytestmark = pytest.mark.gpu


def _summary(raw, sg):
    return np.frombuffer(raw.cpu().numpy().tobytes(), dtype=sg.SUMMARY_DTYPE)[0]


def test_noalloc_matches_regular_entry_twice(cuda, sg, golden):
    torch = cuda
    lib = _lib.load()
    e = golden["sets"]["snr_1.5dB"]
    n = e["n_cw"]
    info, llr = sg.gen_llr(e["seed"], 0, n, ebn0_db=e["ebn0_db"])
    d_llr = torch.from_numpy(llr).cuda()
    d_ref = torch.from_numpy(info).cuda()
    p = sg.params()
    stream = torch.cuda.current_stream().cuda_stream

    ref_sum = torch.zeros(sg.SUMMARY_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    ref_bits = torch.empty((n, 64), dtype=torch.uint8, device="cuda")
    assert lib.sg_decode_summary_device(d_llr.data_ptr(), n, C.byref(p), d_ref.data_ptr(), ref_bits.data_ptr(),
                                        ref_sum.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    expect = _summary(ref_sum, sg)
    assert expect["bit_errors"] > 0  # a noisy point, so the error counts are exercised

    for call in range(2):
        out_sum = torch.full((sg.SUMMARY_DTYPE.itemsize,), 0xAB, dtype=torch.uint8, device="cuda")
        out_bits = torch.empty((n, 64), dtype=torch.uint8, device="cuda")
        st = lib.sg_decode_summary_device_noalloc(d_llr.data_ptr(), n, C.byref(p), d_ref.data_ptr(),
                                                  out_bits.data_ptr(), out_sum.data_ptr(), stream)
        assert st == 0, lib.sg_last_error()
        torch.cuda.synchronize()
        assert _summary(out_sum, sg) == expect, call
        assert torch.equal(out_bits, ref_bits), call
    # without caller bits the decoded bits stay in the static scratch
    out_sum = torch.zeros(sg.SUMMARY_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    assert lib.sg_decode_summary_device_noalloc(d_llr.data_ptr(), n, C.byref(p), d_ref.data_ptr(), None,
                                                out_sum.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    assert _summary(out_sum, sg) == expect


def test_noalloc_tables_on_high_ic_lines(cuda, sg):
    """The allocation-free entry point decodes with its own copy of the
    pattern-order tables, built on the device.  Cubes whose LLR magnitudes
    are large and of several spreads give lines with reliability shifts (IC)
    from about 5 to over 100, and 1% flipped signs make those lines search
    deep into their tables; both entry points must agree, through the
    summaries, the bits and the total guess count."""
    torch = cuda
    lib = _lib.load()
    rng = np.random.default_rng(31337)
    code = sg.encode(sg.gen_info(31337, 0, 96)).astype(np.float64)
    spread = np.repeat([2.0, 6.0, 12.0, 24.0], 24)[:, None]
    mag = rng.uniform(12.0, 30.0, (96, 1)) + rng.uniform(0.0, 1.0, code.shape) * spread
    llr = (1.0 - 2.0 * code) * mag
    flip = rng.random(code.shape) < 0.01
    llr[flip] = -llr[flip]
    llr = np.ascontiguousarray(llr)
    d_llr = torch.from_numpy(llr).cuda()
    n = llr.shape[0]
    p = sg.params()
    want = torch.zeros(sg.SUMMARY_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    want_bits = torch.empty((n, 64), dtype=torch.uint8, device="cuda")
    assert lib.sg_decode_summary_device(d_llr.data_ptr(), n, C.byref(p), None, want_bits.data_ptr(),
                                        want.data_ptr(), None) == 0
    got = torch.zeros(sg.SUMMARY_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    got_bits = torch.empty((n, 64), dtype=torch.uint8, device="cuda")
    assert lib.sg_decode_summary_device_noalloc(d_llr.data_ptr(), n, C.byref(p), None, got_bits.data_ptr(),
                                                got.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert _summary(got, sg) == _summary(want, sg)
    assert torch.equal(got_bits, want_bits)
    _, st, _ = sg.decode(llr)  # host entry point, regular tables
    assert _summary(got, sg)["total_ng"] == int(st["ng"].sum())


def test_noalloc_rejects_oversize(cuda, sg):
    lib = _lib.load()
    p = sg.params()
    st = lib.sg_decode_summary_device_noalloc(None, 16385, C.byref(p), None, None, None, None)
    assert st == 1
    st = lib.sg_decode_summary_device_noalloc(None, 16385, C.byref(p), None, None, 8, None)
    assert st == 1 and b"SG_NOALLOC_MAX_CW" in lib.sg_last_error()
