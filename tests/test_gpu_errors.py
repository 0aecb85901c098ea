"""Bounded device-side waits that give up are reported, and leave the GPU
usable.

The waits are made to run out by setting the wait limit to 0 (nothing is
broken on the device: the bulk copies and the work all complete; the kernels
only stop waiting for them).  Every test restores the default limit and
checks that a normal decode afterwards is exact."""
import ctypes as C

import numpy as np
import pytest

from sogrand_b200 import _lib

pytestmark = pytest.mark.gpu

SG_ERR_TIMEOUT = 6


@pytest.fixture
def limit0(sg):
    lib = _lib.load()
    default = lib.sg_get_wait_limit()
    assert default == 1 << 22
    v0 = lib.sg_decoder_get_variant()
    lib.sg_set_wait_limit(0)
    yield lib
    lib.sg_set_wait_limit(default)
    lib.sg_decoder_set_variant(v0)
    lib.sg_check_device(None)  # clear any flag a failed test left behind


def _variant(lib, name):
    for v in range(lib.sg_decoder_variant_count()):
        if lib.sg_decoder_variant_name(v).decode() == name:
            return v
    raise KeyError(name)


def _cubes(sg, golden, n=6):
    e = golden["sets"]["cfg1_2dB_100"]
    info, llr = sg.gen_llr(e["seed"], 0, n, ebn0_db=e["ebn0_db"])
    return e, info, llr


def test_bulk_copy_wait_gives_up_and_reports(cuda, sg, golden, limit0):
    torch, lib = cuda, limit0
    e, info, llr = _cubes(sg, golden)
    n = llr.shape[0]
    assert lib.sg_check_device(None) == 0  # no flag from earlier work
    lib.sg_decoder_set_variant(_variant(lib, "w8-smem"))  # stages the channel cube by bulk copy
    d_llr = torch.from_numpy(llr).cuda()
    assert d_llr.data_ptr() % 16 == 0
    bits, stats, _ = sg.decode(d_llr)
    torch.cuda.synchronize()
    st = sg.stats_from_device(stats)
    assert (st["converged"] == -2).all() and (st["phases"] == 0).all()
    assert not bits.any().item()
    assert lib.sg_check_device(None) == SG_ERR_TIMEOUT
    assert b"converged = -2" in lib.sg_last_error()
    assert lib.sg_check_device(None) == 0  # read and cleared

    # the summary reports the codewords that were not decoded
    summ, _ = sg.decode_summary(d_llr, ref_info=torch.from_numpy(info).cuda())
    assert summ["timeouts"] == n and summ["nonfinite"] == 0 and summ["converged"] == 0
    assert summ["device_error"] & 1
    assert lib.sg_check_device(None) == SG_ERR_TIMEOUT

    # the allocation-free entry point reports its own call's flags
    p = sg.params()
    raw = torch.zeros(sg.SUMMARY_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    assert lib.sg_decode_summary_device_noalloc(d_llr.data_ptr(), n, C.byref(p), None, None, raw.data_ptr(),
                                                None) == 0
    torch.cuda.synchronize()
    rec = np.frombuffer(raw.cpu().numpy().tobytes(), dtype=sg.SUMMARY_DTYPE)[0]
    assert rec["timeouts"] == n and rec["device_error"] & 1 and rec["blocks"] == n

    # the default limit restores exact decoding on the same context
    lib.sg_set_wait_limit(1 << 22)
    bits, stats, _ = sg.decode(d_llr)
    torch.cuda.synchronize()
    st = sg.stats_from_device(stats)
    b = bits.cpu().numpy()
    for i in range(n):
        assert b[i].tobytes().hex() == e["ref"]["bits"][i]
        assert (st["iterations"][i], int(st["ng"][i])) == (e["twin"]["iterations"][i], e["twin"]["ng"][i])
    assert lib.sg_check_device(None) == 0
    rec_ok = torch.zeros(sg.SUMMARY_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    assert lib.sg_decode_summary_device_noalloc(d_llr.data_ptr(), n, C.byref(p), None, None, rec_ok.data_ptr(),
                                                None) == 0
    torch.cuda.synchronize()
    rec = np.frombuffer(rec_ok.cpu().numpy().tobytes(), dtype=sg.SUMMARY_DTYPE)[0]
    assert rec["timeouts"] == 0 and rec["device_error"] == 0 and rec["total_ng"] == sum(e["twin"]["ng"][:n])


def test_persistent_idle_wait_gives_up_and_batch_completes(cuda, sg, golden, limit0):
    torch, lib = cuda, limit0
    e, info, llr = _cubes(sg, golden, n=8)
    n = llr.shape[0]
    d_llr = torch.from_numpy(llr).cuda()
    bits = torch.zeros((n, 64), dtype=torch.uint8, device="cuda")
    stats = torch.zeros((n, 32), dtype=torch.uint8, device="cuda")
    h = C.c_void_p()
    assert lib.sg_batch_create(C.byref(h)) == 0
    try:
        p = sg.params()
        assert lib.sg_batch_decode(h, d_llr.data_ptr(), n, C.byref(p), bits.data_ptr(), None, stats.data_ptr(),
                                   None) == 0
        torch.cuda.synchronize()
        # idle warps gave up, the warps holding lines finished the batch
        assert lib.sg_batch_check(h) == SG_ERR_TIMEOUT
        b = bits.cpu().numpy()
        st = sg.stats_from_device(stats)
        for i in range(n):
            assert b[i].tobytes().hex() == e["ref"]["bits"][i]
            assert int(st["ng"][i]) == e["twin"]["ng"][i]
        lib.sg_set_wait_limit(1 << 22)
        assert lib.sg_batch_decode(h, d_llr.data_ptr(), n, C.byref(p), bits.data_ptr(), None, stats.data_ptr(),
                                   None) == 0
        torch.cuda.synchronize()
        assert lib.sg_batch_check(h) == 0
    finally:
        lib.sg_batch_destroy(h)


def test_host_pipeline_reports_timeout(cuda, sg, golden, limit0):
    lib = limit0
    e, info, llr = _cubes(sg, golden, n=4)
    with pytest.raises(sg.SograndError) as ex:
        sg.decode(llr)
    assert ex.value.status == SG_ERR_TIMEOUT
    lib.sg_set_wait_limit(1 << 22)
    bits, st, _ = sg.decode(llr)
    assert [b.tobytes().hex() for b in bits] == e["ref"]["bits"][:4]
