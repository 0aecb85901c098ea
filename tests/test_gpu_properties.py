"""GPU properties at scale and edge cases of the C ABI (size-independent
checks: round trips, batching invariance, determinism, error paths)."""
import ctypes as C
import hashlib
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_noiseless_round_trip_at_scale(cuda, sg):
    """encode -> BPSK without noise -> decode: with |LLR| = 12 every line's
    hard decision is a codeword whose list confidence already exceeds
    1 - 1e-5, so every codeword stops after the first phase, one guess per
    line."""
    torch = cuda
    n = 20000
    info = sg.gen_info(31, 0, n)
    cw = sg.encode(info)
    llr = torch.from_numpy(np.where(cw == 0, 12.0, -12.0)).cuda()
    bits, raw, _ = sg.decode(llr)
    torch.cuda.synchronize()
    st = sg.stats_from_device(raw)
    assert np.array_equal(bits.cpu().numpy(), info)
    assert np.all(st["iterations"] == 0.5) and np.all(st["ng"] == 256) and np.all(st["converged"] == 1)


def test_device_generator_equals_host(cuda, sg):
    torch = cuda
    for kw in (dict(ebn0_db=2.0), dict(ebn0_range=(1.0, 3.0))):
        hi, hl = sg.gen_llr(99, 1000, 48, **kw)
        di, dl = sg.gen_llr(99, 1000, 48, device="cuda", **kw)
        torch.cuda.synchronize()
        assert np.array_equal(di.cpu().numpy(), hi)
        assert np.array_equal(dl.cpu().numpy().view(np.int64), hl.view(np.int64))


def test_device_generator_unaligned_output(cuda, sg):
    """LLR output that is 8- but not 16-byte aligned takes the generator's
    scalar stores and gives the same values; output that is not 8-byte
    aligned is rejected."""
    from sogrand_b200 import _lib

    torch = cuda
    lib = _lib.load()
    n = 5
    hi, hl = sg.gen_llr(321, 7, n, ebn0_range=(1.0, 3.0))
    buf = torch.zeros(n * 4096 + 2, dtype=torch.float64, device="cuda")
    base = buf.data_ptr()
    assert base % 16 == 0
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.sg_gen_llr_device(321, 7, n, 0.0, 1.0, 3.0, None, base + 8, stream) == 0
    torch.cuda.synchronize()
    got = buf[1:1 + n * 4096].cpu().numpy().reshape(n, 4096)
    assert np.array_equal(got.view(np.int64), hl.view(np.int64))
    assert buf[0].item() == 0.0 and buf[-1].item() == 0.0
    assert lib.sg_gen_llr_device(321, 7, n, 0.0, 1.0, 3.0, None, base + 4, stream) == 1
    assert b"8-byte aligned" in lib.sg_last_error()


def test_device_api_equals_host_api_and_batching(cuda, sg):
    torch = cuda
    _, llr = sg.gen_llr(7, 0, 24, ebn0_db=1.5)
    hb, hs, hl = sg.decode(llr, want_lapp=True)
    db, draw, dl = sg.decode(torch.from_numpy(llr).cuda(), want_lapp=True)
    torch.cuda.synchronize()
    assert np.array_equal(db.cpu().numpy(), hb)
    assert np.array_equal(sg.stats_from_device(draw), hs)
    assert np.array_equal(dl.cpu().numpy().view(np.int64), hl.view(np.int64))
    # any sub-batch decodes the same codewords identically
    for a, b in ((0, 1), (5, 17), (23, 24)):
        sb, ss, _ = sg.decode(llr[a:b])
        assert np.array_equal(sb, hb[a:b]) and np.array_equal(ss, hs[a:b])


def test_unaligned_input_uses_plain_loads(cuda, sg):
    """A cube pointer that is 8- but not 16-byte aligned takes the plain-load
    path and gives the same result."""
    torch = cuda
    _, llr = sg.gen_llr(8, 0, 4, ebn0_db=2.0)
    buf = torch.zeros(4 * 4096 + 1, dtype=torch.float64, device="cuda")
    buf[1:] = torch.from_numpy(llr.ravel()).cuda()
    view = buf[1:]
    assert view.data_ptr() % 16 == 8
    b1, s1, _ = sg.decode(view)
    b2, s2, _ = sg.decode(torch.from_numpy(llr).cuda())
    torch.cuda.synchronize()
    assert torch.equal(b1, b2) and torch.equal(s1, s2)


def test_nonfinite_codeword_is_reported(cuda, sg):
    _, llr = sg.gen_llr(9, 0, 3, ebn0_db=2.5)
    good_b, good_s, _ = sg.decode(llr)
    bad = llr.copy()
    bad[1, 777] = np.nan
    with pytest.raises(sg.SograndError) as e:
        sg.decode(bad)
    assert e.value.status == 3
    from sogrand_b200 import _lib

    lib = _lib.load()
    bits = np.zeros((3, 64), np.uint8)
    st = np.zeros(3, sg.STATS_DTYPE)
    p = sg.params()
    r = lib.sg_decode_host(bad.ctypes.data, 3, C.byref(p), bits.ctypes.data, None, st.ctypes.data)
    assert r == 3
    assert st["converged"][1] == -1 and np.all(bits[1] == 0)
    for i in (0, 2):
        assert np.array_equal(bits[i], good_b[i]) and st[i] == good_s[i]


def test_host_pipeline_matches_device_across_chunks(cuda, sg):
    """sg_decode_host decodes in 16384-codeword chunks on two streams with
    the batched decoder.  Over three chunks (the last one partial) its bits,
    statistics and soft output equal the device entry point's (the plain
    decoder), and a non-finite codeword in the middle chunk is reported
    without disturbing the others."""
    torch = cuda
    from sogrand_b200 import _lib

    n = 2 * 16384 + 1000
    _, dllr = sg.gen_llr(77, 0, n, ebn0_db=2.5, device="cuda")
    db, draw, dl = sg.decode(dllr, want_lapp=True)
    torch.cuda.synchronize()
    llr = dllr.cpu().numpy()
    ref_bits, ref_st, ref_lapp = db.cpu().numpy(), sg.stats_from_device(draw), dl.cpu().numpy()
    del dllr, db, draw, dl
    bad = 20000
    llr[bad, 5] = np.inf
    bits = np.zeros((n, 64), np.uint8)
    st = np.zeros(n, sg.STATS_DTYPE)
    lapp = np.zeros((n, 4096))
    r = _lib.load().sg_decode_host(llr.ctypes.data, n, C.byref(sg.params()), bits.ctypes.data, lapp.ctypes.data,
                                   st.ctypes.data)
    assert r == 3  # SG_ERR_NONFINITE, after decoding the rest
    keep = np.arange(n) != bad
    assert np.array_equal(bits[keep], ref_bits[keep])
    assert np.array_equal(st[keep], ref_st[keep])
    assert np.array_equal(lapp[keep].view(np.int64), ref_lapp[keep].view(np.int64))
    assert st["converged"][bad] == -1 and np.all(bits[bad] == 0)


def test_determinism_and_stats_at_scale(cuda, sg):
    torch = cuda
    n = 4096
    _, llr = sg.gen_llr(2026, 0, n, ebn0_db=2.0, device="cuda")
    b1, s1, _ = sg.decode(llr)
    b2, s2, _ = sg.decode(llr)
    torch.cuda.synchronize()
    assert torch.equal(b1, b2) and torch.equal(s1, s2)
    st = sg.stats_from_device(s1)
    assert 4.0 < st["iterations"].mean() < 6.0
    assert 1.6e6 < st["ng"].mean() < 2.4e6
    assert (st["converged"] == 1).mean() > 0.99


def test_cli_drop_in(cuda, sg, tmp_path):
    """The cubic_decoder CLI: same argv, files and statistics lines as the
    reference decoder process."""
    info, llr = sg.gen_llr(5, 0, 6, ebn0_db=2.0)
    llr.tofile(tmp_path / "llr.bin")
    exe = os.path.join(ROOT, "sogrand_b200", "bin", "cubic_decoder")
    out = subprocess.run([exe, str(tmp_path / "llr.bin"), str(tmp_path / "dec.bin")], check=True,
                         capture_output=True, text=True).stdout.splitlines()
    bits, st, _ = sg.decode(llr)
    assert (tmp_path / "dec.bin").read_bytes() == bits.tobytes()
    assert out[0] == "Decoding complete. 6 block(s) decoded."
    assert out[1] == "Average iterations per block: %.2f" % st["iterations"].mean()
    assert out[2] == "Average NG per block: %.2f" % (st["ng"].sum() / 6)
    assert out[4] == "Average NG_p per block: %.2f" % (st["ng_p"].sum() / 6)
    assert out[-1].startswith("Throughput: ")


def test_file_decoder_chunks_and_edges(cuda, sg, tmp_path):
    """sg_decode_file in small chunks (the reader, both lanes and the in-order
    writes all exercised), with a trailing partial cube (ignored, as the
    reference's fread loop ignores it) and a non-finite cube (reported after
    the rest is decoded); and an empty file."""
    info, llr = sg.gen_llr(8, 0, 40, ebn0_db=2.0)
    llr = llr.copy()
    llr[13, 77] = np.nan
    path = tmp_path / "llr.bin"
    with open(path, "wb") as f:
        f.write(llr.tobytes())
        f.write(b"\0" * 1000)  # partial cube
    want_bits, want_st, _ = sg.decode(np.delete(llr, 13, axis=0))
    for chunk in (7, 16, 0):
        with pytest.raises(sg.SograndError) as ex:
            sg.decode_file(str(path), str(tmp_path / "dec.bin"), chunk_cw=chunk)
        assert ex.value.status == 3  # SG_ERR_NONFINITE
        got = np.frombuffer((tmp_path / "dec.bin").read_bytes(), np.uint8).reshape(-1, 64)
        assert got.shape[0] == 40 and not got[13].any()
        assert np.array_equal(np.delete(got, 13, axis=0), want_bits), chunk
    llr[13, 77] = 0.5
    path.write_bytes(llr.tobytes())
    bits, st, _ = sg.decode(llr)
    s = sg.decode_file(str(path), str(tmp_path / "dec.bin"), chunk_cw=9)
    assert (tmp_path / "dec.bin").read_bytes() == bits.tobytes()
    assert s["blocks"] == 40 and s["total_ng"] == int(st["ng"].sum())
    assert s["total_iterations"] == float(st["iterations"].sum())
    (tmp_path / "empty.bin").write_bytes(b"")
    s = sg.decode_file(str(tmp_path / "empty.bin"), str(tmp_path / "dec.bin"))
    assert s["blocks"] == 0 and (tmp_path / "dec.bin").read_bytes() == b""


def test_guess_ceiling_bounds_the_decoder(cuda, sg):
    """The per-guess arithmetic ceiling is positive and above the decoder's
    own guess rate on the same GPU."""
    import ctypes as C
    import time

    from sogrand_b200 import _lib

    torch = cuda
    lib = _lib.load()
    ceil = C.c_double()
    assert lib.sg_guess_ceiling(2000, 0, C.byref(ceil)) == 0
    tab = C.c_double()
    assert lib.sg_guess_ceiling(2000, 1, C.byref(tab)) == 0 and tab.value > 0
    assert lib.sg_guess_ceiling(2000, 2, C.byref(tab)) == 1
    _, llr = sg.gen_llr(99, 0, 4096, ebn0_db=2.0, device="cuda")
    sg.decode(llr)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, raw, _ = sg.decode(llr)
    torch.cuda.synchronize()
    rate = sg.stats_from_device(raw)["ng"].sum() / (time.perf_counter() - t0)
    assert ceil.value > rate > 0


def test_host_entry_point_from_two_threads(cuda, sg):
    """sg_decode_host keeps its device buffers per device and serialises
    calls on one device: two threads decoding different inputs at the same
    time get exactly the results of one-at-a-time calls."""
    import threading

    ins = [sg.gen_llr(90 + k, 0, 40, ebn0_db=2.0)[1] for k in range(2)]
    want = [sg.decode(x) for x in ins]
    got = [None, None]

    def run(k):
        got[k] = sg.decode(ins[k])

    threads = [threading.Thread(target=run, args=(k,)) for k in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for k in range(2):
        assert np.array_equal(got[k][0], want[k][0]) and np.array_equal(got[k][1], want[k][1])
