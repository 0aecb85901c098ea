"""Batched persistent decoder: bit-identical to the plain decoder and the
twin oracle for every variant; CUDA-graph capture and replay."""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["cfg1_2dB_100", "mixed_1to3dB", "snr_1.0dB"])
def test_batch_variants_match_twin(cuda, sg, golden, name):
    torch = cuda
    from sogrand_b200 import batch as B

    e = golden["sets"][name]
    snr = e["ebn0_db"]
    if isinstance(snr, list):
        _, llr = sg.gen_llr(e["seed"], 0, e["n_cw"], ebn0_range=tuple(snr))
    else:
        _, llr = sg.gen_llr(e["seed"], 0, e["n_cw"], ebn0_db=snr)
    d = torch.from_numpy(llr).cuda()
    t = e["twin"]
    b = B.Batch()
    before = B.get_variant()
    try:
        for v in B.variants():
            B.set_variant(v)
            bits, raw, lapp = b.decode(d, want_lapp=True)
            torch.cuda.synchronize()
            b.check()
            st = sg.stats_from_device(raw)
            bits = bits.cpu().numpy()
            lapp = lapp.cpu().numpy()
            for i in range(e["n_cw"]):
                assert bits[i].tobytes().hex() == t["bits"][i], (v, i)
                assert (st["iterations"][i], int(st["ng"][i]), int(st["ng_p"][i]), int(st["converged"][i])) == \
                    (t["iterations"][i], t["ng"][i], t["ng_p"][i], t["converged"][i]), (v, i)
                assert hashlib.sha256(lapp[i].tobytes()).hexdigest() == t["lapp_sha256"][i], (v, i)
    finally:
        B.set_variant(before)
        b.close()


def test_batch_equals_plain_at_scale_and_graph_replay(cuda, sg):
    torch = cuda
    from sogrand_b200 import batch as B

    _, llr = sg.gen_llr(77, 0, 3000, ebn0_range=(1.0, 3.0), device="cuda")
    pb, pr, _ = sg.decode(llr)
    b = B.Batch()
    bits, stats, _ = b.outputs(3000, llr.device)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        b.capture(llr, bits, stats, stream=stream.cuda_stream)
        for _ in range(2):
            bits.zero_()
            stats.zero_()
            b.replay(stream.cuda_stream)
            stream.synchronize()
            b.check()
            assert torch.equal(bits, pb) and torch.equal(stats, pr)
        # the graph reads the input buffer when replayed
        _, llr2 = sg.gen_llr(78, 0, 3000, ebn0_db=2.5, device="cuda")
        llr.copy_(llr2)
        b.replay(stream.cuda_stream)
        stream.synchronize()
    qb, qr, _ = sg.decode(llr2)
    assert torch.equal(bits, qb) and torch.equal(stats, qr)
    b.close()


def test_batch_small_and_nonfinite(cuda, sg):
    torch = cuda
    from sogrand_b200 import batch as B

    _, llr = sg.gen_llr(5, 0, 5, ebn0_db=2.0)
    llr[3, 7] = np.nan
    d = torch.from_numpy(llr).cuda()
    b = B.Batch()
    bits, raw, _ = b.decode(d)
    torch.cuda.synchronize()
    b.check()
    st = sg.stats_from_device(raw)
    assert st["converged"][3] == -1 and not bits[3].any()
    ok = [0, 1, 2, 4]
    pb, pr, _ = sg.decode(torch.from_numpy(llr[ok]).cuda())
    assert torch.equal(bits[ok], pb) and np.array_equal(st[ok], sg.stats_from_device(pr))
    e, _, _ = b.decode(torch.empty((0, 4096), dtype=torch.float64, device="cuda"))
    assert e.numel() == 0
    b.close()
