"""Device decode + reduction: the reference's averages and the comparator's
error counts computed on the GPU (SOGRAND_C/comparator.c:31-60)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _errs(bits, info):
    x = np.unpackbits(bits.reshape(-1, 64), axis=1) != np.unpackbits(info.reshape(-1, 64), axis=1)
    return int(x.sum()), int(x.any(axis=1).sum())


@pytest.mark.parametrize("name", ["cfg1_2dB_100", "snr_1.0dB"])
def test_summary_matches_per_codeword_results(cuda, sg, golden, name):
    torch = cuda
    e = golden["sets"][name]
    info, llr = sg.gen_llr(e["seed"], 0, e["n_cw"], ebn0_db=e["ebn0_db"])
    summ, bits = sg.decode_summary(torch.from_numpy(llr).cuda(), ref_info=torch.from_numpy(info).cuda(),
                                   want_bits=True)
    t = e["twin"]
    tbits = np.frombuffer(b"".join(bytes.fromhex(b) for b in t["bits"]), np.uint8)
    assert np.array_equal(bits.cpu().numpy().ravel(), tbits)
    be, ble = _errs(tbits, info)
    assert summ["blocks"] == e["n_cw"]
    assert summ["total_ng"] == sum(t["ng"]) and summ["total_ng_p"] == sum(t["ng_p"])
    assert summ["total_iterations"] == sum(t["iterations"])
    assert summ["converged"] == sum(1 for c in t["converged"] if c == 1)
    assert summ["bits_compared"] == 512 * e["n_cw"]
    assert (summ["bit_errors"], summ["block_errors"]) == (be, ble)
    if name == "snr_1.0dB":
        assert be > 0


def test_summary_without_reference_and_edge_cases(cuda, sg):
    torch = cuda
    _, llr = sg.gen_llr(3, 0, 5, ebn0_db=2.5)
    llr[2, 100] = np.inf
    summ, bits = sg.decode_summary(torch.from_numpy(llr).cuda())
    assert bits is None
    assert summ["blocks"] == 5 and summ["nonfinite"] == 1 and summ["bits_compared"] == 0
    empty, _ = sg.decode_summary(torch.empty((0, 4096), dtype=torch.float64, device="cuda"))
    assert all(v == 0 for v in empty.values())
