"""Evaluation of learned weights (sogrand_b200.learn): every decoder sees the
same codewords, and BER differences come with a paired interval."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_paired_evaluation(cuda, sg):
    from sogrand_b200.learn import evaluate_set

    a = np.full(90, 0.7)
    configs = {"plain30": (None, 30), "same": (a, 30), "plain5": (None, 5)}
    out = evaluate_set(configs, 1.5, 600, 777, 0, chunk=256, pairs=[("same", "plain30"), ("plain5", "plain30")])
    c = out["configs"]
    # weights equal to the reference's: identical decodes, a zero-width interval
    assert c["same"]["bit_errors"] == c["plain30"]["bit_errors"]
    same = out["paired"][0]
    assert same["ber_diff"] == 0 and same["ci95"] == [0.0, 0.0]
    # totals agree with the device summary of the same codewords
    info, llr = sg.gen_llr(777, 0, 600, ebn0_db=1.5, device="cuda")
    s, _ = sg.decode_summary(llr, sg.params(Imax=5), ref_info=info)
    assert c["plain5"]["bit_errors"] == s["bit_errors"] and c["plain5"]["block_errors"] == s["block_errors"]
    assert c["plain5"]["avg_iterations"] == s["total_iterations"] / 600
    d = out["paired"][1]
    assert d["ber_diff"] == pytest.approx((c["plain5"]["bit_errors"] - c["plain30"]["bit_errors"]) / (600 * 512))
    assert d["ci95"][0] <= d["ber_diff"] <= d["ci95"][1]
