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


def test_schedule_search(cuda, sg):
    from sogrand_b200.learn import schedule, search_schedules

    assert np.array_equal(schedule(0.7, 0.0, 10), np.full(30, 0.7))
    r = search_schedules(10, 1.5, 400, 4321, [0.6, 0.7], [0.0, 0.3], chunk=200)
    assert len(r["table"]) == 4
    ref = [t for t in r["table"] if t["a"] == 0.7 and t["b"] == 0.0][0]
    # the reference's own weights: the same decodes, a zero-width interval
    assert ref["ber"] == r["plain_ber"] and ref["ber_diff_vs_plain"] == 0 and ref["ci95"] == [0.0, 0.0]
    assert r["best"]["ber"] == min(t["ber"] for t in r["table"])


def test_schedule_search_two_points(cuda, sg):
    from sogrand_b200.learn import search_schedules_multi

    r = search_schedules_multi(10, [(1.5, 300), (2.0, 300)], 777, [0.7, 0.8], [0.0])
    assert len(r["runs"]) == 2 and all(len(run["table"]) == 2 for run in r["runs"])
    ref = [w for w in r["worst_relative_ber_change"] if w["a"] == 0.7][0]
    assert ref["worst"] == 0.0  # the reference's weights change nothing at any point
    assert r["best"]["worst_relative_ber_change"] == min(w["worst"] for w in r["worst_relative_ber_change"])
