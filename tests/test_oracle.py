"""The CPU oracle pinned against the reference's golden vectors.

golden.json / kat_lines.npz were produced by the unmodified reference
(SOGRAND_C/cubic_decoder_final.c, compiled from its sources) by
tests/golden/make_golden.py; the libm build of the oracle must reproduce
them bit for bit, soft values included."""
import hashlib
import multiprocessing as mp

import numpy as np
import pytest

from oracle_api import UINT64_MAX, Oracle, twin_decode_one


@pytest.fixture(scope="module")
def libm(oracle_paths):
    return Oracle(oracle_paths["libm"])


@pytest.fixture(scope="module")
def twin(oracle_paths):
    return Oracle(oracle_paths["twin"])


@pytest.mark.parametrize("tag,L", [("L3", 3), ("L1", 1), ("L4", 4)])
def test_oracle_line_kats_bit_exact(libm, kat, tag, L):
    lapp, le, ng, _ = libm.bitso(kat["llr"], L=L)
    assert np.array_equal(ng, kat[f"{tag}_nguess"])
    assert np.array_equal(lapp.view(np.int64), kat[f"{tag}_lapp"].view(np.int64))
    assert np.array_equal(le.view(np.int64), kat[f"{tag}_le"].view(np.int64))


def test_twin_line_kats_discrete(twin, kat):
    lapp, le, ng, _ = twin.bitso(kat["llr"], L=3)
    assert np.array_equal(ng, kat["L3_nguess"])
    assert np.array_equal(lapp > 0, kat["L3_lapp"] > 0)
    assert np.abs(lapp - kat["L3_lapp"]).max() < 1e-6


def test_fixture_inputs_regenerate(sg, golden):
    for name, e in golden["sets"].items():
        snr = e["ebn0_db"]
        if isinstance(snr, list):
            info, llr = sg.gen_llr(e["seed"], 0, e["n_cw"], ebn0_range=tuple(snr))
        else:
            info, llr = sg.gen_llr(e["seed"], 0, e["n_cw"], ebn0_db=snr)
        assert hashlib.sha256(llr.tobytes()).hexdigest() == e["llr_sha256"], name
        assert hashlib.sha256(info.tobytes()).hexdigest() == e["info_sha256"], name


def test_oracle_codewords_match_reference(sg, golden, oracle_paths):
    """Whole decodes of config-1 codewords (100 cw at 2 dB), libm oracle vs
    the reference: bits, iterations, NG, NG_p and the final L_APP bytes."""
    e = golden["sets"]["cfg1_2dB_100"]
    _, llr = sg.gen_llr(e["seed"], 0, e["n_cw"], ebn0_db=e["ebn0_db"])
    idx = [0, 1, 2, 3, 63, 99]
    with mp.get_context("spawn").Pool(len(idx)) as pool:
        res = pool.map(twin_decode_one, [(oracle_paths["libm"], llr[i], {}) for i in idx])
    for i, (bits, st, lapp) in zip(idx, res):
        r = e["ref"]
        assert bits.tobytes().hex() == r["bits"][i]
        assert (st[0], st[1], st[2], st[3]) == (r["iterations"][i], r["ng"][i], r["ng_p"][i], r["converged"][i])
        assert hashlib.sha256(lapp.tobytes()).hexdigest() == r["lapp_sha256"][i]


def test_reference_vs_twin_differences_are_recorded(golden):
    """The twin (reference algorithm + the kernel's exp/log) differs from the
    reference only where glibc's exp/log round differently; the fixtures
    record exactly which codewords, and never in the decoded bits at 2 dB."""
    e = golden["sets"]["cfg1_2dB_100"]
    r, t = e["ref"], e["twin"]
    diff = [i for i in range(e["n_cw"]) if (r["ng"][i], r["iterations"][i]) != (t["ng"][i], t["iterations"][i])]
    assert len(diff) == e["ref_vs_twin_discrete_mismatches"] <= 2
    assert r["bits"] == t["bits"]


def test_early_termination_oracle(libm, sg):
    info = sg.gen_info(9, 0, 1)
    cw = sg.encode(info)[0]
    lapp = np.where(cw == 0, 1.0, -1.0)
    assert libm.lib.sgo_early_termination(np.ascontiguousarray(lapp)) == 1
    lapp[1234] = -lapp[1234]
    assert libm.lib.sgo_early_termination(np.ascontiguousarray(lapp)) == 0
