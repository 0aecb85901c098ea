"""Code construction, encoder and seeded channel (host paths)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from oracle_api import Oracle


@pytest.fixture(scope="module")
def libm(oracle_paths):
    return Oracle(oracle_paths["libm"])


def test_encoder_matches_oracle(sg, libm):
    info = sg.gen_info(1, 0, 8)
    cw = sg.encode(info)
    for c in range(8):
        out = np.zeros(4096, np.uint8)
        libm.lib.sgo_encode(np.ascontiguousarray(np.unpackbits(info[c])), out)
        assert np.array_equal(out, cw[c])


def test_encoder_matches_reference_binary(sg, tmp_path):
    exe = os.path.join(ROOT, "oracle", "_ref", "cubic_encoder")
    if not os.path.exists(exe):
        pytest.skip("reference binaries are built only where the reference sources are")
    info = sg.gen_info(2, 0, 5)
    info.tofile(tmp_path / "i.bin")
    subprocess.run([exe, str(tmp_path / "i.bin"), str(tmp_path / "e.bin")], check=True, capture_output=True)
    e = np.unpackbits(np.fromfile(tmp_path / "e.bin", np.uint8)).reshape(5, 4096)
    assert np.array_equal(e, sg.encode(info))


def test_codewords_pass_early_termination(sg, libm):
    cw = sg.encode(sg.gen_info(3, 0, 4))
    for c in cw:
        lapp = np.ascontiguousarray(np.where(c == 0, 2.0, -2.0))
        assert libm.lib.sgo_early_termination(lapp) == 1


def test_sigma_matches_channel_sim(sg, libm):
    for eb in [1.0, 1.5, 2.0, 2.5, 3.0]:
        assert sg.channel_sigma(eb) == libm.lib.sgo_sigma(eb)
    assert abs(sg.channel_sigma(2.0) - 1.588656) < 1e-6


def test_generator_is_counter_based(sg):
    i1, l1 = sg.gen_llr(77, 0, 6, ebn0_db=2.0)
    i2, l2 = sg.gen_llr(77, 3, 3, ebn0_db=2.0)
    assert np.array_equal(l1[3:], l2) and np.array_equal(i1[3:], i2)
    _, l3 = sg.gen_llr(78, 0, 6, ebn0_db=2.0)
    assert not np.array_equal(l1, l3)


def test_generator_statistics(sg):
    info, llr = sg.gen_llr(5, 0, 40, ebn0_db=2.0)
    s = sg.channel_sigma(2.0)
    x = 1.0 - 2.0 * sg.encode(info).astype(np.float64)
    z = (llr * s * s / 2.0 - x) / s
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1.0) < 0.01
    assert abs(np.mean(np.unpackbits(info)) - 0.5) < 0.01


def test_mixed_snr_range(sg):
    _, llr = sg.gen_llr(5, 0, 64, ebn0_range=(1.0, 3.0))
    assert np.isfinite(llr).all()
    spread = [np.mean(np.abs(l)) for l in llr]
    assert max(spread) > 1.2 * min(spread)


def test_reference_arm_inputs_equal_library_generator(sg, tmp_path):
    """The CPU legs of bench.py write their LLR files with the oracle's build
    of the generator, so the process timing the reference never loads this
    library; the files must hold exactly the bench stream's codewords."""
    import bench

    files = bench.ref_inputs(str(tmp_path), 3)
    _, llr = sg.gen_llr(bench.SEED, 0, 3, ebn0_db=bench.EBN0)
    for c, f in enumerate(files):
        assert np.fromfile(f).tobytes() == llr[c].tobytes(), c
