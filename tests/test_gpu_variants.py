"""Every kernel configuration gives the same bits as the twin oracle."""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_all_variants_identical(cuda, sg, golden):
    """Every plain-kernel variant, through the device entry point (the host
    entry point runs the batched decoder)."""
    from sogrand_b200 import autotune

    torch = cuda
    e = golden["sets"]["snr_1.5dB"]
    _, llr = sg.gen_llr(e["seed"], 0, 12, ebn0_db=e["ebn0_db"])
    t = e["twin"]
    dllr = torch.from_numpy(llr).cuda()
    before = autotune.get_variant()
    try:
        for name in autotune.variants():
            autotune.set_variant(name)
            db, draw, dl = sg.decode(dllr, want_lapp=True)
            torch.cuda.synchronize()
            bits, stats, lapp = db.cpu().numpy(), sg.stats_from_device(draw), dl.cpu().numpy()
            for i in range(12):
                assert bits[i].tobytes().hex() == t["bits"][i], (name, i)
                assert int(stats["ng"][i]) == t["ng"][i], (name, i)
                assert stats["iterations"][i] == t["iterations"][i], (name, i)
                assert hashlib.sha256(lapp[i].tobytes()).hexdigest() == t["lapp_sha256"][i], (name, i)
    finally:
        autotune.set_variant(before)
